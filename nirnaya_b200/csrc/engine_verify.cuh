// Host side of the device solution check (nir_pdhg_verify,
// nir_pdhg_batch_verify; include/nir_pdhg.h).  Included at the end of
// engine.cu.  The check reads the handle's resident LP as given:
//   - the row-major copy of A with the original values (A.v_orig, each
//     row's entries in ascending column order, the transpose's stable
//     sort);
//   - the original cost and the bounds sanitised to +-inf, which the
//     reference's is_finite_bound test treats like the raw bounds.
// The kernels are in k_verify.cuh.
#pragma once

namespace {

void verify_buffers(nir_pdhg* h, int count) {
    auto& v = h->vfy;
    if (v.ready) {
        // the per-instance arrays were sized by the first call
        if (count > v.count)
            throw std::invalid_argument("a check of " + std::to_string(count) + " instances on a handle whose check buffers hold " +
                                        std::to_string(v.count));
        return;
    }
    v.count = count;
    v.x = h->alloc<double>(h->n);
    v.vt = h->alloc<int8_t>(h->n);
    v.rv = h->alloc<double>(h->m);
    v.rs = h->alloc<int8_t>(h->m);
    v.obj = h->alloc<double>(count);
    v.claimed = h->alloc<double>(count);
    v.offset = h->alloc<double>(count);
    v.fb = h->alloc<long long>(count);
    v.b = h->alloc<nir::vfy::Rec>(count);
    v.g = h->alloc<nir::vfy::Rec>(count);
    v.rep = h->alloc<nir_verify_report>(count);
    v.row_off = h->alloc<int>(2);
    v.col_off = h->alloc<int>(2);
    const int ro[2] = {0, h->m}, co[2] = {0, h->n};
    h2d(h, v.row_off, ro, sizeof(ro));
    h2d(h, v.col_off, co, sizeof(co));
    v.ready = true;
}

// count instances laid out by d_row_off / d_col_off (count + 1 entries on
// the device) and d_row_inst (the instance of every row; null for one
// instance).  d_x: the points on the device.  vt_host, claimed_host may be
// null.
void verify_impl(nir_pdhg* h, int count, const int* d_row_off, const int* d_col_off, const int* d_row_inst,
                 const double* offsets, const double* d_x, const int8_t* vt_host, const double* claimed_host,
                 double tol, nir_verify_report* out) {
    verify_buffers(h, count);
    auto& v = h->vfy;
    cudaStream_t s = h->stream;
    const int8_t* d_vt = nullptr;
    if (vt_host && h->n > 0) {
        NIR_CUDA(cudaMemcpyAsync(v.vt, vt_host, size_t(h->n), cudaMemcpyHostToDevice, s));
        d_vt = v.vt;
    }
    std::vector<double> claimed(size_t(count), std::numeric_limits<double>::quiet_NaN());
    if (claimed_host) claimed.assign(claimed_host, claimed_host + count);
    NIR_CUDA(cudaMemcpyAsync(v.claimed, claimed.data(), size_t(count) * sizeof(double), cudaMemcpyHostToDevice, s));
    NIR_CUDA(cudaMemcpyAsync(v.offset, offsets, size_t(count) * sizeof(double), cudaMemcpyHostToDevice, s));
    auto* b = static_cast<nir::vfy::Rec*>(v.b);
    auto* g = static_cast<nir::vfy::Rec*>(v.g);
    nir::vfy::k_vfy_cols<<<count, nir::vfy::kVfyBlock, 0, s>>>(d_col_off, d_x, h->l, h->u, d_vt, v.fb, b, g);
    NIR_LAUNCHED();
    const long long threads = (long long)count + h->m;
    const unsigned grid = unsigned((threads + nir::vfy::kVfyBlock - 1) / nir::vfy::kVfyBlock);
    nir::vfy::k_vfy_rows<<<grid, nir::vfy::kVfyBlock, 0, s>>>(count, h->m, d_row_off, d_col_off, d_row_inst, h->A.rp,
                                                              h->A.ci, h->A.v_orig, d_x, h->rl, h->ru, h->c, v.offset,
                                                              v.fb, h->d_row_orig, v.rv, v.rs, v.obj);
    NIR_LAUNCHED();
    nir::vfy::k_vfy_report<<<count, nir::vfy::kVfyBlock, 0, s>>>(d_row_off, d_col_off, v.rv, v.rs, v.fb, b, g, v.obj,
                                                                 v.claimed, tol, v.rep);
    NIR_LAUNCHED();
    h->launches += 3;
    // the host vectors above stay alive until this synchronous copy ends
    d2h(h, out, v.rep, size_t(count) * sizeof(nir_verify_report));
}

}  // namespace

extern "C" {

int nir_pdhg_verify(nir_pdhg* h, const double* x, const int8_t* vartype, double claimed_obj, double tol,
                    nir_verify_report* out) {
    if (!h || !out) {
        g_err = !h ? "null handle" : "null report";
        return NIR_STATUS_INPUT_ERROR;
    }
    if (!x && !h->last_x) {
        g_err = "no point given and no solve has returned one";
        return NIR_STATUS_INPUT_ERROR;
    }
    try {
        NIR_CUDA(cudaSetDevice(h->device));
        verify_buffers(h, 1);
        const double* d_x = h->last_x;
        if (x) {
            if (h->n > 0)
                NIR_CUDA(cudaMemcpyAsync(h->vfy.x, x, size_t(h->n) * sizeof(double), cudaMemcpyHostToDevice, h->stream));
            d_x = h->vfy.x;
        }
        verify_impl(h, 1, h->vfy.row_off, h->vfy.col_off, nullptr, &h->offset, d_x, vartype, &claimed_obj, tol, out);
        return 0;
    } catch (const std::invalid_argument& e) {
        g_err = e.what();
        return NIR_STATUS_INPUT_ERROR;
    } catch (const std::exception& e) {
        g_err = e.what();
        return NIR_STATUS_INTERNAL_ERROR;
    }
}

int nir_pdhg_batch_verify(nir_pdhg_batch* b, const double* x, const int8_t* vartype, const double* claimed_obj,
                          double tol, nir_verify_report* out) {
    if (!b || !b->h || !out) {
        g_err = !out ? "null report" : "null handle";
        return NIR_STATUS_INPUT_ERROR;
    }
    if (!x && !b->solved) {
        g_err = "no point given and no batch solve has returned one";
        return NIR_STATUS_INPUT_ERROR;
    }
    nir_pdhg* h = b->h;
    try {
        NIR_CUDA(cudaSetDevice(h->device));
        verify_buffers(h, b->count);
        const double* d_x = h->out_x;
        if (x) {
            if (h->n > 0)
                NIR_CUDA(cudaMemcpyAsync(h->vfy.x, x, size_t(h->n) * sizeof(double), cudaMemcpyHostToDevice, h->stream));
            d_x = h->vfy.x;
        }
        verify_impl(h, b->count, b->d_row_off, b->d_col_off, b->d_row_inst, b->offsets.data(), d_x, vartype,
                    claimed_obj, tol, out);
        return 0;
    } catch (const std::invalid_argument& e) {
        g_err = e.what();
        return NIR_STATUS_INPUT_ERROR;
    } catch (const std::exception& e) {
        g_err = e.what();
        return NIR_STATUS_INTERNAL_ERROR;
    }
}

}  // extern "C"
