// Host side of the batched solve (nir_pdhg_batch_*, include/nir_pdhg.h).
// Included at the end of engine.cu: it reuses the single-LP handle (device
// transpose, preconditioning, launch chunks, status snapshots) for the
// block-diagonal layout of the batch, with the kernels of k_batch.cuh.
#pragma once

struct nir_pdhg_batch {
    nir_pdhg* h = nullptr;                        // the block-diagonal LP
    int count = 0;
    std::vector<int> row_off, col_off;            // count + 1
    std::vector<double> offsets;                  // objective offsets
    int* d_row_off = nullptr;
    int* d_col_off = nullptr;
    int* d_row_inst = nullptr;
    int* d_col_inst = nullptr;
    // the blocks of each orientation, instance by instance (no block crosses
    // an instance), in the layout the autotuner picked for it, one set per
    // layout choice used, built once each
    struct Orient2 {
        int lay = nir::kLayWarp;
        int cap = 256;          // warp row-block capacity
        void* blk = nullptr;    // int2 (warp) or int4 with the instance in .w (CTA)
        int nblk = 0;
        int* lo = nullptr;      // first block of each instance (count + 1)
        int* ci = nullptr;      // CTA layout: padded column indices (warp: the CSR's)
        double* v64 = nullptr;  // CTA layout: padded scaled values (warp: the CSR's)
        float* v32 = nullptr;
    };
    struct Layout {
        LayChoice choice;
        Orient2 a, at;          // A (rows) and A' (columns)
        double* part = nullptr;
    };
    std::deque<Layout> layouts;
    Layout* cur = nullptr;
    nir::DevState* insts = nullptr;
    // the running instances and their block prefixes (k_bcompact)
    int *d_act_inst = nullptr, *d_act_off_a = nullptr, *d_act_off_at = nullptr, *d_act_n = nullptr;
    double *d_bnorm = nullptr, *d_cnorm = nullptr, *d_offset = nullptr, *d_norm = nullptr;
    ChunkGraph graphs[2];
    bool solved = false;  // h->out_x holds the points the last batch solve returned
    ~nir_pdhg_batch() {
        if (h && h->device >= 0) cudaSetDevice(h->device);
        for (auto& g : graphs) {
            if (g.ge) cudaGraphExecDestroy(g.ge);
            if (g.g) cudaGraphDestroy(g.g);
        }
        delete h;  // frees every device buffer allocated through it
    }
};

namespace {

// The blocks of one orientation in layout `lay`, built instance by
// instance so that no block crosses an instance; the CTA layout also gets
// the padded stream of its column indices (values are padded after each
// preconditioning, batch_pad_values).
void batch_blocks(nir_pdhg_batch* B, Orient& o, const std::vector<int>& off, int lay, int cap,
                  nir_pdhg_batch::Orient2* out) {
    nir_pdhg* h = B->h;
    std::vector<int> lo;
    out->lay = lay;
    out->cap = cap;
    if (lay == nir::kLayWarp) {
        std::vector<int> owner;
        const std::vector<int2> all = nir::build_batch_row_blocks(o.h_rp, off, cap, &owner, &lo);
        out->nblk = int(owner.size());
        int2* blk = h->alloc<int2>(all.size());
        h2d(h, blk, all.data(), all.size() * sizeof(int2));
        out->blk = blk;
        out->ci = o.ci;
        out->v64 = o.v64;
        out->v32 = o.v32;
    } else {
        const std::vector<int4> all = nir::build_batch_cta_blocks(o.h_rp, off, cap, &lo);
        out->nblk = int(all.size()) - 1;
        int4* blk = h->alloc<int4>(all.size());
        h2d(h, blk, all.data(), all.size() * sizeof(int4));
        out->blk = blk;
        const size_t q = size_t(all.back().z);
        out->ci = h->allocz<int>(q, 8);
        out->v64 = h->allocz<double>(q, 8);
        out->v32 = h->allocz<float>(q, 8);
        if (out->nblk > 0 && o.nnz > 0) {
            const unsigned g = unsigned(std::max(1, std::min(out->nblk, 4 * h->sms)));
            nir::k_pad_stream<double><<<g, nir::kBlock, 0, h->stream>>>(blk, out->nblk, o.ci, o.v_orig, out->ci,
                                                                        out->v64);
            NIR_LAUNCHED();
        }
    }
    out->lo = h->alloc<int>(lo.size());
    h2d(h, out->lo, lo.data(), lo.size() * sizeof(int));
    NIR_CUDA(cudaStreamSynchronize(h->stream));
}

// The scaled values (written by precondition) into the padded streams of
// the orientations that use the CTA layout.
void batch_pad_values(nir_pdhg_batch* B) {
    nir_pdhg* h = B->h;
    for (int t = 0; t < 2; ++t) {
        const nir_pdhg_batch::Orient2& L = t ? B->cur->at : B->cur->a;
        const Orient& o = t ? h->At : h->A;
        if (L.lay != nir::kLayCta || L.nblk <= 0 || o.nnz <= 0) continue;
        const int4* blk = static_cast<const int4*>(L.blk);
        const unsigned g = unsigned(std::max(1, std::min(L.nblk, 4 * h->sms)));
        nir::k_pad_stream<double><<<g, nir::kBlock, 0, h->stream>>>(blk, L.nblk, o.ci, o.v64, nullptr, L.v64);
        nir::k_pad_stream<float><<<g, nir::kBlock, 0, h->stream>>>(blk, L.nblk, o.ci, o.v32, nullptr, L.v32);
        NIR_LAUNCHED();
    }
}

template <typename TV>
const TV* bvals(const nir_pdhg_batch::Orient2& L);
template <>
const float* bvals<float>(const nir_pdhg_batch::Orient2& L) {
    return L.v32;
}
template <>
const double* bvals<double>(const nir_pdhg_batch::Orient2& L) {
    return L.v64;
}

nir::BatchArgs bargs(nir_pdhg_batch* B, bool transpose, double* part, int i, int halpern, int phase, double rho) {
    nir_pdhg* h = B->h;
    const Orient& o = transpose ? h->At : h->A;
    const nir_pdhg_batch::Orient2& L = transpose ? B->cur->at : B->cur->a;
    return nir::BatchArgs{nir::Lay{L.blk, L.nblk, L.cap, o.rp, L.ci},
                          part,
                          B->insts,
                          i,
                          halpern,
                          phase,
                          rho,
                          L.lo,
                          B->d_act_inst,
                          transpose ? B->d_act_off_at : B->d_act_off_a,
                          B->d_act_n};
}

// Lists the running instances and their block prefixes for the layouts in
// use (after the states are set, and after every check).
void launch_bcompact(nir_pdhg_batch* B) {
    nir_pdhg* h = B->h;
    nir::k_bcompact<<<1, nir::kBlock, 0, h->stream>>>(B->count, B->insts, B->cur->a.lo, B->cur->at.lo, B->d_act_inst,
                                                      B->d_act_off_a, B->d_act_off_at, B->d_act_n);
    NIR_LAUNCHED();
    h->launches += 1;
}

// Calls f(LP, LD) with the batch layouts of A' and A.
template <class F>
void with_batch_lays(const nir_pdhg_batch* B, F&& f) {
    using W = std::integral_constant<int, nir::kLayWarp>;
    using Cc = std::integral_constant<int, nir::kLayCta>;
    const bool pc = B->cur->at.lay == nir::kLayCta, dc = B->cur->a.lay == nir::kLayCta;
    if (pc && dc) f(Cc{}, Cc{});
    else if (pc) f(Cc{}, W{});
    else if (dc) f(W{}, Cc{});
    else f(W{}, W{});
}

// One launch chunk of the batch; TV = value type, TX = iterate type, LP /
// LD = layouts of A' / A.
template <typename TV, typename TX, int LP, int LD>
void launch_batch_chunk_l(nir_pdhg_batch* B, const SolveCfg& cfg, int phase) {
    nir_pdhg* h = B->h;
    cudaStream_t s = h->stream;
    const int K = cfg.K;
    const nir_pdhg_batch::Orient2& LA = B->cur->a;
    const nir_pdhg_batch::Orient2& LT = B->cur->at;
    double* P = B->cur->part;
    double* D = P + 2 * size_t(std::max(LT.nblk, 1));
    double* KR = D + 2 * size_t(std::max(LA.nblk, 1));
    double* KC = KR + 4 * size_t(std::max(LA.nblk, 1));
    const size_t sp = lay_smem<LP, TX>(), sd = lay_smem<LD, TX>();
    const int gp1 = lay_grid<LP, TX>(h, nir::k_bprimal<LP, TV, TX, true>, LT.nblk);
    const int gp0 = lay_grid<LP, TX>(h, nir::k_bprimal<LP, TV, TX, false>, LT.nblk);
    const int gd1 = lay_grid<LD, TX>(h, nir::k_bdual<LD, TV, TX, true>, LA.nblk);
    const int gd0 = lay_grid<LD, TX>(h, nir::k_bdual<LD, TV, TX, false>, LA.nblk);
    const int gkr = lay_grid<LD, double>(h, nir::k_bkkt_rows<LD, TX>, LA.nblk);
    const int gkc = lay_grid<LP, double>(h, nir::k_bkkt_cols<LP, TX>, LT.nblk);
    int i_first = 0;
    if (cfg.persistent && K > 1) {
        // iterations 0..K-2 in one cooperative launch; the check pair below
        const int gc = std::min(lay_grid<LP, TX>(h, nir::k_bchunk<LP, LD, TV, TX>, LT.nblk),
                                lay_grid<LD, TX>(h, nir::k_bchunk<LP, LD, TV, TX>, LA.nblk));
        nir::BatchArgs ap = bargs(B, true, P, 0, cfg.halpern, phase, cfg.p.reflection);
        nir::BatchArgs ad = bargs(B, false, D, 0, cfg.halpern, phase, cfg.p.reflection);
        nir::ChunkPtrs<TV, TX> v{bvals<TV>(LT),  bvals<TV>(LA),  Vec<TX>::x(h),  Vec<TX>::xb(h), Vec<TX>::xp(h),
                                 Vec<TX>::y(h),  Vec<TX>::yp(h), Vec<TX>::c(h),  Vec<TX>::l(h),  Vec<TX>::u(h),
                                 Vec<TX>::x0(h), Vec<TX>::rl(h), Vec<TX>::ru(h), Vec<TX>::y0(h)};
        nir::GridSync gs{h->gs_count, h->gs_gen, h->gs_err, unsigned(gc) + (cfg.barrier_test ? 1u : 0u),
                         cfg.barrier_test ? 200000000LL : 2000000000LL};
        nir::DevState* insts = B->insts;
        int i0 = 0, iters = K - 1, count = B->count;
        void* args[] = {&ap, &ad, &v, &i0, &iters, &gs, &insts, &count};
        NIR_CUDA(cudaLaunchCooperativeKernel((const void*)nir::k_bchunk<LP, LD, TV, TX>, dim3(gc), dim3(nir::kBlock),
                                             args, std::max(sp, sd), s));
        h->launches += 1;
        i_first = K - 1;
    }
    for (int i = i_first; i < K; ++i) {
        const bool check = (i == K - 1);
        nir::BatchArgs ap = bargs(B, true, P, i, cfg.halpern, phase, cfg.p.reflection);
        nir::BatchArgs ad = bargs(B, false, D, i, cfg.halpern, phase, cfg.p.reflection);
        if (check)
            nir::k_bprimal<LP, TV, TX, true><<<gp1, nir::kBlock, sp, s>>>(
                ap, bvals<TV>(LT), Vec<TX>::y(h), Vec<TX>::x(h), Vec<TX>::xb(h), Vec<TX>::xp(h), Vec<TX>::c(h),
                Vec<TX>::l(h), Vec<TX>::u(h), Vec<TX>::x0(h));
        else
            nir::k_bprimal<LP, TV, TX, false><<<gp0, nir::kBlock, sp, s>>>(
                ap, bvals<TV>(LT), Vec<TX>::y(h), Vec<TX>::x(h), Vec<TX>::xb(h), Vec<TX>::xp(h), Vec<TX>::c(h),
                Vec<TX>::l(h), Vec<TX>::u(h), Vec<TX>::x0(h));
        NIR_LAUNCHED();
        if (check)
            nir::k_bdual<LD, TV, TX, true><<<gd1, nir::kBlock, sd, s>>>(ad, bvals<TV>(LA), Vec<TX>::xb(h),
                                                                        Vec<TX>::y(h), Vec<TX>::yp(h), Vec<TX>::rl(h),
                                                                        Vec<TX>::ru(h), Vec<TX>::y0(h));
        else
            nir::k_bdual<LD, TV, TX, false><<<gd0, nir::kBlock, sd, s>>>(ad, bvals<TV>(LA), Vec<TX>::xb(h),
                                                                         Vec<TX>::y(h), Vec<TX>::yp(h), Vec<TX>::rl(h),
                                                                         Vec<TX>::ru(h), Vec<TX>::y0(h));
        NIR_LAUNCHED();
        h->launches += 2;
    }
    nir::BatchArgs kr = bargs(B, false, KR, 0, 0, phase, 0.0);
    nir::k_bkkt_rows<LD, TX><<<gkr, nir::kBlock, lay_smem<LD, double>(), s>>>(kr, LA.v64, Vec<TX>::xp(h),
                                                                             Vec<TX>::yp(h), h->dr, h->rl, h->ru);
    nir::BatchArgs kc = bargs(B, true, KC, 0, 0, phase, 0.0);
    nir::k_bkkt_cols<LP, TX><<<gkc, nir::kBlock, lay_smem<LP, double>(), s>>>(kc, LT.v64, Vec<TX>::xp(h),
                                                                             Vec<TX>::yp(h), h->dc, h->c, h->l, h->u);
    NIR_LAUNCHED();
    nir::CtlArgs ca{};
    ca.K = K;
    ca.tol = cfg.p.tol;
    ca.feas_tol = cfg.p.feas_tol;
    ca.restarts_on = cfg.restarts;
    ca.mixed = (cfg.mixed && phase == 0) ? 1 : 0;
    ca.phase = phase;
    ca.suff = cfg.p.restart_sufficient;
    ca.nec = cfg.p.restart_necessary;
    ca.art = cfg.p.restart_artificial;
    ca.theta = cfg.p.primal_weight_smoothing;
    ca.polish_stall = cfg.p.polish_stall_checks;
    ca.polish_switch = cfg.p.polish_switch_kkt;
    ca.anchor_at_restart = cfg.p.restart_anchor ? 1 : 0;
    ca.weight_decades = cfg.p.primal_weight_decades;
    ca.hist = nullptr;
    nir::BatchCtlArgs cb{P, D, KR, KC, LT.nblk, LA.nblk, LT.lo, LA.lo, B->d_bnorm, B->d_cnorm, B->d_offset};
    nir::k_bcontrol<<<B->count, nir::kBlock, 0, s>>>(ca, cb, B->insts);
    nir::k_bapply_restart<TX><<<grid_for(std::max(h->n, h->m)), nir::kBlock, 0, s>>>(
        h->n, h->m, B->d_col_inst, B->d_row_inst, B->insts, phase, Vec<TX>::x(h), Vec<TX>::x0(h), Vec<TX>::xp(h),
        Vec<TX>::y(h), Vec<TX>::y0(h), Vec<TX>::yp(h));
    launch_bcompact(B);  // the next chunk visits the blocks of the instances still running
    nir::k_bsnap<<<1, nir::kBlock, 0, s>>>(B->count, B->insts, h->snap.ring, h->snap.d_seq);
    NIR_LAUNCHED();
    h->launches += 7;
}

template <typename TV, typename TX>
void launch_batch_chunk(nir_pdhg_batch* B, const SolveCfg& cfg, int phase) {
    with_batch_lays(B, [&](auto lp, auto ld) {
        launch_batch_chunk_l<TV, TX, decltype(lp)::value, decltype(ld)::value>(B, cfg, phase);
    });
}

template <typename TV, typename TX>
void warm_batch_cfgs(nir_pdhg_batch* B) {
    nir_pdhg* h = B->h;
    with_batch_lays(B, [&](auto lp, auto ld) {
        constexpr int LP = decltype(lp)::value, LD = decltype(ld)::value;
        const int na = B->cur->a.nblk, nt = B->cur->at.nblk;
        lay_grid<LP, TX>(h, nir::k_bprimal<LP, TV, TX, true>, nt);
        lay_grid<LP, TX>(h, nir::k_bprimal<LP, TV, TX, false>, nt);
        lay_grid<LD, TX>(h, nir::k_bdual<LD, TV, TX, true>, na);
        lay_grid<LD, TX>(h, nir::k_bdual<LD, TV, TX, false>, na);
        lay_grid<LD, double>(h, nir::k_bkkt_rows<LD, TX>, na);
        lay_grid<LP, double>(h, nir::k_bkkt_cols<LP, TX>, nt);
        lay_grid<LP, TX>(h, nir::k_bchunk<LP, LD, TV, TX>, nt);
        lay_grid<LD, TX>(h, nir::k_bchunk<LP, LD, TV, TX>, na);
    });
}

void batch_create_impl(nir_pdhg_batch* B, const nir_lp_view* lps, int count, int device) {
    B->count = count;
    long long m = 0, n = 0, nnz = 0;
    B->row_off.push_back(0);
    B->col_off.push_back(0);
    for (int i = 0; i < count; ++i) {
        validate_lp(&lps[i]);
        m += lps[i].nrow;
        n += lps[i].ncol;
        nnz += lps[i].nnz;
        if (m >= (1LL << 31) - 1 || n >= (1LL << 31) - 1 || nnz >= (1LL << 31) - 1)
            throw std::invalid_argument("batch too large for 32-bit indices");
        B->row_off.push_back(int(m));
        B->col_off.push_back(int(n));
        B->offsets.push_back(lps[i].obj_offset);
    }
    std::vector<int64_t> start(n + 1, 0);
    std::vector<int> index(nnz);
    std::vector<double> value(nnz), cost(n), lo(n), up(n), rlo(m), rup(m);
    long long k = 0;
    for (int i = 0; i < count; ++i) {
        const nir_lp_view& v = lps[i];
        const int c0 = B->col_off[i], r0 = B->row_off[i];
        for (int j = 0; j < v.ncol; ++j) {
            for (long long q = v.col_start[j]; q < v.col_start[j + 1]; ++q) {
                index[k] = v.row_index[q] + r0;
                value[k] = v.value[q];
                ++k;
            }
            start[c0 + j + 1] = k;
            cost[c0 + j] = v.cost[j];
            lo[c0 + j] = v.collo[j];
            up[c0 + j] = v.colup[j];
        }
        for (int r = 0; r < v.nrow; ++r) {
            rlo[r0 + r] = v.rowlo[r];
            rup[r0 + r] = v.rowup[r];
        }
    }
    nir_lp_view all{};
    all.nrow = int(m);
    all.ncol = int(n);
    all.nnz = nnz;
    all.col_start = start.data();
    all.row_index = index.data();
    all.value = value.data();
    all.cost = cost.data();
    all.collo = lo.data();
    all.colup = up.data();
    all.rowlo = rlo.data();
    all.rowup = rup.data();
    B->h = new nir_pdhg();
    B->h->device = -1;
    create_impl(B->h, &all, device);
    nir_pdhg* h = B->h;
    std::vector<int> row_inst(m), col_inst(n);
    for (int i = 0; i < count; ++i) {
        for (int r = B->row_off[i]; r < B->row_off[i + 1]; ++r) row_inst[r] = i;
        for (int j = B->col_off[i]; j < B->col_off[i + 1]; ++j) col_inst[j] = i;
    }
    B->d_row_inst = h->alloc<int>(m);
    B->d_col_inst = h->alloc<int>(n);
    if (m) h2d(h, B->d_row_inst, row_inst.data(), m * sizeof(int));
    if (n) h2d(h, B->d_col_inst, col_inst.data(), n * sizeof(int));
    B->d_row_off = h->alloc<int>(count + 1);
    B->d_col_off = h->alloc<int>(count + 1);
    h2d(h, B->d_row_off, B->row_off.data(), (count + 1) * sizeof(int));
    h2d(h, B->d_col_off, B->col_off.data(), (count + 1) * sizeof(int));
    B->insts = h->alloc<nir::DevState>(count);
    B->d_act_inst = h->alloc<int>(count);
    B->d_act_off_a = h->alloc<int>(size_t(count) + 1);
    B->d_act_off_at = h->alloc<int>(size_t(count) + 1);
    B->d_act_n = h->alloc<int>(1);
    B->d_bnorm = h->alloc<double>(count);
    B->d_cnorm = h->alloc<double>(count);
    B->d_offset = h->alloc<double>(count);
    B->d_norm = h->alloc<double>(count);
}

int batch_solve_impl(nir_pdhg_batch* B, const nir_pdhg_params& p, int (*poll)(void*), void* ctx, double* x_out,
                     double* y_out, nir_pdhg_info* infos, nir_pdhg_info* total) {
    nir_pdhg* h = B->h;
    cudaStream_t s = h->stream;
    const double t0 = now_sec();
    const int n = h->n, m = h->m, I = B->count;
    B->solved = false;  // out_x serves as scratch until the final unscale
    if (p.algorithm != NIR_ALGO_PDLP) throw std::invalid_argument("the batch runs NIR_ALGO_PDLP only");
    if (p.check_every < 1 || p.reflection < 0.0 || p.reflection > 1.0 || !(p.tol >= 0.0))
        throw std::invalid_argument("invalid parameters");
    // layouts timed on the block-diagonal matrix, then built per instance
    const LayChoice lc = pick_layouts(h, p);
    auto same = [](const LayChoice& a, const LayChoice& b) {
        return a.lay_a == b.lay_a && a.cap_a == b.cap_a && a.lay_at == b.lay_at && a.cap_at == b.cap_at;
    };
    if (!B->cur || !same(B->cur->choice, lc)) {
        B->cur = nullptr;
        for (auto& l : B->layouts)
            if (same(l.choice, lc)) B->cur = &l;
        if (!B->cur) {
            B->layouts.emplace_back();
            nir_pdhg_batch::Layout& l = B->layouts.back();
            l.choice = lc;
            batch_blocks(B, h->A, B->row_off, lc.lay_a, lc.lay_a == nir::kLayCta ? kCtaCap : lc.cap_a, &l.a);
            batch_blocks(B, h->At, B->col_off, lc.lay_at, lc.lay_at == nir::kLayCta ? kCtaCap : lc.cap_at, &l.at);
            l.part = h->alloc<double>(6 * size_t(std::max(l.a.nblk, 1)) + 6 * size_t(std::max(l.at.nblk, 1)));
            B->cur = &l;
        }
    }
    SolveCfg cfg;
    cfg.p = p;
    cfg.K = p.check_every;
    cfg.halpern = 1;
    cfg.restarts = 1;
    cfg.mixed = (p.precision == NIR_PREC_MIXED) ? 1 : 0;
    {
        // persistent chunks on request, as for one LP
        int coop = 0;
        NIR_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, h->device));
        const bool want = p.persistent == 1 || p.persistent == 2;
        if (want && !coop) throw std::invalid_argument("persistent chunks need cooperative launch support");
        cfg.persistent = want ? 1 : 0;
        cfg.barrier_test = (want && p.persistent == 2) ? 1 : 0;
        if (cfg.persistent) {
            NIR_CUDA(cudaMemsetAsync(h->gs_count, 0, sizeof(unsigned), s));
            NIR_CUDA(cudaMemsetAsync(h->gs_gen, 0, sizeof(unsigned), s));
            NIR_CUDA(cudaMemsetAsync(h->gs_err, 0, sizeof(int), s));
        }
    }
    precondition(h, p, p.ruiz_iters > 0 || p.pock_chambolle);
    batch_pad_values(B);
    // per-instance ||A_i||_2 by power iteration on the block-diagonal matrix
    const unsigned gwm = grid_for((long long)m * 32), gwn = grid_for((long long)n * 32);
    nir::k_power_start_batch<<<grid_for(n), nir::kBlock, 0, s>>>(n, B->d_col_inst, B->d_col_off, h->tmp_n);
    nir::k_seg_norm<<<I, nir::kBlock, 0, s>>>(B->d_col_off, h->tmp_n, B->d_norm);
    nir::k_seg_scale<<<grid_for(n), nir::kBlock, 0, s>>>(n, B->d_col_inst, B->d_norm, h->tmp_n);
    for (int r = 0; r < std::max(1, p.power_iters); ++r) {
        nir::k_spmv_warp64<<<gwm, nir::kBlock, 0, s>>>(m, h->A.rp, h->A.ci, h->A.v64, h->tmp_n, h->tmp_m);
        nir::k_spmv_warp64<<<gwn, nir::kBlock, 0, s>>>(n, h->At.rp, h->At.ci, h->At.v64, h->tmp_m, h->tmp_n);
        nir::k_seg_norm<<<I, nir::kBlock, 0, s>>>(B->d_col_off, h->tmp_n, B->d_norm);
        nir::k_seg_scale<<<grid_for(n), nir::kBlock, 0, s>>>(n, B->d_col_inst, B->d_norm, h->tmp_n);
    }
    NIR_LAUNCHED();
    std::vector<double> nrm(I), dc(n), dr(m);
    d2h(h, nrm.data(), B->d_norm, I * sizeof(double));
    d2h(h, dc.data(), h->dc, n * sizeof(double));
    d2h(h, dr.data(), h->dr, m * sizeof(double));
    std::vector<nir::DevState> st0(I);
    std::vector<double> bn(I), cn(I);
    for (int i = 0; i < I; ++i) {
        DD cs, bs, co, bo;
        for (int j = B->col_off[i]; j < B->col_off[i + 1]; ++j) {
            cs = dd_add_prod(cs, h->h_c[j] * dc[j], h->h_c[j] * dc[j]);
            co = dd_add_prod(co, h->h_c[j], h->h_c[j]);
        }
        for (int r = B->row_off[i]; r < B->row_off[i + 1]; ++r) {
            double b = 0.0;
            if (std::isfinite(h->h_rl[r])) b = std::fabs(h->h_rl[r]);
            if (std::isfinite(h->h_ru[r])) b = std::max(b, std::fabs(h->h_ru[r]));
            bo = dd_add_prod(bo, b, b);
            bs = dd_add_prod(bs, b * dr[r], b * dr[r]);
        }
        const double csn = std::sqrt(cs.hi + cs.lo), bsn = std::sqrt(bs.hi + bs.lo);
        const double sig = std::sqrt(nrm[i]);
        nir::DevState& d = st0[i];
        d = nir::DevState{};
        d.max_iters = p.max_iters;
        d.best_kkt = INFINITY;
        d.eta = p.step_factor / std::max(sig, 1e-30);
        d.omega = (csn > 1e-10 && bsn > 1e-10) ? csn / bsn : 1.0;
        d.log_omega0 = std::log(d.omega);
        d.tau = d.eta / d.omega;
        d.sigma = d.eta * d.omega;
        cn[i] = std::sqrt(co.hi + co.lo);
        bn[i] = std::sqrt(bo.hi + bo.lo);
    }
    h2d(h, B->insts, st0.data(), I * sizeof(nir::DevState));
    launch_bcompact(B);
    h2d(h, B->d_bnorm, bn.data(), I * sizeof(double));
    h2d(h, B->d_cnorm, cn.data(), I * sizeof(double));
    h2d(h, B->d_offset, B->offsets.data(), I * sizeof(double));
    nir::k_init_iterates<<<grid_for(std::max(n, m)), nir::kBlock, 0, s>>>(
        n, m, nullptr, nullptr, h->dc, h->dr, h->l64, h->u64, h->x64, h->x064, h->y64, h->y064, h->x32, h->x032,
        h->y32, h->y032, h->l32, h->u32);
    NIR_LAUNCHED();
    // occupancy queries before any capture
    if (p.precision == NIR_PREC_FP32) warm_batch_cfgs<float, float>(B);
    if (p.precision == NIR_PREC_MIXED) warm_batch_cfgs<float, double>(B);
    if (p.precision != NIR_PREC_FP32) warm_batch_cfgs<double, double>(B);
    NIR_CUDA(cudaStreamSynchronize(s));
    const double t_setup = now_sec();
    const bool fp64_first = (p.precision == NIR_PREC_FP64);
    // prec: 0 = (float values, float iterates), 1 = (float, double), 2 = (double, double)
    auto run_phase = [&](int phase, int prec) {
        auto launch = [&, phase, prec]() {
            if (prec == 2) launch_batch_chunk<double, double>(B, cfg, phase);
            else if (prec == 1) launch_batch_chunk<float, double>(B, cfg, phase);
            else launch_batch_chunk<float, float>(B, cfg, phase);
        };
        const int per = 2 * cfg.K + 7;
        if (p.use_graphs && !cfg.persistent) {
            KeyHash k;
            k.add(chunk_key(h, cfg, phase, prec)).add(B->cur->a.blk).add(B->cur->at.blk).add(B->cur->a.lay);
            k.add(B->cur->at.lay).add(B->cur->a.cap).add(B->cur->at.cap).add(B->cur->part).add(B->insts);
            ChunkGraph& g = B->graphs[phase];
            if (!(g.ge && g.valid && g.key == k.h)) {
                // capture into the handle's slot, then keep it with the batch
                std::swap(g, h->graphs[1 + phase]);
                chunk_graph(h, 1 + phase, k.h, launch);
                std::swap(g, h->graphs[1 + phase]);
            }
            cudaGraphExec_t ge = g.ge;
            return run_chunks(h, p, poll, ctx, t0, phase, per, [&]() { NIR_CUDA(cudaGraphLaunch(ge, s)); }, nullptr);
        }
        return run_chunks(h, p, poll, ctx, t0, phase, 0, launch, nullptr);
    };
    LoopResult R;
    std::vector<long long> it_switch(I, -1);  // iteration of each instance's FP32->FP64 hand-over
    if (p.max_iters > 0) {
        R = run_phase(0, fp64_first ? 2 : (p.precision == NIR_PREC_MIXED ? 1 : 0));
        if (!R.stopped_by_host && cfg.mixed && !R.last.done && R.last.phase == 1) {
            std::vector<nir::DevState> sw(I);
            d2h(h, sw.data(), B->insts, I * sizeof(nir::DevState));
            for (int i = 0; i < I; ++i)
                if (!sw[i].done && sw[i].phase == 1) it_switch[i] = sw[i].iter;
            // instances whose FP32-value phase stalled carry on with the FP64
            // values; their iterates are FP64 already (a pure precision change)
            R = run_phase(1, 2);
        }
    }
    std::vector<nir::DevState> st(I);
    d2h(h, st.data(), B->insts, I * sizeof(nir::DevState));
    nir::k_bunscale_out<<<grid_for(std::max(n, m)), nir::kBlock, 0, s>>>(
        n, m, B->d_col_inst, B->d_row_inst, B->insts, h->xp32, h->yp32, h->xp64, h->yp64,
        p.precision != NIR_PREC_FP32 ? 1 : 0, h->dc,
        h->dr, h->out_x, h->out_y);
    NIR_LAUNCHED();
    std::vector<double> x(n), y(m);
    d2h(h, x.data(), h->out_x, n * sizeof(double));
    d2h(h, y.data(), h->out_y, m * sizeof(double));
    B->solved = true;
    if (x_out) std::memcpy(x_out, x.data(), n * sizeof(double));
    if (y_out) std::memcpy(y_out, y.data(), m * sizeof(double));
    const double t_end = now_sec();
    int worst = NIR_STATUS_OPTIMAL;
    long long iters = 0, iters64 = 0;
    for (int i = 0; i < I; ++i) {
        nir_pdhg_info inf{};
        const nir::DevState& d = st[i];
        inf.status = d.done ? d.status : (R.stopped_by_host ? NIR_STATUS_TIME_LIMIT : NIR_STATUS_ITERATION_LIMIT);
        if (p.max_iters <= 0) inf.status = NIR_STATUS_ITERATION_LIMIT;
        inf.iterations = d.iter;
        inf.iterations_fp64 = fp64_first ? d.iter : (it_switch[i] >= 0 ? d.iter - it_switch[i] : 0);
        inf.restarts = d.restarts;
        inf.rel_kkt = d.kkt;
        inf.rel_primal = d.kp;
        inf.rel_dual = d.kd;
        inf.rel_gap = d.kg;
        inf.max_rel_row_viol = d.max_rel_row;
        inf.primal_weight = d.omega;
        inf.step_size = d.eta;
        DD o;
        o.hi = B->offsets[i];
        for (int j = B->col_off[i]; j < B->col_off[i + 1]; ++j)
            if (h->h_c[j] != 0.0 && x[j] != 0.0) o = dd_add_prod(o, h->h_c[j], x[j]);
        inf.objective = o.hi + o.lo;
        inf.setup_seconds = t_setup - t0;
        inf.solve_seconds = t_end - t_setup;
        inf.iterations_to_tol = (inf.status == NIR_STATUS_OPTIMAL) ? inf.iterations : -1;
        if (infos) infos[i] = inf;
        if (inf.status != NIR_STATUS_OPTIMAL && worst == NIR_STATUS_OPTIMAL) worst = inf.status;
        iters = std::max<long long>(iters, d.iter);
        iters64 = std::max<long long>(iters64, inf.iterations_fp64);
    }
    if (total) {
        std::memset(total, 0, sizeof(*total));
        total->status = worst;
        total->iterations = iters;
        total->iterations_fp64 = iters64;
        total->setup_seconds = t_setup - t0;
        total->solve_seconds = t_end - t_setup;
        total->kernel_launches = h->launches;
    }
    return worst;
}

}  // namespace

extern "C" {

int nir_pdhg_batch_create(const nir_lp_view* lps, int32_t count, int device, nir_pdhg_batch** out) {
    if (!out || !lps || count < 1) {
        g_err = "invalid arguments";
        return NIR_STATUS_INPUT_ERROR;
    }
    *out = nullptr;
    auto B = std::make_unique<nir_pdhg_batch>();
    try {
        batch_create_impl(B.get(), lps, count, device);
    } catch (const std::invalid_argument& e) {
        g_err = e.what();
        return NIR_STATUS_INPUT_ERROR;
    } catch (const std::exception& e) {
        g_err = e.what();
        return NIR_STATUS_INTERNAL_ERROR;
    }
    *out = B.release();
    return 0;
}

int nir_pdhg_batch_solve(nir_pdhg_batch* b, const nir_pdhg_params* p_in, int (*poll)(void*), void* poll_ctx,
                         double* x_out, double* y_out, nir_pdhg_info* infos, nir_pdhg_info* total) {
    if (!b || !b->h) {
        g_err = "null handle";
        return NIR_STATUS_INPUT_ERROR;
    }
    nir_pdhg_params p;
    if (p_in) p = *p_in;
    else nir_pdhg_default_params(&p);
    try {
        NIR_CUDA(cudaSetDevice(b->h->device));
        b->h->launches = 0;
        return batch_solve_impl(b, p, poll, poll_ctx, x_out, y_out, infos, total);
    } catch (const std::invalid_argument& e) {
        g_err = e.what();
        return NIR_STATUS_INPUT_ERROR;
    } catch (const std::exception& e) {
        g_err = e.what();
        return NIR_STATUS_INTERNAL_ERROR;
    }
}

void nir_pdhg_batch_free(nir_pdhg_batch* b) { delete b; }

}  // extern "C"
