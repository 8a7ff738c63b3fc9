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
    // warp row blocks per instance, built for one capacity
    int cap = 0;
    int2 *blkA = nullptr, *blkAt = nullptr;
    int *instA = nullptr, *instAt = nullptr;
    int nblkA = 0, nblkAt = 0;
    int *d_a_lo = nullptr, *d_at_lo = nullptr;
    double* part = nullptr;
    struct Layout {
        int cap;
        int2 *blkA, *blkAt;
        int *instA, *instAt;
        int nblkA, nblkAt;
        int *a_lo, *at_lo;
        double* part;
    };
    std::vector<Layout> layouts;  // one per capacity used, built once each
    nir::DevState* insts = nullptr;
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

// Warp row blocks of one orientation, built instance by instance so that
// no block crosses an instance; also the instance of every block and each
// instance's first block.
void batch_blocks(nir_pdhg_batch* B, const std::vector<int>& rp, const std::vector<int>& off, int cap, int2** blk,
                  int** inst, int* nblk, int** d_lo) {
    nir_pdhg* h = B->h;
    std::vector<int> owner, lo;
    const std::vector<int2> all = nir::build_batch_row_blocks(rp, off, cap, &owner, &lo);
    *nblk = int(owner.size());
    *blk = h->alloc<int2>(all.size());
    h2d(h, *blk, all.data(), all.size() * sizeof(int2));
    *inst = h->alloc<int>(std::max<size_t>(owner.size(), 1));
    if (!owner.empty()) h2d(h, *inst, owner.data(), owner.size() * sizeof(int));
    *d_lo = h->alloc<int>(lo.size());
    h2d(h, *d_lo, lo.data(), lo.size() * sizeof(int));
}

nir::BatchArgs bargs(nir_pdhg_batch* B, bool transpose, double* part, int i, int halpern, int phase, double rho) {
    nir_pdhg* h = B->h;
    const Orient& o = transpose ? h->At : h->A;
    return nir::BatchArgs{transpose ? B->blkAt : B->blkA, transpose ? B->nblkAt : B->nblkA, B->cap, o.rp, o.ci,
                          transpose ? B->instAt : B->instA, part, B->insts, i, halpern, phase, rho};
}

template <typename T>
void launch_batch_chunk(nir_pdhg_batch* B, const SolveCfg& cfg, int phase) {
    nir_pdhg* h = B->h;
    cudaStream_t s = h->stream;
    const int K = cfg.K;
    double* P = B->part;
    double* D = P + 2 * size_t(std::max(B->nblkAt, 1));
    double* KR = D + 2 * size_t(std::max(B->nblkA, 1));
    double* KC = KR + 4 * size_t(std::max(B->nblkA, 1));
    const LaunchCfg cp1 = warp_cfg<T>(h, nir::k_bprimal<T, true>, B->nblkAt);
    const LaunchCfg cp0 = warp_cfg<T>(h, nir::k_bprimal<T, false>, B->nblkAt);
    const LaunchCfg cd1 = warp_cfg<T>(h, nir::k_bdual<T, true>, B->nblkA);
    const LaunchCfg cd0 = warp_cfg<T>(h, nir::k_bdual<T, false>, B->nblkA);
    const LaunchCfg ckr = warp_cfg<double>(h, nir::k_bkkt_rows<T>, B->nblkA);
    const LaunchCfg ckc = warp_cfg<double>(h, nir::k_bkkt_cols<T>, B->nblkAt);
    for (int i = 0; i < K; ++i) {
        const bool check = (i == K - 1);
        nir::BatchArgs ap = bargs(B, true, P, i, cfg.halpern, phase, cfg.p.reflection);
        nir::BatchArgs ad = bargs(B, false, D, i, cfg.halpern, phase, cfg.p.reflection);
        if (check)
            nir::k_bprimal<T, true><<<cp1.grid, nir::kBlock, cp1.smem, s>>>(
                ap, View<T>::valAt(h), View<T>::y(h), View<T>::x(h), View<T>::xb(h), View<T>::xp(h), View<T>::c(h),
                View<T>::l(h), View<T>::u(h), View<T>::x0(h));
        else
            nir::k_bprimal<T, false><<<cp0.grid, nir::kBlock, cp0.smem, s>>>(
                ap, View<T>::valAt(h), View<T>::y(h), View<T>::x(h), View<T>::xb(h), View<T>::xp(h), View<T>::c(h),
                View<T>::l(h), View<T>::u(h), View<T>::x0(h));
        NIR_LAUNCHED();
        if (check)
            nir::k_bdual<T, true><<<cd1.grid, nir::kBlock, cd1.smem, s>>>(ad, View<T>::valA(h), View<T>::xb(h),
                                                                        View<T>::y(h), View<T>::yp(h), View<T>::rl(h),
                                                                        View<T>::ru(h), View<T>::y0(h));
        else
            nir::k_bdual<T, false><<<cd0.grid, nir::kBlock, cd0.smem, s>>>(ad, View<T>::valA(h), View<T>::xb(h),
                                                                         View<T>::y(h), View<T>::yp(h), View<T>::rl(h),
                                                                         View<T>::ru(h), View<T>::y0(h));
        NIR_LAUNCHED();
        h->launches += 2;
    }
    nir::BatchArgs kr = bargs(B, false, KR, 0, 0, phase, 0.0);
    nir::k_bkkt_rows<T><<<ckr.grid, nir::kBlock, ckr.smem, s>>>(kr, h->A.v64, View<T>::xp(h), View<T>::yp(h), h->dr,
                                                                h->rl, h->ru);
    nir::BatchArgs kc = bargs(B, true, KC, 0, 0, phase, 0.0);
    nir::k_bkkt_cols<T><<<ckc.grid, nir::kBlock, ckc.smem, s>>>(kc, h->At.v64, View<T>::xp(h), View<T>::yp(h), h->dc,
                                                                h->c, h->l, h->u);
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
    nir::BatchCtlArgs cb{P, D, KR, KC, B->nblkAt, B->nblkA, B->d_at_lo, B->d_a_lo, B->d_bnorm, B->d_cnorm, B->d_offset};
    nir::k_bcontrol<<<B->count, nir::kBlock, 0, s>>>(ca, cb, B->insts);
    nir::k_bapply_restart<T><<<grid_for(std::max(h->n, h->m)), nir::kBlock, 0, s>>>(
        h->n, h->m, B->d_col_inst, B->d_row_inst, B->insts, phase, View<T>::x(h), View<T>::x0(h), View<T>::xp(h),
        View<T>::y(h), View<T>::y0(h), View<T>::yp(h));
    nir::k_bsnap<<<1, nir::kBlock, 0, s>>>(B->count, B->insts, h->snap.ring, h->snap.d_seq);
    NIR_LAUNCHED();
    h->launches += 7;
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
    if (p.spmv_block_nnz > nir::kWarpCapMax) throw std::invalid_argument("spmv_block_nnz must be in [1, 256]");
    if (p.check_every < 1 || p.reflection < 0.0 || p.reflection > 1.0 || !(p.tol >= 0.0))
        throw std::invalid_argument("invalid parameters");
    const int cap = pick_cap(h, p);  // timed on the block-diagonal matrix
    if (B->cap != cap) {
        bool found = false;
        for (const auto& l : B->layouts)
            if (l.cap == cap) {
                B->blkA = l.blkA;
                B->blkAt = l.blkAt;
                B->instA = l.instA;
                B->instAt = l.instAt;
                B->nblkA = l.nblkA;
                B->nblkAt = l.nblkAt;
                B->d_a_lo = l.a_lo;
                B->d_at_lo = l.at_lo;
                B->part = l.part;
                found = true;
            }
        if (!found) {
            batch_blocks(B, h->A.h_rp, B->row_off, cap, &B->blkA, &B->instA, &B->nblkA, &B->d_a_lo);
            batch_blocks(B, h->At.h_rp, B->col_off, cap, &B->blkAt, &B->instAt, &B->nblkAt, &B->d_at_lo);
            B->part = h->alloc<double>(6 * size_t(std::max(B->nblkA, 1)) + 6 * size_t(std::max(B->nblkAt, 1)));
            B->layouts.push_back({cap, B->blkA, B->blkAt, B->instA, B->instAt, B->nblkA, B->nblkAt, B->d_a_lo,
                                  B->d_at_lo, B->part});
        }
        B->cap = cap;
    }
    SolveCfg cfg;
    cfg.p = p;
    cfg.K = p.check_every;
    cfg.halpern = 1;
    cfg.restarts = 1;
    cfg.mixed = (p.precision == NIR_PREC_MIXED) ? 1 : 0;
    precondition(h, p, p.ruiz_iters > 0 || p.pock_chambolle);
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
    h2d(h, B->d_bnorm, bn.data(), I * sizeof(double));
    h2d(h, B->d_cnorm, cn.data(), I * sizeof(double));
    h2d(h, B->d_offset, B->offsets.data(), I * sizeof(double));
    nir::k_init_iterates<<<grid_for(std::max(n, m)), nir::kBlock, 0, s>>>(
        n, m, nullptr, nullptr, h->dc, h->dr, h->l64, h->u64, h->x64, h->x064, h->y64, h->y064, h->x32, h->x032,
        h->y32, h->y032, h->l32, h->u32);
    NIR_LAUNCHED();
    // occupancy queries before any capture
    warp_cfg<float>(h, nir::k_bprimal<float, true>, B->nblkAt);
    warp_cfg<float>(h, nir::k_bprimal<float, false>, B->nblkAt);
    warp_cfg<float>(h, nir::k_bdual<float, true>, B->nblkA);
    warp_cfg<float>(h, nir::k_bdual<float, false>, B->nblkA);
    warp_cfg<double>(h, nir::k_bprimal<double, true>, B->nblkAt);
    warp_cfg<double>(h, nir::k_bprimal<double, false>, B->nblkAt);
    warp_cfg<double>(h, nir::k_bdual<double, true>, B->nblkA);
    warp_cfg<double>(h, nir::k_bdual<double, false>, B->nblkA);
    warp_cfg<double>(h, nir::k_bkkt_rows<float>, B->nblkA);
    warp_cfg<double>(h, nir::k_bkkt_cols<float>, B->nblkAt);
    warp_cfg<double>(h, nir::k_bkkt_rows<double>, B->nblkA);
    warp_cfg<double>(h, nir::k_bkkt_cols<double>, B->nblkAt);
    NIR_CUDA(cudaStreamSynchronize(s));
    const double t_setup = now_sec();
    const bool fp64_first = (p.precision == NIR_PREC_FP64);
    auto run_phase = [&](int phase, bool f64) {
        auto launch = [&, phase, f64]() {
            if (f64) launch_batch_chunk<double>(B, cfg, phase);
            else launch_batch_chunk<float>(B, cfg, phase);
        };
        const int per = 2 * cfg.K + 7;
        if (p.use_graphs) {
            KeyHash k;
            k.add(chunk_key(h, cfg, phase, f64)).add(B->blkA).add(B->blkAt).add(B->part).add(B->insts);
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
        R = run_phase(0, fp64_first);
        if (!R.stopped_by_host && cfg.mixed && !R.last.done && R.last.phase == 1) {
            std::vector<nir::DevState> sw(I);
            d2h(h, sw.data(), B->insts, I * sizeof(nir::DevState));
            for (int i = 0; i < I; ++i)
                if (!sw[i].done && sw[i].phase == 1) it_switch[i] = sw[i].iter;
            // instances that stalled in FP32 carry on in FP64 (pure precision change)
            nir::k_to_double<<<grid_for(n), nir::kBlock, 0, s>>>(n, h->x32, h->x64);
            nir::k_to_double<<<grid_for(n), nir::kBlock, 0, s>>>(n, h->x032, h->x064);
            nir::k_to_double<<<grid_for(n), nir::kBlock, 0, s>>>(n, h->xp32, h->xp64);
            nir::k_to_double<<<grid_for(m), nir::kBlock, 0, s>>>(m, h->y32, h->y64);
            nir::k_to_double<<<grid_for(m), nir::kBlock, 0, s>>>(m, h->y032, h->y064);
            nir::k_to_double<<<grid_for(m), nir::kBlock, 0, s>>>(m, h->yp32, h->yp64);
            NIR_LAUNCHED();
            R = run_phase(1, true);
        }
    }
    std::vector<nir::DevState> st(I);
    d2h(h, st.data(), B->insts, I * sizeof(nir::DevState));
    nir::k_bunscale_out<<<grid_for(std::max(n, m)), nir::kBlock, 0, s>>>(
        n, m, B->d_col_inst, B->d_row_inst, B->insts, h->xp32, h->yp32, h->xp64, h->yp64, fp64_first ? 1 : 0, h->dc,
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
