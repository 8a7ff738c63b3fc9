// Batched PDLP: many LPs of uneven sizes in one launch per half-iteration.
//
// The instances are laid out block-diagonally in one handle: instance i
// owns rows [row_off[i], row_off[i+1]) and columns [col_off[i],
// col_off[i+1]), and its blocks (which never cross an instance) are
// contiguous, in either layout of k_iter.cuh.  Every instance keeps its own DevState on the device:
// step sizes, primal weight, Halpern counter, restart anchor, precision
// phase and convergence flag.  The iteration kernels visit the blocks of
// the instances still running (k_bcompact), and in a check launch
// leave one partial sum per quantity and block; the controller then runs
// one CTA per instance, reducing that instance's block range in a fixed
// order (deterministic) and applying the same update as the single-LP
// controller.
#pragma once

#include "k_iter.cuh"
#include "k_setup.cuh"

namespace nir {

struct BatchArgs {
    Lay lay;              // blocks never cross an instance
    double* part;         // per-block partials: part[q * nblk + block]
    const DevState* inst;
    int i_in_chunk;
    int halpern;
    int phase;
    double rho;
    // the blocks the kernels visit: those of the instances still running,
    // listed by k_bcompact after every check (blocks of instance i are
    // [blk_lo[i], blk_lo[i+1]) in this orientation)
    const int* blk_lo;
    const int* act_inst;  // running instances, ascending
    const int* act_off;   // their first visited block in this orientation's list (act_n + 1 entries)
    const int* act_n;
};

__device__ __forceinline__ bool inst_active(const DevState& s, int phase) { return !s.done && s.phase == phase; }

// Block of the v-th visited position (v < act_off[nact]) and its instance:
// the running instance whose range holds v (binary search over the running
// instances), then the offset within its blocks.
__device__ __forceinline__ int visited_block(const BatchArgs& a, int v, int nact, int& inst) {
    int lo = 0, hi = nact - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(a.act_off + mid) <= v) lo = mid;
        else hi = mid - 1;
    }
    inst = __ldg(a.act_inst + lo);
    return __ldg(a.blk_lo + inst) + (v - __ldg(a.act_off + lo));
}

// Lists the running instances (not done, in either phase) and the prefix of
// their block counts in both orientations.  One CTA; a fixed scan order.
__global__ void __launch_bounds__(kBlock) k_bcompact(int count, const DevState* __restrict__ insts,
                                                     const int* __restrict__ a_lo, const int* __restrict__ at_lo,
                                                     int* __restrict__ act_inst, int* __restrict__ act_off_a,
                                                     int* __restrict__ act_off_at, int* __restrict__ act_n) {
    __shared__ int sh[3][kWarps];
    __shared__ int carry[3];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry[0] = carry[1] = carry[2] = 0;
    __syncthreads();
    for (int base = 0; base < count; base += kBlock) {
        const int i = base + threadIdx.x;
        const bool run = i < count && !insts[i].done;
        int v[3] = {run ? 1 : 0, run ? a_lo[i + 1] - a_lo[i] : 0, run ? at_lo[i + 1] - at_lo[i] : 0};
        int incl[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            int x = v[q];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            incl[q] = x;
            if (lane == 31) sh[q][w] = x;
        }
        __syncthreads();
        int pre[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            int before = carry[q];
            for (int k = 0; k < w; ++k) before += sh[q][k];
            pre[q] = before + incl[q] - v[q];
        }
        if (run) {
            act_inst[pre[0]] = i;
            act_off_a[pre[0]] = pre[1];
            act_off_at[pre[0]] = pre[2];
        }
        __syncthreads();
        if (threadIdx.x == kBlock - 1) {
#pragma unroll
            for (int q = 0; q < 3; ++q) carry[q] = pre[q] + v[q];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        act_off_a[carry[0]] = carry[1];
        act_off_at[carry[0]] = carry[2];
        *act_n = carry[0];
    }
}

// Warp layout: reduces each per-lane quantity over the warp into the
// block's partial slot and clears it for the next block.
template <class Epi>
__device__ __forceinline__ void flush_warp_partials(Epi& epi, double* __restrict__ part, int nblk, int b) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int q = 0; q < Epi::NQ; ++q) {
        const double v = (Epi::kLastIsMax && q == Epi::NQ - 1) ? warp_max(epi.q[q]) : warp_sum(epi.q[q]);
        if (lane == 0) part[q * nblk + b] = v;
        epi.q[q] = 0.0;
    }
}

// CTA layout: the same over the CTA.
template <class Epi>
__device__ __forceinline__ void flush_cta_partials(Epi& epi, double* __restrict__ part, int nblk, int b,
                                                   double* s_red) {
#pragma unroll
    for (int q = 0; q < Epi::NQ; ++q) {
        const double v = (Epi::kLastIsMax && q == Epi::NQ - 1) ? block_max(epi.q[q], s_red) : block_sum(epi.q[q], s_red);
        if (threadIdx.x == 0) part[q * nblk + b] = v;
        epi.q[q] = 0.0;
    }
}

// The layout's SpMV over the batch: per block, the instance decides whether
// the block runs and with which scalars (SetFn(epi, DevState&)).  In the CTA
// layout the decision is the same for every thread of the CTA.
template <int LAY, typename TA, typename TV, typename TX, class Epi, bool COH = false, class SetFn>
__device__ __forceinline__ void lay_spmv_batch(const BatchArgs& a, const TV* __restrict__ val,
                                               const TX* __restrict__ x, Epi& epi, SetFn set, double* s_red) {
    const Lay& L = a.lay;
    if constexpr (LAY == kLayWarp) {
        extern __shared__ __align__(16) unsigned char nir_smem[];
        const int w = threadIdx.x >> 5;
        TA* s_prod = reinterpret_cast<TA*>(nir_smem) + w * kWarpCapMax;
        const int2* blk = static_cast<const int2*>(L.blk);
        const int G = gridDim.x * kWarps;
        const int nact = __ldg(a.act_n);
        const int total = nact > 0 ? __ldg(a.act_off + nact) : 0;
        int pos = blockIdx.x * kWarps + w;
        if (pos >= total) return;
        int inst = 0;
        int b = visited_block(a, pos, nact, inst);
        int2 d0 = __ldg(blk + b), d1 = __ldg(blk + b + 1);
        bool act = inst_active(a.inst[inst], a.phase);
        int c[kWarpU];
        TV v[kWarpU];
        stream_load<TV>(d0, d1, act ? L.cap : -1, L.ci, val, c, v);
        for (;;) {
            const int pn = pos + G;
            const bool has_next = pn < total;
            int2 n0 = make_int2(0, 0), n1 = make_int2(0, 0);
            int inst_n = 0, bn = 0;
            bool act_n = false;
            if (has_next) {
                bn = visited_block(a, pn, nact, inst_n);
                n0 = __ldg(blk + bn);
                n1 = __ldg(blk + bn + 1);
                act_n = inst_active(a.inst[inst_n], a.phase);
            }
            int cn[kWarpU];
            TV vn[kWarpU];
            stream_load<TV>(n0, n1, act_n ? L.cap : -1, L.ci, val, cn, vn);
            if (act) {
                set(epi, a.inst[inst]);
                warp_process<TA, TV, TX, Epi, COH>(d0, d1, L.cap, L.rp, L.ci, val, x, epi, s_prod, c, v);
                if (Epi::NQ > 0) flush_warp_partials(epi, a.part, L.nblk, b);
            }
            if (!has_next) break;
#pragma unroll
            for (int q = 0; q < kWarpU; ++q) {
                c[q] = cn[q];
                v[q] = vn[q];
            }
            d0 = n0;
            d1 = n1;
            inst = inst_n;
            act = act_n;
            b = bn;
            pos = pn;
        }
    } else {
        __shared__ CtaShared<TA> sm[2];
        const int4* blk = static_cast<const int4*>(L.blk);
        int k = 0;
        const int nact = __ldg(a.act_n);
        const int total = nact > 0 ? __ldg(a.act_off + nact) : 0;
        for (int pos = blockIdx.x; pos < total; pos += gridDim.x) {
            int inst = 0;
            const int b = visited_block(a, pos, nact, inst);
            const int4 d0 = __ldg(blk + b), d1 = __ldg(blk + b + 1);
            const DevState& s = a.inst[inst];
            if (!inst_active(s, a.phase)) continue;
            set(epi, s);
            cta_block<TA, TV, TX, LAY, Epi, COH>(d0, d1, L.rp, L.ci, val, x, epi, sm[k & 1]);
            ++k;
            if (Epi::NQ > 0) flush_cta_partials(epi, a.part, L.nblk, b, s_red);
        }
    }
}

template <int LAY, typename TV, typename TX, bool CHECK>
__global__ void __launch_bounds__(kBlock, (lay_min_blocks<LAY, TV, TX, true>()))
    k_bprimal(BatchArgs a, const TV* __restrict__ val, const TX* __restrict__ y, TX* __restrict__ x,
              TX* __restrict__ xbar, TX* __restrict__ xplus, const TX* __restrict__ c, const TX* __restrict__ lo,
              const TX* __restrict__ up, const TX* __restrict__ x0) {
    __shared__ double s_red[kWarps];
    PrimalEpi<TX, CHECK> epi;
    epi.x = x;
    epi.xbar = xbar;
    epi.xplus = xplus;
    epi.c = c;
    epi.lo = lo;
    epi.up = up;
    epi.x0 = x0;
    epi.halpern = a.halpern;
    lay_spmv_batch<LAY, TX, TV, TX>(a, val, y, epi, [&](PrimalEpi<TX, CHECK>& e, const DevState& s) {
        e.s = step_scalars<TX>(&s, a.i_in_chunk, a.halpern, a.rho);
    }, s_red);
}

template <int LAY, typename TV, typename TX, bool CHECK>
__global__ void __launch_bounds__(kBlock, (lay_min_blocks<LAY, TV, TX, true>()))
    k_bdual(BatchArgs a, const TV* __restrict__ val, const TX* __restrict__ xbar, TX* __restrict__ y,
            TX* __restrict__ yplus, const TX* __restrict__ rl, const TX* __restrict__ ru, const TX* __restrict__ y0) {
    __shared__ double s_red[kWarps];
    DualEpi<TX, CHECK> epi;
    epi.y = y;
    epi.yplus = yplus;
    epi.rl = rl;
    epi.ru = ru;
    epi.y0 = y0;
    epi.halpern = a.halpern;
    lay_spmv_batch<LAY, TX, TV, TX>(a, val, xbar, epi, [&](DualEpi<TX, CHECK>& e, const DevState& s) {
        e.s = step_scalars<TX>(&s, a.i_in_chunk, a.halpern, a.rho);
    }, s_red);
}

template <int LAY, typename TX>
__global__ void __launch_bounds__(kBlock)
    k_bkkt_rows(BatchArgs a, const double* __restrict__ val, const TX* __restrict__ xplus,
                const TX* __restrict__ yplus, const double* __restrict__ dr, const double* __restrict__ rl,
                const double* __restrict__ ru) {
    __shared__ double s_red[kWarps];
    KktRowEpi<TX> epi;
    epi.dr = dr;
    epi.rl = rl;
    epi.ru = ru;
    epi.yplus = yplus;
    lay_spmv_batch<LAY, double, double, TX>(a, val, xplus, epi, [](KktRowEpi<TX>&, const DevState&) {}, s_red);
}

template <int LAY, typename TX>
__global__ void __launch_bounds__(kBlock)
    k_bkkt_cols(BatchArgs a, const double* __restrict__ val, const TX* __restrict__ xplus,
                const TX* __restrict__ yplus, const double* __restrict__ dc, const double* __restrict__ c,
                const double* __restrict__ l, const double* __restrict__ u) {
    __shared__ double s_red[kWarps];
    KktColEpi<TX> epi;
    epi.dc = dc;
    epi.c = c;
    epi.l = l;
    epi.u = u;
    epi.xplus = xplus;
    lay_spmv_batch<LAY, double, double, TX>(a, val, yplus, epi, [](KktColEpi<TX>&, const DevState&) {}, s_red);
}

struct BatchCtlArgs {
    const double* partP;   // 2 x nP (A' blocks)
    const double* partD;   // 2 x nD (A blocks)
    const double* partKR;  // 4 x nD
    const double* partKC;  // 4 x nP
    int nP, nD;
    const int* at_lo;      // instance i's A' blocks: [at_lo[i], at_lo[i+1])
    const int* a_lo;       // instance i's A blocks:  [a_lo[i], a_lo[i+1])
    const double* bnorm;   // per instance, original space
    const double* cnorm;
    const double* offset;
};

__device__ inline double range_sum(const double* __restrict__ p, int lo, int hi, double* sh) {
    double s = 0.0;
    for (int i = lo + threadIdx.x; i < hi; i += kBlock) s += p[i];
    return block_sum(s, sh);
}

__device__ inline double range_max(const double* __restrict__ p, int lo, int hi, double* sh) {
    double s = 0.0;
    for (int i = lo + threadIdx.x; i < hi; i += kBlock) s = fmax(s, p[i]);
    return block_max(s, sh);
}

// One CTA per instance.
__global__ void __launch_bounds__(kBlock) k_bcontrol(CtlArgs a, BatchCtlArgs b, DevState* insts) {
    __shared__ double sh[kWarps];
    const int i = blockIdx.x;
    DevState* st = insts + i;
    if (st->done || st->phase != a.phase) return;
    const int p0 = b.at_lo[i], p1 = b.at_lo[i + 1], d0 = b.a_lo[i], d1 = b.a_lo[i + 1];
    CtlSums s;
    s.dx2 = range_sum(b.partP, p0, p1, sh);
    s.dxa2 = range_sum(b.partP + b.nP, p0, p1, sh);
    s.dy2 = range_sum(b.partD, d0, d1, sh);
    s.dya2 = range_sum(b.partD + b.nD, d0, d1, sh);
    s.pres2 = range_sum(b.partKR, d0, d1, sh);
    s.dobj_r = range_sum(b.partKR + b.nD, d0, d1, sh);
    s.ywrong2 = range_sum(b.partKR + 2 * b.nD, d0, d1, sh);
    s.maxrel = range_max(b.partKR + 3 * b.nD, d0, d1, sh);
    s.dres2 = range_sum(b.partKC, p0, p1, sh);
    s.dobj_c = range_sum(b.partKC + b.nP, p0, p1, sh);
    s.pobj_c = range_sum(b.partKC + 2 * b.nP, p0, p1, sh);
    s.xviol2 = range_sum(b.partKC + 3 * b.nP, p0, p1, sh);
    if (threadIdx.x != 0) return;
    control_update(a, st, s, b.bnorm[i], b.cnorm[i], b.offset[i], nullptr);
}

template <typename T>
__global__ void k_bapply_restart(int n, int m, const int* __restrict__ col_inst, const int* __restrict__ row_inst,
                                 const DevState* __restrict__ insts, int phase, T* __restrict__ x, T* __restrict__ x0,
                                 const T* __restrict__ xplus, T* __restrict__ y, T* __restrict__ y0,
                                 const T* __restrict__ yplus) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) {
        const DevState& s = insts[col_inst[t]];
        if (s.apply_restart && !s.done && s.phase == phase) {
            const T v = xplus[t];
            x[t] = v;
            x0[t] = v;
        }
    }
    if (t < m) {
        const DevState& s = insts[row_inst[t]];
        if (s.apply_restart && !s.done && s.phase == phase) {
            const T v = yplus[t];
            y[t] = v;
            y0[t] = v;
        }
    }
}

// Batch status for the host: done = every instance finished, phase = 1
// once no instance is still running in phase 0.
__global__ void k_bsnap(int count, const DevState* __restrict__ insts, HostSnap* __restrict__ ring,
                        long long* __restrict__ seq) {
    __shared__ double sh[kWarps];
    double ndone = 0.0, nphase0 = 0.0, maxit = 0.0;
    for (int i = threadIdx.x; i < count; i += kBlock) {
        const DevState& s = insts[i];
        ndone += s.done ? 1.0 : 0.0;
        nphase0 += (!s.done && s.phase == 0) ? 1.0 : 0.0;
        maxit = fmax(maxit, double(s.iter));
    }
    ndone = block_sum(ndone, sh);
    nphase0 = block_sum(nphase0, sh);
    maxit = block_max(maxit, sh);
    if (threadIdx.x != 0) return;
    const long long s = *seq + 1;
    *seq = s;
    HostSnap h{};
    h.seq = s;
    h.iter = (long long)maxit;
    h.done = (int(ndone) == count) ? 1 : 0;
    h.phase = (int(nphase0) == 0) ? 1 : 0;
    h.restarts = int(ndone);
    ring[s % kSnapRing] = h;
    __threadfence_system();
}

// Per-instance norms over contiguous ranges (power iteration).
__global__ void k_seg_norm(const int* __restrict__ off, const double* __restrict__ w, double* __restrict__ norm) {
    __shared__ double sh[kWarps];
    const int i = blockIdx.x;
    double s = 0.0;
    for (int j = off[i] + threadIdx.x; j < off[i + 1]; j += kBlock) s += w[j] * w[j];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) norm[i] = sqrt(s);
}

__global__ void k_seg_scale(int n, const int* __restrict__ inst_of, const double* __restrict__ norm,
                            double* __restrict__ w) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const double d = norm[inst_of[j]];
    w[j] = d > 0.0 ? w[j] / d : 0.0;
}

// Output of a batch: each instance from the precision it ended in.
__global__ void k_bunscale_out(int n, int m, const int* __restrict__ col_inst, const int* __restrict__ row_inst,
                               const DevState* __restrict__ insts, const float* __restrict__ xp32,
                               const float* __restrict__ yp32, const double* __restrict__ xp64,
                               const double* __restrict__ yp64, int all64, const double* __restrict__ dc,
                               const double* __restrict__ dr, double* __restrict__ xo, double* __restrict__ yo) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) {
        const bool f64 = all64 || insts[col_inst[t]].phase == 1;
        xo[t] = (f64 ? xp64[t] : double(xp32[t])) * dc[t];
    }
    if (t < m) {
        const bool f64 = all64 || insts[row_inst[t]].phase == 1;
        yo[t] = (f64 ? yp64[t] : double(yp32[t])) * dr[t];
    }
}

}  // namespace nir
