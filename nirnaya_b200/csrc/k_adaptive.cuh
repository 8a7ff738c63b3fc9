// The hot path: a warp-granular CSR-adaptive SpMV with the PDHG update
// fused into its epilogue.
//
// A matrix orientation (A, or the stored transpose A') is cut into warp row
// blocks of at most `cap` (<= 256) nonzeros and at most 32 rows; a longer row
// gets a block of its own.  Block b is described by blk[b] = (first row,
// first nonzero), so one 8-byte load gives a warp its whole range.
// Persistent warps walk their blocks with register double buffering (the
// next block's index/value stream is in flight while the current one is
// gathered and reduced); within a block the lanes stream consecutive
// nonzeros (coalesced), gather x, leave the products in the warp's shared
// slice, and teams of lanes reduce each row by a fixed shuffle tree before
// the team leader runs the epilogue.  No block-wide barrier is involved.
// The reduction order depends only on the layout, so results are
// deterministic run to run, and no atomics are used.  Each epilogue reads
// and writes only its own row's vector entries, so the update of x (or y)
// happens in the same pass as the SpMV: one read of A per half-iteration.
//
// Reference correspondence: the primal epilogue is
// src/gpu/pdhg_solver.hpp:71-78 (x+ = proj(x - tau(c - A'y)), xbar = 2x+ - x),
// the dual epilogue :84-89 (y += sigma(proj(A xbar - y/sigma) - A xbar)),
// extended by the Halpern/reflection step of the restarted method.
#pragma once

#include "dev_common.cuh"
#include "row_blocks.hpp"

namespace nir {

// ---------------------------------------------------------------- core

// kWarpU, kWarpCapMax and kRowsPerWarpBlock: row_blocks.hpp

// Loads of the matrix stream (column indices and values), each read once
// per launch.  NIR_STREAM_LOAD selects the cache policy: 0 = read-only
// path (__ldg), 1 = L2 only, bypassing L1 (__ldcg), 2 = streaming,
// evict-first (__ldcs, the default: 5% faster FP64 iterations on the
// 5M-nonzero power-law workload than 0 or 1, since the stream no longer
// pushes the gathered vector out of the caches).
#ifndef NIR_STREAM_LOAD
#define NIR_STREAM_LOAD 2
#endif
// Gathers of the multiplied vector.  A kernel that runs several
// iterations (the persistent chunk kernel) rewrites that vector between
// its grid barriers, so it must gather through L2 (coherent, ld.global.cg)
// rather than through the read-only path, which may serve a stale line.
template <bool COH, typename T>
__device__ __forceinline__ T gather_ld(const T* p) {
    if (COH) return __ldcg(p);
    return __ldg(p);
}

// Same choice for the per-row operands of the iteration epilogues (cost,
// bounds, Halpern anchor), also read once per launch; streaming them
// measured 2% slower than __ldg, so the default keeps the read-only path.
#ifndef NIR_VEC_LOAD
#define NIR_VEC_LOAD 0
#endif
template <typename T>
__device__ __forceinline__ T vec_ld(const T* p) {
#if NIR_VEC_LOAD == 2
    return __ldcs(p);
#else
    return __ldg(p);
#endif
}
template <typename T>
__device__ __forceinline__ T stream_ld(const T* p) {
#if NIR_STREAM_LOAD == 1
    return __ldcg(p);
#elif NIR_STREAM_LOAD == 2
    return __ldcs(p);
#else
    return __ldg(p);
#endif
}

// Minimum resident CTAs per SM the iteration kernels are compiled for
// (register budget 65536 / (kBlock * n)): 3 (80 registers) with 4-byte
// values, 2 (128) with 8-byte values, both without spills.  Forcing 4 / 3
// spilled and measured no faster on the 5M-nonzero power-law workload.
#ifndef NIR_ITER_MINB32
#define NIR_ITER_MINB32 3
#endif
#ifndef NIR_ITER_MINB64
#define NIR_ITER_MINB64 2
#endif
template <typename T>
constexpr int iter_min_blocks() {
    return sizeof(T) == 4 ? NIR_ITER_MINB32 : NIR_ITER_MINB64;
}

// Dynamic shared memory of an iteration kernel: one product slice per warp.
template <typename TA>
__host__ __device__ constexpr int warp_smem_bytes() {
    return kWarps * kWarpCapMax * int(sizeof(TA));
}

// Loads the index/value stream of a packed warp row block into registers
// (lane l gets nonzeros l, l+32, ...).  Long rows are not preloaded.
template <typename TV>
__device__ __forceinline__ void stream_load(int2 d0, int2 d1, int cap, const int* __restrict__ ci,
                                            const TV* __restrict__ val, int (&c)[kWarpU], TV (&v)[kWarpU]) {
    const int lane = threadIdx.x & 31;
    const int p0 = d0.y, nnzb = d1.y - d0.y;
    // a packed block whole, or the first round of a long row; nothing for
    // cap < 0 (a block that will not run)
    const int lim = (cap < 0) ? 0 : min(nnzb, 32 * kWarpU);
#pragma unroll
    for (int q = 0; q < kWarpU; ++q) {
        const int k = lane + 32 * q;
        const bool ok = k < lim;
        c[q] = ok ? stream_ld(ci + p0 + k) : 0;
        v[q] = ok ? stream_ld(val + p0 + k) : TV(0);
    }
}

// One warp processes one warp row block whose stream (c, v) is already in
// registers.  A block holds either at most kRowsPerWarpBlock rows with at
// most `cap` (<= 256) nonzeros in total, or one row of any length.
//  * Packed rows: gathers of x for the staged indices, epilogue operands
//    and row pointers are issued together; products go to the warp's
//    shared slice; after __syncwarp a team of T lanes (T a power of two,
//    T * rows <= 32) sums each row by a fixed shuffle tree and the team
//    leader applies the epilogue.
//  * One long row: the warp strides over it from global memory, 256
//    nonzeros per round.
template <typename TA, typename TV, typename TX, class Epi, bool COH = false>
__device__ __forceinline__ void warp_process(int2 d0, int2 d1, int cap, const int* __restrict__ rp,
                                             const int* __restrict__ ci, const TV* __restrict__ val,
                                             const TX* __restrict__ x, Epi& epi, TA* s_prod, const int (&c)[kWarpU],
                                             const TV (&v)[kWarpU]) {
    const int lane = threadIdx.x & 31;
    const int r0 = d0.x, p0 = d0.y, r1 = d1.x, p1 = d1.y;
    const int nrows = r1 - r0, nnzb = p1 - p0;
    constexpr int U = kWarpU;
    typename Epi::Pre pre{};
    if (nnzb > cap) {
        // one long row in rounds of 32*U nonzeros; the first round's stream
        // is already in (c, v).  Each round's stream is requested before the
        // previous round's gathers are consumed (with 8-byte values this
        // takes the kernels to 128 registers, still 2 CTAs per SM, and made
        // the C2 A x 1.3 % and the C4 A' y 3.6 % faster).  Per lane the
        // products are summed in the same order as without the overlap.
        if (lane == 0) pre = epi.prefetch(r0);
        TA s = TA(0);
        int cc[U];
        TV vv[U];
#pragma unroll
        for (int q = 0; q < U; ++q) {
            cc[q] = c[q];
            vv[q] = v[q];
        }
        for (int base = p0 + lane; base < p1; base += 32 * U) {
            TX xv[U];
#pragma unroll
            for (int q = 0; q < U; ++q) xv[q] = (base + 32 * q < p1) ? gather_ld<COH>(x + cc[q]) : TX(0);
            const int nb = base + 32 * U;
            int cn[U];
            TV vn[U];
#pragma unroll
            for (int q = 0; q < U; ++q) {
                const int k = nb + 32 * q;
                cn[q] = (k < p1) ? stream_ld(ci + k) : 0;
                vn[q] = (k < p1) ? stream_ld(val + k) : TV(0);
            }
#pragma unroll
            for (int q = 0; q < U; ++q) s += TA(vv[q]) * TA(xv[q]);
#pragma unroll
            for (int q = 0; q < U; ++q) {
                cc[q] = cn[q];
                vv[q] = vn[q];
            }
        }
        s = warp_sum(s);
        if (lane == 0) epi.row(r0, s, pre);
        return;
    }
    int T = 32;
    while (T > 1 && T * nrows > 32) T >>= 1;
    const int team = lane / T, tl = lane & (T - 1);
    const int r = r0 + team;
    const bool mine = r < r1;
    TX xv[U];
#pragma unroll
    for (int q = 0; q < U; ++q) xv[q] = (lane + 32 * q < nnzb) ? gather_ld<COH>(x + c[q]) : TX(0);
    if (mine && tl == 0) pre = epi.prefetch(r);
    int ra = 0, re = 0;
    if (mine) {
        // clamped to the staged stream: a descriptor list that does not
        // match rp can give wrong sums but never leaves the warp's slice
        ra = max(__ldg(rp + r) - p0, 0);
        re = min(__ldg(rp + r + 1) - p0, nnzb);
    }
#pragma unroll
    for (int q = 0; q < U; ++q)
        if (lane + 32 * q < nnzb) s_prod[lane + 32 * q] = TA(v[q]) * TA(xv[q]);
    __syncwarp();
    TA s = TA(0);
    for (int k = ra + tl; k < re; k += T) s += s_prod[k];
    for (int o = T >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (mine && tl == 0) epi.row(r, s, pre);
    __syncwarp();  // the slice is rewritten by the next block
}

// Persistent warps: warp g of G takes warp row blocks g, g+G, g+2G, ...
// While it gathers and reduces one block, the next block's index/value
// stream and the descriptor after that are already in flight (register
// double buffering).  The per-row reduction order depends only on the
// layout, so results do not depend on the grid.
template <typename TA, typename TV, typename TX, class Epi, bool COH = false>
__device__ __forceinline__ void rowblock_spmv(const int2* __restrict__ blk, int nblk, int cap,
                                              const int* __restrict__ rp, const int* __restrict__ ci,
                                              const TV* __restrict__ val, const TX* __restrict__ x, Epi& epi,
                                              TA* /*s_red*/) {
    extern __shared__ __align__(16) unsigned char nir_smem[];
    const int w = threadIdx.x >> 5;
    TA* s_prod = reinterpret_cast<TA*>(nir_smem) + w * kWarpCapMax;
    const int G = gridDim.x * kWarps;
    int b = blockIdx.x * kWarps + w;
    if (b >= nblk) return;
    int2 d0 = __ldg(blk + b), d1 = __ldg(blk + b + 1);
    int c[kWarpU];
    TV v[kWarpU];
    stream_load<TV>(d0, d1, cap, ci, val, c, v);
    int2 n0 = make_int2(0, 0), n1 = make_int2(0, 0);
    if (b + G < nblk) {
        n0 = __ldg(blk + b + G);
        n1 = __ldg(blk + b + G + 1);
    }
    for (;;) {
        const bool has_next = b + G < nblk;
        int cn[kWarpU];
        TV vn[kWarpU];
        stream_load<TV>(n0, n1, has_next ? cap : -1, ci, val, cn, vn);
        int2 m0 = make_int2(0, 0), m1 = make_int2(0, 0);
        if (b + 2 * G < nblk) {
            m0 = __ldg(blk + b + 2 * G);
            m1 = __ldg(blk + b + 2 * G + 1);
        }
        warp_process<TA, TV, TX, Epi, COH>(d0, d1, cap, rp, ci, val, x, epi, s_prod, c, v);
        if (!has_next) break;
#pragma unroll
        for (int q = 0; q < kWarpU; ++q) {
            c[q] = cn[q];
            v[q] = vn[q];
        }
        d0 = n0;
        d1 = n1;
        n0 = m0;
        n1 = m1;
        b += G;
    }
}

// Block-reduces each per-thread quantity and stores it at
// part[q * gridDim.x + blockIdx.x].  The last quantity is a max when
// Epi::kLastIsMax.
template <class Epi>
__device__ __forceinline__ void write_partials(const Epi& epi, double* __restrict__ part, double* s_red) {
#pragma unroll
    for (int q = 0; q < Epi::NQ; ++q) {
        double v = (Epi::kLastIsMax && q == Epi::NQ - 1) ? block_max(epi.q[q], s_red) : block_sum(epi.q[q], s_red);
        if (threadIdx.x == 0) part[q * gridDim.x + blockIdx.x] = v;
    }
}

// ---------------------------------------------------------------- plain SpMV

template <typename TA>
struct PlainEpi {
    static constexpr int NQ = 0;
    static constexpr bool kLastIsMax = false;
    struct Pre {};
    double q[1];
    TA* y;
    __device__ Pre prefetch(int) const { return Pre{}; }
    __device__ void row(int r, TA s, const Pre&) { y[r] = s; }
};

template <typename TA, typename TV, typename TX>
__global__ void __launch_bounds__(kBlock, iter_min_blocks<TA>()) k_spmv_adaptive(const int2* __restrict__ blk, int nblk, int cap,
                                                          const int* __restrict__ rp, const int* __restrict__ ci,
                                                          const TV* __restrict__ val, const TX* __restrict__ x,
                                                          TA* __restrict__ y) {
    __shared__ TA s_red[kWarps];
    PlainEpi<TA> epi;
    epi.y = y;
    rowblock_spmv<TA, TV, TX>(blk, nblk, cap, rp, ci, val, x, epi, s_red);
}

// ---------------------------------------------------------------- PDHG step

// Scalars every iteration kernel needs, derived from DevState at launch.
template <typename T>
struct StepScalars {
    T tau, sigma, isigma, w, onemw, rho;  // isigma = 1 / sigma: the dual step multiplies
};

template <typename T>
__device__ __forceinline__ StepScalars<T> step_scalars(const DevState* st, int i_in_chunk, int halpern, double rho) {
    StepScalars<T> s;
    s.tau = T(st->tau);
    s.sigma = T(st->sigma);
    s.isigma = T(1.0 / st->sigma);
    if (halpern) {
        const double k = double(st->k_base + i_in_chunk);
        s.w = T((k + 1.0) / (k + 2.0));
        s.onemw = T(1.0 / (k + 2.0));
        s.rho = T(rho);
    } else {
        s.w = T(1);
        s.onemw = T(0);
        s.rho = T(0);
    }
    return s;
}

template <typename T, bool CHECK>
struct PrimalEpi {
    static constexpr int NQ = CHECK ? 2 : 0;
    static constexpr bool kLastIsMax = false;
    struct Pre {
        T x, c, lo, up, x0;
    };
    double q[2] = {0.0, 0.0};
    T* __restrict__ x;
    T* __restrict__ xbar;
    T* __restrict__ xplus;
    const T* __restrict__ c;
    const T* __restrict__ lo;
    const T* __restrict__ up;
    const T* __restrict__ x0;
    StepScalars<T> s;
    int halpern;
    __device__ Pre prefetch(int j) const {
        Pre p;
        p.x = x[j];
        p.c = vec_ld(c + j);
        p.lo = vec_ld(lo + j);
        p.up = vec_ld(up + j);
        p.x0 = (halpern || CHECK) ? vec_ld(x0 + j) : T(0);
        return p;
    }
    __device__ void row(int j, T aty, const Pre& p) {
        const T xj = p.x;
        const T xp = clamp_box(xj - s.tau * (p.c - aty), p.lo, p.up);
        xbar[j] = T(2) * xp - xj;
        T xn = xp;
        if (halpern) xn = s.w * ((T(1) + s.rho) * xp - s.rho * xj) + s.onemw * p.x0;
        x[j] = xn;
        if (CHECK) {
            xplus[j] = xp;
            const double d = double(xj) - double(xp);
            const double e = double(xp) - double(p.x0);
            q[0] += d * d;
            q[1] += e * e;
        }
    }
};

template <typename T, bool CHECK>
struct DualEpi {
    static constexpr int NQ = CHECK ? 2 : 0;
    static constexpr bool kLastIsMax = false;
    struct Pre {
        T y, rl, ru, y0;
    };
    double q[2] = {0.0, 0.0};
    T* __restrict__ y;
    T* __restrict__ yplus;
    const T* __restrict__ rl;
    const T* __restrict__ ru;
    const T* __restrict__ y0;
    StepScalars<T> s;
    int halpern;
    __device__ Pre prefetch(int i) const {
        Pre p;
        p.y = y[i];
        p.rl = vec_ld(rl + i);
        p.ru = vec_ld(ru + i);
        p.y0 = (halpern || CHECK) ? vec_ld(y0 + i) : T(0);
        return p;
    }
    __device__ void row(int i, T ax, const Pre& p) {
        const T yi = p.y;
        const T pr = clamp_box(ax - yi * s.isigma, p.rl, p.ru);
        const T yp = yi + s.sigma * (pr - ax);
        T yn = yp;
        if (halpern) yn = s.w * ((T(1) + s.rho) * yp - s.rho * yi) + s.onemw * p.y0;
        y[i] = yn;
        if (CHECK) {
            yplus[i] = yp;
            const double d = double(yi) - double(yp);
            const double e = double(yp) - double(p.y0);
            q[0] += d * d;
            q[1] += e * e;
        }
    }
};

// ---------------------------------------------------------------- KKT (FP64)

// Rows of A at (x+, y+): primal residual, dual-objective row terms,
// wrong-sign multipliers and the checker's relative row violation, all in
// the original (unscaled) space.  ax is (A_scaled x_scaled)_i = dr_i (A x)_i.
template <typename TX>
struct KktRowEpi {
    static constexpr int NQ = 4;
    static constexpr bool kLastIsMax = true;
    struct Pre {
        double d, lo, hi;
        TX y;
    };
    double q[4] = {0.0, 0.0, 0.0, 0.0};
    const double* __restrict__ dr;
    const double* __restrict__ rl;  // original row bounds, +-inf = none
    const double* __restrict__ ru;
    const TX* __restrict__ yplus;
    __device__ Pre prefetch(int i) const { return Pre{__ldg(dr + i), __ldg(rl + i), __ldg(ru + i), yplus[i]}; }
    __device__ void row(int i, double ax_s, const Pre& p) {
        const double ax = ax_s / p.d;
        const double lo = p.lo, hi = p.hi;
        double v = 0.0, b = 0.0;
        if (ax < lo) {
            v = ax - lo;
            b = lo;
        } else if (ax > hi) {
            v = ax - hi;
            b = hi;
        }
        q[0] += v * v;
        if (v != 0.0) q[3] = fmax(q[3], fabs(v) / (1.0 + fabs(b)));
        const double yi = double(p.y) * p.d;
        if (yi > 0.0) {
            if (isfinite(lo)) q[1] += lo * yi;
            else q[2] += yi * yi;
        } else if (yi < 0.0) {
            if (isfinite(hi)) q[1] += hi * yi;
            else q[2] += yi * yi;
        }
    }
};

// Columns (rows of A') at (x+, y+): dual residual after the bound
// multipliers absorb what they can, their dual-objective terms, the
// primal objective and column-box violations, in the original space.
template <typename TX>
struct KktColEpi {
    static constexpr int NQ = 4;
    static constexpr bool kLastIsMax = false;
    struct Pre {
        double d, c, lo, hi;
        TX x;
    };
    double q[4] = {0.0, 0.0, 0.0, 0.0};
    const double* __restrict__ dc;
    const double* __restrict__ c;   // original cost
    const double* __restrict__ l;   // original column bounds, +-inf = none
    const double* __restrict__ u;
    const TX* __restrict__ xplus;
    __device__ Pre prefetch(int j) const {
        return Pre{__ldg(dc + j), __ldg(c + j), __ldg(l + j), __ldg(u + j), xplus[j]};
    }
    __device__ void row(int j, double aty_s, const Pre& p) {
        const double rc = p.c - aty_s / p.d;
        const double lo = p.lo, hi = p.hi;
        double lam = 0.0;
        if (rc > 0.0 && isfinite(lo)) lam = rc;
        if (rc < 0.0 && isfinite(hi)) lam = rc;
        const double r = rc - lam;
        q[0] += r * r;
        if (lam > 0.0) q[1] += lo * lam;
        else if (lam < 0.0) q[1] += hi * lam;
        const double xj = double(p.x) * p.d;
        q[2] += p.c * xj;
        double xv = 0.0;
        if (xj < lo) xv = xj - lo;
        else if (xj > hi) xv = xj - hi;
        q[3] += xv * xv;
    }
};

// ---------------------------------------------------------------- controller

struct CtlArgs {
    const double* partP;   // primal kernel partials, 2 x nP
    const double* partD;   // dual kernel partials, 2 x nD
    const double* partKR;  // KKT row partials, 4 x nKR
    const double* partKC;  // KKT column partials, 4 x nKC
    int nP, nD, nKR, nKC;  // grids of the kernels that wrote them
    double offset;
    double tol, feas_tol;
    int K;
    int restarts_on;       // PDLP
    int mixed;             // FP32 phase may hand over to FP64
    int phase;
    double suff, nec, art, theta;
    int polish_stall;
    double polish_switch;
    int anchor_at_restart; // 1: the residual at a restart becomes the new anchor
    double weight_decades; // primal weight stays within this many decades of its start
    double* hist;          // ring of kHist entries x 8 doubles
};

constexpr int kHist = 4096;

// The scalar part of a check (thread 0 only): relative KKT in the original
// space, termination, FP32->FP64 hand-over, fixed-point-residual restart
// test and primal-weight update.  Shared by the single-LP controller and
// the per-instance batch controller.
struct CtlSums {
    double dx2, dxa2, dy2, dya2, pres2, dobj_r, ywrong2, maxrel, dres2, dobj_c, pobj_c, xviol2;
};

// Relative KKT error in the original space from the KKT kernels' sums:
// primal residual (rows and column bounds) over 1 + ||b||, dual residual
// (reduced costs of the wrong sign and row duals of the wrong sign) over
// 1 + ||c||, and the relative duality gap.
struct KktVal {
    double kkt, kp, kd, kg, pobj, dobj;
};

__device__ inline KktVal kkt_from_sums(const CtlSums& s, double bnorm, double cnorm, double offset) {
    KktVal k;
    k.pobj = s.pobj_c + offset;
    k.dobj = s.dobj_r + s.dobj_c + offset;
    k.kp = sqrt(s.pres2 + s.xviol2) / (1.0 + bnorm);
    k.kd = sqrt(s.dres2 + s.ywrong2) / (1.0 + cnorm);
    k.kg = fabs(k.pobj - k.dobj) / (1.0 + fabs(k.pobj) + fabs(k.dobj));
    k.kkt = fmax(k.kp, fmax(k.kd, k.kg));
    return k;
}

__device__ void control_update(const CtlArgs& a, DevState* st, const CtlSums& sums, double bnorm, double cnorm,
                               double offset, double* hist) {
    const double dx2 = sums.dx2, dxa2 = sums.dxa2, dy2 = sums.dy2, dya2 = sums.dya2;
    const double maxrel = sums.maxrel;

    const long long it = st->iter + a.K;
    st->iter = it;
    const KktVal kv = kkt_from_sums(sums, bnorm, cnorm, offset);
    const double pobj = kv.pobj, dobj = kv.dobj, kp = kv.kp, kd = kv.kd, kg = kv.kg, kkt = kv.kkt;
    const double omega = st->omega;
    const double res = sqrt(omega * dx2 + dy2 / omega);
    st->kkt = kkt;
    st->kp = kp;
    st->kd = kd;
    st->kg = kg;
    st->pobj = pobj;
    st->dobj = dobj;
    st->max_rel_row = maxrel;
    st->res = res;
    st->kkt_iter = it;
    st->apply_restart = 0;
    if (hist) {
        double* h = hist + 8 * ((it / a.K) % kHist);
        h[0] = double(it);
        h[1] = kkt;
        h[2] = kp;
        h[3] = kd;
        h[4] = kg;
        h[5] = res;
        h[6] = omega;
        h[7] = double(a.phase);
    }
    if (!isfinite(kkt) || !isfinite(res)) {
        st->done = 1;
        st->status = 11;  // NIR_STATUS_NUMERICAL_TROUBLE
        return;
    }
    if (kkt <= a.tol && (a.feas_tol <= 0.0 || maxrel <= a.feas_tol)) {
        st->done = 1;
        st->status = 0;
        return;
    }
    if (it >= st->max_iters) {
        st->done = 1;
        st->status = 6;
        return;
    }
    // hand over from FP32 to the FP64 polish when FP32 stops improving
    if (a.mixed) {
        if (kkt < 0.8 * st->best_kkt) {
            st->best_kkt = kkt;
            st->stall = 0;
        } else {
            st->stall += 1;
        }
        // a plateau counts as a stall once it has lasted polish_stall
        // checks and half of the checks so far, within a factor 30 of the
        // tolerance: PDLP's own plateaus grow with its restart lengths (an
        // artificial restart at 0.36 of the iterations so far) and sit at
        // any KKT level, while the rounding of the FP32 matrix values
        // (2^-24 relative) shows only near the tolerance.  A hand-over
        // inside an ordinary plateau only slows the solve down: on the
        // power-law LP the FP32-value phase converges by itself in the same
        // iterations, and a rule that also handed over after a plateau of
        // three quarters of the run at any level fired there at 19,000 of
        // 155,000 iterations.
        const long long checks = it / max(a.K, 1);
        const bool near = st->stall >= max((long long)a.polish_stall, checks / 2) && kkt <= 30.0 * a.tol;
        if (near || kkt <= a.polish_switch) {
            st->switch_request = 1;
            st->phase = 1;
            return;
        }
    }
    if (!a.restarts_on) {
        st->k_base += a.K;
        return;
    }
    // fixed-point-residual restart test
    const long long k_after = st->k_base + a.K;
    bool restart = false;
    const double it_phase = double(it - st->it_phase);
    if (!st->have_anchor) {
        st->r_anchor = res;
        st->have_anchor = 1;
        st->r_prev = res;
        restart = (double(k_after) >= a.art * it_phase);
    } else {
        restart = (res <= a.suff * st->r_anchor) || (res <= a.nec * st->r_anchor && res > st->r_prev) ||
                  (double(k_after) >= a.art * it_phase);
        st->r_prev = res;
    }
    if (restart) {
        const double dxa = sqrt(dxa2), dya = sqrt(dya2);
        if (dxa > 1e-10 && dya > 1e-10 && isfinite(dxa) && isfinite(dya)) {
            // log-space smoothing toward ||dy||/||dx||, with two guards
            // against a runaway (a primal pinned at its bounds makes dx tiny,
            // a larger weight shrinks the primal step further): at most a
            // factor 10 per restart, and within `weight_decades` decades of
            // the initial weight
            const double lo = log(omega) - 2.302585092994046, hi = log(omega) + 2.302585092994046;
            double lw = a.theta * log(dya / dxa) + (1.0 - a.theta) * log(omega);
            lw = fmin(fmax(lw, lo), hi);
            const double span = 2.302585092994046 * a.weight_decades;
            lw = fmin(fmax(lw, st->log_omega0 - span), st->log_omega0 + span);
            st->omega = exp(lw);
        }
        st->tau = st->eta / st->omega;
        st->sigma = st->eta * st->omega;
        st->apply_restart = 1;
        st->restarts += 1;
        st->k_base = 0;
        // the new anchor is z+ = T(z); ||z+ - T(z+)|| <= ||z - T(z)|| = res
        st->have_anchor = a.anchor_at_restart;
        st->r_anchor = res;
        st->r_prev = res;
    } else {
        st->k_base = k_after;
    }
}


__global__ void __launch_bounds__(kBlock) k_control(CtlArgs a, DevState* st) {
    __shared__ double sh[kWarps];
    if (st->done || st->phase != a.phase) return;
    const double dx2 = block_sum_array(a.partP, a.nP, sh);
    const double dxa2 = block_sum_array(a.partP + a.nP, a.nP, sh);
    const double dy2 = block_sum_array(a.partD, a.nD, sh);
    const double dya2 = block_sum_array(a.partD + a.nD, a.nD, sh);
    const double pres2 = block_sum_array(a.partKR, a.nKR, sh);
    const double dobj_r = block_sum_array(a.partKR + a.nKR, a.nKR, sh);
    const double ywrong2 = block_sum_array(a.partKR + 2 * a.nKR, a.nKR, sh);
    const double maxrel = block_max_array(a.partKR + 3 * a.nKR, a.nKR, sh);
    const double dres2 = block_sum_array(a.partKC, a.nKC, sh);
    const double dobj_c = block_sum_array(a.partKC + a.nKC, a.nKC, sh);
    const double pobj_c = block_sum_array(a.partKC + 2 * a.nKC, a.nKC, sh);
    const double xviol2 = block_sum_array(a.partKC + 3 * a.nKC, a.nKC, sh);
    if (threadIdx.x != 0) return;
    const CtlSums sums{dx2, dxa2, dy2, dya2, pres2, dobj_r, ywrong2, maxrel, dres2, dobj_c, pobj_c, xviol2};
    control_update(a, st, sums, st->bnorm, st->cnorm, a.offset, a.hist);
}

// KKT probe of the reference loop (after a chunk's KKT kernels): records
// the relative KKT of the current iterate and the first iteration at which
// it is at most tol.  Reads the iterate only.
__global__ void __launch_bounds__(kBlock) k_ref_probe(const double* __restrict__ partKR, int nKR,
                                                      const double* __restrict__ partKC, int nKC, double bnorm,
                                                      double cnorm, double offset, double tol, DevState* st) {
    __shared__ double sh[kWarps];
    if (st->done) return;  // the KKT kernels skipped this chunk
    CtlSums s{};
    s.pres2 = block_sum_array(partKR, nKR, sh);
    s.dobj_r = block_sum_array(partKR + nKR, nKR, sh);
    s.ywrong2 = block_sum_array(partKR + 2 * nKR, nKR, sh);
    s.maxrel = block_max_array(partKR + 3 * nKR, nKR, sh);
    s.dres2 = block_sum_array(partKC, nKC, sh);
    s.dobj_c = block_sum_array(partKC + nKC, nKC, sh);
    s.pobj_c = block_sum_array(partKC + 2 * nKC, nKC, sh);
    s.xviol2 = block_sum_array(partKC + 3 * nKC, nKC, sh);
    if (threadIdx.x != 0) return;
    const KktVal k = kkt_from_sums(s, bnorm, cnorm, offset);
    st->kkt = k.kkt;
    st->kp = k.kp;
    st->kd = k.kd;
    st->kg = k.kg;
    st->pobj = k.pobj;
    st->dobj = k.dobj;
    st->max_rel_row = s.maxrel;
    st->kkt_iter = st->iter;
    if (st->probe_hit < 0 && k.kkt <= tol) st->probe_hit = st->iter;
}

// Restart: the anchor and the iterate become (x+, y+).
template <typename T>
__global__ void k_apply_restart(int n, int m, const DevState* __restrict__ st, int phase, T* __restrict__ x,
                                T* __restrict__ x0, const T* __restrict__ xplus, T* __restrict__ y,
                                T* __restrict__ y0, const T* __restrict__ yplus) {
    if (!st->apply_restart || st->done || st->phase != phase) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) {
        const T v = xplus[t];
        x[t] = v;
        x0[t] = v;
    }
    if (t < m) {
        const T v = yplus[t];
        y[t] = v;
        y0[t] = v;
    }
}

}  // namespace nir
