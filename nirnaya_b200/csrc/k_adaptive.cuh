// The hot path: CSR-adaptive SpMV over row blocks with the PDHG update
// fused into its epilogue.
//
// A matrix orientation (A, or the stored transpose A') is cut into row
// blocks holding at most `cap` nonzeros (one row per block if the row is
// longer).  One CUDA block of kBlock threads takes one row block:
//  * several rows: the block streams the row block's index/value pairs
//    with consecutive threads on consecutive nonzeros (coalesced), forms the
//    products val*x[col] into shared memory, then teams of T threads (T a
//    power of two <= 32 chosen from the row count) reduce one row each by a
//    fixed shuffle tree and the team leader runs the epilogue for that row;
//  * one long row: all threads stride over it and a block tree reduces.
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

namespace nir {

// ---------------------------------------------------------------- core

template <typename TA, typename TV, typename TX, class Epi>
__device__ __forceinline__ void rowblock_spmv(const int* __restrict__ blk, const int* __restrict__ rp,
                                              const int* __restrict__ ci, const TV* __restrict__ val,
                                              const TX* __restrict__ x, Epi& epi, TA* s_prod, TA* s_red) {
    const int b = blockIdx.x;
    const int tid = threadIdx.x;
    const int r0 = blk[b], r1 = blk[b + 1];
    const int nrows = r1 - r0;
    const int p0 = rp[r0], p1 = rp[r1];
    const int nnzb = p1 - p0;
    if (nrows == 1) {
        TA s = TA(0);
        int k = p0 + tid;
        for (; k + 3 * kBlock < p1; k += 4 * kBlock) {
            int c0 = __ldg(ci + k), c1 = __ldg(ci + k + kBlock), c2 = __ldg(ci + k + 2 * kBlock),
                c3 = __ldg(ci + k + 3 * kBlock);
            TV v0 = __ldg(val + k), v1 = __ldg(val + k + kBlock), v2 = __ldg(val + k + 2 * kBlock),
               v3 = __ldg(val + k + 3 * kBlock);
            TA a0 = TA(v0) * TA(__ldg(x + c0)), a1 = TA(v1) * TA(__ldg(x + c1));
            TA a2 = TA(v2) * TA(__ldg(x + c2)), a3 = TA(v3) * TA(__ldg(x + c3));
            s += (a0 + a1) + (a2 + a3);
        }
        for (; k < p1; k += kBlock) s += TA(__ldg(val + k)) * TA(__ldg(x + __ldg(ci + k)));
        s = block_sum(s, s_red);
        if (tid == 0) epi.row(r0, s);
        return;
    }
    // stage the products of the whole row block
    {
        int k = tid;
        for (; k + 3 * kBlock < nnzb; k += 4 * kBlock) {
            int c0 = __ldg(ci + p0 + k), c1 = __ldg(ci + p0 + k + kBlock), c2 = __ldg(ci + p0 + k + 2 * kBlock),
                c3 = __ldg(ci + p0 + k + 3 * kBlock);
            TV v0 = __ldg(val + p0 + k), v1 = __ldg(val + p0 + k + kBlock), v2 = __ldg(val + p0 + k + 2 * kBlock),
               v3 = __ldg(val + p0 + k + 3 * kBlock);
            TX x0 = __ldg(x + c0), x1 = __ldg(x + c1), x2 = __ldg(x + c2), x3 = __ldg(x + c3);
            s_prod[k] = TA(v0) * TA(x0);
            s_prod[k + kBlock] = TA(v1) * TA(x1);
            s_prod[k + 2 * kBlock] = TA(v2) * TA(x2);
            s_prod[k + 3 * kBlock] = TA(v3) * TA(x3);
        }
        for (; k < nnzb; k += kBlock) s_prod[k] = TA(__ldg(val + p0 + k)) * TA(__ldg(x + __ldg(ci + p0 + k)));
    }
    __syncthreads();
    // team size: largest power of two <= kBlock / nrows, at most 32
    int T = 32;
    while (T > 1 && T * nrows > kBlock) T >>= 1;
    const int team = tid / T, lane = tid & (T - 1), nteams = kBlock / T;
    const int rounds = (nrows + nteams - 1) / nteams;  // uniform across the block
    for (int q = 0; q < rounds; ++q) {
        const int r = r0 + q * nteams + team;
        TA s = TA(0);
        if (r < r1) {
            const int a = rp[r] - p0, e = rp[r + 1] - p0;
            for (int k = a + lane; k < e; k += T) s += s_prod[k];
        }
        for (int o = T >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0 && r < r1) epi.row(r, s);
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

template <typename TA>
__device__ __forceinline__ TA* smem_products() {
    extern __shared__ __align__(16) unsigned char nir_smem[];
    return reinterpret_cast<TA*>(nir_smem);
}

// ---------------------------------------------------------------- plain SpMV

template <typename TA>
struct PlainEpi {
    static constexpr int NQ = 0;
    static constexpr bool kLastIsMax = false;
    double q[1];
    TA* y;
    __device__ void row(int r, TA s) { y[r] = s; }
};

template <typename TA, typename TV, typename TX>
__global__ void __launch_bounds__(kBlock) k_spmv_adaptive(const int* __restrict__ blk, const int* __restrict__ rp,
                                                          const int* __restrict__ ci, const TV* __restrict__ val,
                                                          const TX* __restrict__ x, TA* __restrict__ y) {
    __shared__ TA s_red[kWarps];
    PlainEpi<TA> epi;
    epi.y = y;
    rowblock_spmv<TA, TV, TX>(blk, rp, ci, val, x, epi, smem_products<TA>(), s_red);
}

// ---------------------------------------------------------------- PDHG step

// Scalars every iteration kernel needs, derived from DevState at launch.
template <typename T>
struct StepScalars {
    T tau, sigma, w, onemw, rho;
};

template <typename T>
__device__ __forceinline__ StepScalars<T> step_scalars(const DevState* st, int i_in_chunk, int halpern, double rho) {
    StepScalars<T> s;
    s.tau = T(st->tau);
    s.sigma = T(st->sigma);
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
    __device__ void row(int j, T aty) {
        const T xj = x[j];
        const T xp = clamp_box(xj - s.tau * (c[j] - aty), lo[j], up[j]);
        xbar[j] = T(2) * xp - xj;
        T xn = xp;
        T a0 = T(0);
        if (halpern) {
            a0 = x0[j];
            xn = s.w * ((T(1) + s.rho) * xp - s.rho * xj) + s.onemw * a0;
        }
        x[j] = xn;
        if (CHECK) {
            xplus[j] = xp;
            const double d = double(xj) - double(xp);
            const double e = double(xp) - double(halpern ? a0 : x0[j]);
            q[0] += d * d;
            q[1] += e * e;
        }
    }
};

template <typename T, bool CHECK>
struct DualEpi {
    static constexpr int NQ = CHECK ? 2 : 0;
    static constexpr bool kLastIsMax = false;
    double q[2] = {0.0, 0.0};
    T* __restrict__ y;
    T* __restrict__ yplus;
    const T* __restrict__ rl;
    const T* __restrict__ ru;
    const T* __restrict__ y0;
    StepScalars<T> s;
    int halpern;
    __device__ void row(int i, T ax) {
        const T yi = y[i];
        const T p = clamp_box(ax - yi / s.sigma, rl[i], ru[i]);
        const T yp = yi + s.sigma * (p - ax);
        T yn = yp;
        T a0 = T(0);
        if (halpern) {
            a0 = y0[i];
            yn = s.w * ((T(1) + s.rho) * yp - s.rho * yi) + s.onemw * a0;
        }
        y[i] = yn;
        if (CHECK) {
            yplus[i] = yp;
            const double d = double(yi) - double(yp);
            const double e = double(yp) - double(halpern ? a0 : y0[i]);
            q[0] += d * d;
            q[1] += e * e;
        }
    }
};

struct IterArgs {
    const int* blk;
    const int* rp;
    const int* ci;
    double* part;
    const DevState* st;
    int i_in_chunk;
    int halpern;
    int phase;     // the kernel runs only while st->phase == phase
    double rho;
};

template <typename T, bool CHECK>
__global__ void __launch_bounds__(kBlock) k_primal(IterArgs a, const T* __restrict__ val, const T* __restrict__ y,
                                                   T* __restrict__ x, T* __restrict__ xbar, T* __restrict__ xplus,
                                                   const T* __restrict__ c, const T* __restrict__ lo,
                                                   const T* __restrict__ up, const T* __restrict__ x0) {
    __shared__ double s_red[kWarps];
    if (a.st->done || a.st->phase != a.phase) return;
    PrimalEpi<T, CHECK> epi;
    epi.x = x;
    epi.xbar = xbar;
    epi.xplus = xplus;
    epi.c = c;
    epi.lo = lo;
    epi.up = up;
    epi.x0 = x0;
    epi.s = step_scalars<T>(a.st, a.i_in_chunk, a.halpern, a.rho);
    epi.halpern = a.halpern;
    rowblock_spmv<T, T, T>(a.blk, a.rp, a.ci, val, y, epi, smem_products<T>(), reinterpret_cast<T*>(s_red));
    if (CHECK) write_partials(epi, a.part, s_red);
}

template <typename T, bool CHECK>
__global__ void __launch_bounds__(kBlock) k_dual(IterArgs a, const T* __restrict__ val, const T* __restrict__ xbar,
                                                 T* __restrict__ y, T* __restrict__ yplus, const T* __restrict__ rl,
                                                 const T* __restrict__ ru, const T* __restrict__ y0) {
    __shared__ double s_red[kWarps];
    if (a.st->done || a.st->phase != a.phase) return;
    DualEpi<T, CHECK> epi;
    epi.y = y;
    epi.yplus = yplus;
    epi.rl = rl;
    epi.ru = ru;
    epi.y0 = y0;
    epi.s = step_scalars<T>(a.st, a.i_in_chunk, a.halpern, a.rho);
    epi.halpern = a.halpern;
    rowblock_spmv<T, T, T>(a.blk, a.rp, a.ci, val, xbar, epi, smem_products<T>(), reinterpret_cast<T*>(s_red));
    if (CHECK) write_partials(epi, a.part, s_red);
}

// ---------------------------------------------------------------- KKT (FP64)

// Rows of A at (x+, y+): primal residual, dual-objective row terms,
// wrong-sign multipliers and the checker's relative row violation, all in
// the original (unscaled) space.  ax is (A_scaled x_scaled)_i = dr_i (A x)_i.
template <typename TX>
struct KktRowEpi {
    static constexpr int NQ = 4;
    static constexpr bool kLastIsMax = true;
    double q[4] = {0.0, 0.0, 0.0, 0.0};
    const double* __restrict__ dr;
    const double* __restrict__ rl;  // original row bounds, +-inf = none
    const double* __restrict__ ru;
    const TX* __restrict__ yplus;
    __device__ void row(int i, double ax_s) {
        const double d = dr[i];
        const double ax = ax_s / d;
        const double lo = rl[i], hi = ru[i];
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
        const double yi = double(yplus[i]) * d;
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
    double q[4] = {0.0, 0.0, 0.0, 0.0};
    const double* __restrict__ dc;
    const double* __restrict__ c;   // original cost
    const double* __restrict__ l;   // original column bounds, +-inf = none
    const double* __restrict__ u;
    const TX* __restrict__ xplus;
    __device__ void row(int j, double aty_s) {
        const double d = dc[j];
        const double rc = c[j] - aty_s / d;
        const double lo = l[j], hi = u[j];
        double lam = 0.0;
        if (rc > 0.0 && isfinite(lo)) lam = rc;
        if (rc < 0.0 && isfinite(hi)) lam = rc;
        const double r = rc - lam;
        q[0] += r * r;
        if (lam > 0.0) q[1] += lo * lam;
        else if (lam < 0.0) q[1] += hi * lam;
        const double xj = double(xplus[j]) * d;
        q[2] += c[j] * xj;
        double xv = 0.0;
        if (xj < lo) xv = xj - lo;
        else if (xj > hi) xv = xj - hi;
        q[3] += xv * xv;
    }
};

struct KktArgs {
    const int* blk;
    const int* rp;
    const int* ci;
    const double* val;  // scaled FP64 values
    double* part;
    const DevState* st;
    int phase;
};

template <typename TX>
__global__ void __launch_bounds__(kBlock) k_kkt_rows(KktArgs a, const TX* __restrict__ xplus, const TX* __restrict__ yplus,
                                                     const double* __restrict__ dr, const double* __restrict__ rl,
                                                     const double* __restrict__ ru) {
    __shared__ double s_red[kWarps];
    if (a.st->done || a.st->phase != a.phase) return;
    KktRowEpi<TX> epi;
    epi.dr = dr;
    epi.rl = rl;
    epi.ru = ru;
    epi.yplus = yplus;
    rowblock_spmv<double, double, TX>(a.blk, a.rp, a.ci, a.val, xplus, epi, smem_products<double>(), s_red);
    write_partials(epi, a.part, s_red);
}

template <typename TX>
__global__ void __launch_bounds__(kBlock) k_kkt_cols(KktArgs a, const TX* __restrict__ xplus, const TX* __restrict__ yplus,
                                                     const double* __restrict__ dc, const double* __restrict__ c,
                                                     const double* __restrict__ l, const double* __restrict__ u) {
    __shared__ double s_red[kWarps];
    if (a.st->done || a.st->phase != a.phase) return;
    KktColEpi<TX> epi;
    epi.dc = dc;
    epi.c = c;
    epi.l = l;
    epi.u = u;
    epi.xplus = xplus;
    rowblock_spmv<double, double, TX>(a.blk, a.rp, a.ci, a.val, yplus, epi, smem_products<double>(), s_red);
    write_partials(epi, a.part, s_red);
}

// ---------------------------------------------------------------- controller

struct CtlArgs {
    const double* partP;   // primal kernel partials, 2 x nP
    const double* partD;   // dual kernel partials, 2 x nD
    const double* partKR;  // KKT row partials, 4 x nD
    const double* partKC;  // KKT column partials, 4 x nP
    int nP, nD;
    double bnorm, cnorm, offset;
    double tol, feas_tol;
    int K;
    int restarts_on;       // PDLP
    int mixed;             // FP32 phase may hand over to FP64
    int phase;
    double suff, nec, art, theta;
    int polish_stall;
    double polish_switch;
    double* hist;          // ring of kHist entries x 8 doubles
};

constexpr int kHist = 4096;

__global__ void __launch_bounds__(kBlock) k_control(CtlArgs a, DevState* st) {
    __shared__ double sh[kWarps];
    if (st->done || st->phase != a.phase) return;
    const double dx2 = block_sum_array(a.partP, a.nP, sh);
    const double dxa2 = block_sum_array(a.partP + a.nP, a.nP, sh);
    const double dy2 = block_sum_array(a.partD, a.nD, sh);
    const double dya2 = block_sum_array(a.partD + a.nD, a.nD, sh);
    const double pres2 = block_sum_array(a.partKR, a.nD, sh);
    const double dobj_r = block_sum_array(a.partKR + a.nD, a.nD, sh);
    const double ywrong2 = block_sum_array(a.partKR + 2 * a.nD, a.nD, sh);
    const double maxrel = block_max_array(a.partKR + 3 * a.nD, a.nD, sh);
    const double dres2 = block_sum_array(a.partKC, a.nP, sh);
    const double dobj_c = block_sum_array(a.partKC + a.nP, a.nP, sh);
    const double pobj_c = block_sum_array(a.partKC + 2 * a.nP, a.nP, sh);
    const double xviol2 = block_sum_array(a.partKC + 3 * a.nP, a.nP, sh);
    if (threadIdx.x != 0) return;

    const long long it = st->iter + a.K;
    st->iter = it;
    const double pobj = pobj_c + a.offset;
    const double dobj = dobj_r + dobj_c + a.offset;
    const double kp = sqrt(pres2 + xviol2) / (1.0 + a.bnorm);
    const double kd = sqrt(dres2 + ywrong2) / (1.0 + a.cnorm);
    const double kg = fabs(pobj - dobj) / (1.0 + fabs(pobj) + fabs(dobj));
    const double kkt = fmax(kp, fmax(kd, kg));
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
    {
        double* h = a.hist + 8 * ((it / a.K) % kHist);
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
        if (st->stall >= a.polish_stall || kkt <= a.polish_switch) {
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
    if (!st->have_anchor) {
        st->r_anchor = res;
        st->have_anchor = 1;
        st->r_prev = res;
        restart = (double(k_after) >= a.art * double(it));
    } else {
        restart = (res <= a.suff * st->r_anchor) || (res <= a.nec * st->r_anchor && res > st->r_prev) ||
                  (double(k_after) >= a.art * double(it));
        st->r_prev = res;
    }
    if (restart) {
        const double dxa = sqrt(dxa2), dya = sqrt(dya2);
        if (dxa > 1e-10 && dya > 1e-10 && isfinite(dxa) && isfinite(dya)) {
            const double lw = a.theta * log(dya / dxa) + (1.0 - a.theta) * log(omega);
            st->omega = exp(lw);
        }
        st->tau = st->eta / st->omega;
        st->sigma = st->eta * st->omega;
        st->apply_restart = 1;
        st->restarts += 1;
        st->k_base = 0;
        st->have_anchor = 0;
    } else {
        st->k_base = k_after;
    }
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
