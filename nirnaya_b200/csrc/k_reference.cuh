// Kernels of NIR_ALGO_REFERENCE: the reference PDHG loop
// (src/gpu/pdhg_solver.hpp:33-105) in FP64 with the reference's exact
// arithmetic.  Every sum runs in the reference's order on one thread
// (CscMatrix::spmv adds a row's terms in ascending column order, the
// transpose adds a column's terms in ascending row order,
// src/core/csc_matrix.hpp:99-120), and every product and sum is a separate
// correctly rounded operation (__dmul_rn/__dadd_rn: no contraction into
// FMA, as the reference is compiled without it).  The results are
// bit-identical to the reference's.
#pragma once

#include "dev_common.cuh"

namespace nir {

// y[r] = sum_k v[k] * x[ci[k]] over row r, sequentially from +0.0.
__global__ void k_ref_spmv(int rows, const int* __restrict__ rp, const int* __restrict__ ci,
                           const double* __restrict__ v, const double* __restrict__ x, double* __restrict__ y) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    double s = 0.0;
    for (int k = rp[r]; k < rp[r + 1]; ++k) s = __dadd_rn(s, __dmul_rn(v[k], x[ci[k]]));
    y[r] = s;
}

// Power-iteration norm, src/gpu/pdhg_solver.hpp:38-41: one thread adds
// u_j^2 in index order, then norm_est = sqrt(max(1e-12, n2)).
__global__ void k_ref_norm(int n, const double* __restrict__ u, DevState* st) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double n2 = 0.0;
    for (int j = 0; j < n; ++j) n2 = __dadd_rn(n2, __dmul_rn(u[j], u[j]));
    st->ref_norm_est = __dsqrt_rn(smax(1e-12, n2));
}

__global__ void k_ref_div(int n, double* __restrict__ u, const DevState* __restrict__ st) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) u[j] = __ddiv_rn(u[j], st->ref_norm_est);
}

// Fixed steps, src/gpu/pdhg_solver.hpp:43-45.
__global__ void k_ref_steps(DevState* st) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double sigma_max = __dsqrt_rn(st->ref_norm_est);
    double s = __ddiv_rn(0.85, smax(1e-6, sigma_max));
    st->tau = s;
    st->sigma = s;
}

// Box-midpoint start, src/gpu/pdhg_solver.hpp:47-57.
__global__ void k_ref_init(int n, int m, const double* __restrict__ lo, const double* __restrict__ up,
                           double* __restrict__ x, double* __restrict__ y) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) {
        double l = lo[t], u = up[t], v = 0.0;
        if (fin_bound(l) && fin_bound(u)) v = __dmul_rn(0.5, __dadd_rn(l, u));
        else if (fin_bound(l)) v = smax(0.0, l);
        else if (fin_bound(u)) v = smin(0.0, u);
        x[t] = v;
    }
    if (t < m) y[t] = 0.0;
}

// Primal step, src/gpu/pdhg_solver.hpp:69-78, one thread per column j
// (row j of the stored transpose).
__global__ void k_ref_primal(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                             const double* __restrict__ v, const double* __restrict__ y,
                             const double* __restrict__ cost, const double* __restrict__ lo,
                             const double* __restrict__ up, double* __restrict__ x, double* __restrict__ xbar,
                             const DevState* __restrict__ st, int i_in_chunk) {
    if (st->done || st->iter + i_in_chunk >= st->max_iters) return;
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    double s = 0.0;
    for (int k = rp[j]; k < rp[j + 1]; ++k) s = __dadd_rn(s, __dmul_rn(v[k], y[ci[k]]));
    const double tau = st->tau;
    double xj = x[j];
    double cand = __dsub_rn(xj, __dmul_rn(tau, __dsub_rn(cost[j], s)));
    if (fin_bound(lo[j])) cand = smax(lo[j], cand);
    if (fin_bound(up[j])) cand = smin(up[j], cand);
    xbar[j] = __dsub_rn(__dmul_rn(2.0, cand), xj);
    x[j] = cand;
}

// Dual step and the row-violation maximum, src/gpu/pdhg_solver.hpp:80-95,
// one thread per row.  Each block writes its violation maximum to part[].
__global__ void k_ref_dual(int m, const int* __restrict__ rp, const int* __restrict__ ci,
                           const double* __restrict__ v, const double* __restrict__ xbar,
                           const double* __restrict__ rlo, const double* __restrict__ rup, double* __restrict__ y,
                           double* __restrict__ part, const DevState* __restrict__ st, int i_in_chunk) {
    __shared__ double sh[kWarps];
    if (st->done || st->iter + i_in_chunk >= st->max_iters) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double viol = 0.0;
    if (i < m) {
        double a = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k) a = __dadd_rn(a, __dmul_rn(v[k], xbar[ci[k]]));
        const double sigma = st->sigma;
        double yi = y[i];
        double r = __dsub_rn(a, __ddiv_rn(yi, sigma));
        double lo = rlo[i], hi = rup[i];
        if (fin_bound(lo)) r = smax(lo, r);
        if (fin_bound(hi)) r = smin(hi, r);
        y[i] = __dadd_rn(yi, __dmul_rn(sigma, __dsub_rn(r, a)));
        if (fin_bound(lo)) viol = smax(viol, __dsub_rn(lo, a));
        if (fin_bound(hi)) viol = smax(viol, __dsub_rn(a, hi));
    }
    // max is order-independent, so the tree gives the reference's value
    double bm = block_max(viol, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = bm;
}

// Stop test after iteration `it`, src/gpu/pdhg_solver.hpp:97-100, and the
// iteration count of PdhgResult (iterations = it + 1 at a stop, max_iters
// at the cap).  Launched after every dual step; the last one of a chunk of
// K iterations advances st->iter.
__global__ void k_ref_stop(const double* __restrict__ part, int nblk, DevState* st, int i_in_chunk, int K) {
    __shared__ double sh[kWarps];
    if (st->done) return;
    const long long it = st->iter + i_in_chunk;
    if (it >= st->max_iters) return;
    const bool test = (it > 20) && ((it & 31) == 0);
    double mx = 0.0;
    if (test) mx = block_max_array(part, nblk, sh);
    if (threadIdx.x != 0) return;
    if (test && mx <= 1e-6) {
        st->done = 1;
        st->ref_stopped = 1;
        st->status = 0;
        st->ref_iterations = it + 1;
        return;
    }
    if (it + 1 >= st->max_iters) {
        st->done = 1;
        st->status = 6;  // NIR_STATUS_ITERATION_LIMIT
        st->ref_iterations = st->max_iters;
        return;
    }
    if (i_in_chunk == K - 1) {
        st->iter += K;
        st->ref_iterations = st->iter;
    }
}

}  // namespace nir
