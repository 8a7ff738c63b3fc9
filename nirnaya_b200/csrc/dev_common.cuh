// Device-side common definitions of the PDHG engine.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace nir {

constexpr int kBlock = 256;      // threads per block of every iteration kernel
constexpr int kWarps = kBlock / 32;
constexpr int kMaxQ = 6;         // per-block partial quantities a kernel may emit

// The reference's `is_finite_bound` (src/core/types.hpp:49-51).
__host__ __device__ inline bool fin_bound(double b) { return isfinite(b) && fabs(b) < 1e20; }

// std::max(a, b) / std::min(a, b) with their exact tie and signed-zero
// behaviour: max returns a unless a < b, min returns a unless b < a.
__host__ __device__ inline double smax(double a, double b) { return (a < b) ? b : a; }
__host__ __device__ inline double smin(double a, double b) { return (b < a) ? b : a; }

template <typename T>
__device__ inline T clamp_box(T v, T lo, T hi) {  // lo/hi may be +-inf
    return fmin(fmax(v, lo), hi);
}

// Solver state kept on the device.  The controller kernel (one block) is
// the only writer during a solve; iteration kernels only read it.
struct DevState {
    // step sizes and weight (FP64)
    double eta, omega, tau, sigma;
    double log_omega0;     // log of the initial primal weight (bounds the updates)
    long long it_phase;    // iteration at which the current phase began
    // restart bookkeeping
    long long iter;        // completed iterations
    long long k_base;      // Halpern inner count at the start of the current chunk
    long long max_iters;
    double r_anchor;       // fixed-point residual measured after the last restart
    double r_prev;
    int have_anchor;
    int apply_restart;     // set by the controller for the restart kernel of this check
    int restarts;
    // termination
    int done;              // 1 = stop iterating (status holds why)
    int status;            // NIR_STATUS_*
    int phase;             // 0 = primary precision, 1 = FP64 polish
    int switch_request;    // controller asks the host to switch to the FP64 phase
    int stall;             // checks without a 0.8x KKT improvement
    double best_kkt;
    // last KKT evaluation (original space)
    double kkt, kp, kd, kg, pobj, dobj, max_rel_row;
    double res;            // last fixed-point residual
    long long kkt_iter;
    // reference-algorithm scalars
    double ref_norm_est;
    long long ref_iterations;
    int ref_stopped;
    int pad_;
    long long probe_hit;   // reference loop: first probed iteration with rel KKT <= tol (-1: none yet)
    double bnorm, cnorm;   // ||b||, ||c|| of the original LP: the relative KKT's denominators
};

// Deterministic block-wide sum / max over kBlock threads: a fixed shuffle
// tree inside each warp, then warp 0 combines the warp results in order.
template <typename T>
__device__ inline T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename T>
__device__ inline T warp_max(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// All kBlock threads must call; result valid in every thread.
template <typename T>
__device__ inline T block_sum(T v, T* sh /* >= kWarps */) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    T r = 0;
    if (w == 0) {
        r = (lane < kWarps) ? sh[lane] : T(0);
        r = warp_sum(r);
        if (lane == 0) sh[0] = r;
    }
    __syncthreads();
    r = sh[0];
    __syncthreads();
    return r;
}

template <typename T>
__device__ inline T block_max(T v, T* sh) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    v = warp_max(v);
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    T r = 0;
    if (w == 0) {
        r = (lane < kWarps) ? sh[lane] : T(0);
        r = warp_max(r);
        if (lane == 0) sh[0] = r;
    }
    __syncthreads();
    r = sh[0];
    __syncthreads();
    return r;
}

// Sum of part[0..n) by one block in a fixed order (thread t takes
// t, t+kBlock, ...; then the block tree).  Every thread gets the result.
__device__ inline double block_sum_array(const double* __restrict__ part, int n, double* sh) {
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += kBlock) s += part[i];
    return block_sum(s, sh);
}

__device__ inline double block_max_array(const double* __restrict__ part, int n, double* sh) {
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += kBlock) s = fmax(s, part[i]);
    return block_max(s, sh);
}

}  // namespace nir
