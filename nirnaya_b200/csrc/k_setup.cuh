// Setup kernels: CSC -> CSR transpose on the device, diagonal
// preconditioning (Ruiz l-inf passes + one Pock-Chambolle alpha=1 pass,
// factors rounded to powers of two so scaling is exact), the power
// iteration for ||A||_2 and the scaled problem vectors.
#pragma once

#include "dev_common.cuh"

namespace nir {

// col_of[k] = column of CSC entry k (one thread per column).
__global__ void k_expand_cols(int n, const long long* __restrict__ start, int* __restrict__ col_of) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    for (long long k = start[j]; k < start[j + 1]; ++k) col_of[k] = j;
}

__global__ void k_iota(long long n, int* __restrict__ v) {
    long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (k < n) v[k] = int(k);
}

// row_ptr[i] = first position of key >= i in the sorted row keys.
__global__ void k_row_ptr_from_sorted(int m, long long nnz, const int* __restrict__ keys, int* __restrict__ rp) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > m) return;
    long long lo = 0, hi = nnz;
    while (lo < hi) {
        long long mid = (lo + hi) >> 1;
        if (keys[mid] < i) lo = mid + 1;
        else hi = mid;
    }
    rp[i] = int(lo);
}

__global__ void k_gather_csr(long long nnz, const int* __restrict__ perm, const int* __restrict__ col_of,
                             const double* __restrict__ v_in, int* __restrict__ ci, double* __restrict__ v_out) {
    long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (p >= nnz) return;
    int k = perm[p];
    ci[p] = col_of[k];
    v_out[p] = v_in[k];
}

__global__ void k_offsets_to_int(int n1, const long long* __restrict__ in, int* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n1) out[i] = int(in[i]);
}

// Sanitise bounds: anything the reference does not treat as a finite bound
// (src/core/types.hpp:49-51) becomes -inf (lower) or +inf (upper).
__global__ void k_sanitize_bounds(int n, const double* __restrict__ lo_in, const double* __restrict__ up_in,
                                  double* __restrict__ lo, double* __restrict__ up) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    double l = lo_in[j], u = up_in[j];
    lo[j] = fin_bound(l) ? l : -INFINITY;
    up[j] = fin_bound(u) ? u : INFINITY;
}

// ---------------------------------------------------------------- scaling

// One warp per row: out[r] = max (mode 0) or sum (mode 1) over the row of
// |v| * d_row[r] * d_col[ci].  Deterministic shuffle tree.
__global__ void k_row_stat(int rows, const int* __restrict__ rp, const int* __restrict__ ci,
                           const double* __restrict__ v, const double* __restrict__ d_row,
                           const double* __restrict__ d_col, int mode, double* __restrict__ out) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= rows) return;
    const double dr = d_row[warp];
    double acc = 0.0;
    for (int k = rp[warp] + lane; k < rp[warp + 1]; k += 32) {
        double a = fabs(v[k]) * dr * d_col[ci[k]];
        acc = mode == 0 ? fmax(acc, a) : acc + a;
    }
    acc = mode == 0 ? warp_max(acc) : warp_sum(acc);
    if (lane == 0) out[warp] = acc;
}

// d[i] /= sqrt(stat[i]) where stat > 0.
__global__ void k_apply_stat(int n, const double* __restrict__ stat, double* __restrict__ d) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = stat[i];
    if (s > 0.0 && isfinite(s)) d[i] /= sqrt(s);
}

// Nearest power of two (in the log sense), exponent clamped to +-60.
__global__ void k_round_pow2(int n, double* __restrict__ d) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v = d[i];
    if (!(v > 0.0) || !isfinite(v)) {
        d[i] = 1.0;
        return;
    }
    int e;
    double f = frexp(v, &e);  // v = f * 2^e, f in [0.5, 1)
    int k = (f >= 0.70710678118654752440) ? e : e - 1;
    k = k > 60 ? 60 : (k < -60 ? -60 : k);
    d[i] = ldexp(1.0, k);
}

// Scaled values of one orientation: v = (orig * dr_i) * dc_j with i the row
// of A and j the column of A, identical bits in both orientations.
__global__ void k_scale_values(int rows, const int* __restrict__ rp, const int* __restrict__ ci,
                               const double* __restrict__ orig, const double* __restrict__ d_this,
                               const double* __restrict__ d_other, int this_is_row_of_A, double* __restrict__ v64,
                               float* __restrict__ v32) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= rows) return;
    const double dt = d_this[warp];
    for (int k = rp[warp] + lane; k < rp[warp + 1]; k += 32) {
        const double dother = d_other[ci[k]];
        const double s = this_is_row_of_A ? (orig[k] * dt) * dother : (orig[k] * dother) * dt;
        v64[k] = s;
        v32[k] = float(s);
    }
}

// Scaled vectors: c^ = c*dc, l^ = l/dc, u^ = u/dc (columns);
// rl^ = rl*dr, ru^ = ru*dr (rows).  Infinite bounds stay infinite.
__global__ void k_scale_vectors(int n, int m, const double* __restrict__ c, const double* __restrict__ l,
                                const double* __restrict__ u, const double* __restrict__ rl,
                                const double* __restrict__ ru, const double* __restrict__ dc,
                                const double* __restrict__ dr, double* __restrict__ c64, double* __restrict__ l64,
                                double* __restrict__ u64, double* __restrict__ rl64, double* __restrict__ ru64,
                                float* __restrict__ c32, float* __restrict__ l32, float* __restrict__ u32,
                                float* __restrict__ rl32, float* __restrict__ ru32) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) {
        double d = dc[t];
        double cc = c[t] * d, ll = l[t] / d, uu = u[t] / d;
        c64[t] = cc;
        l64[t] = ll;
        u64[t] = uu;
        c32[t] = float(cc);
        l32[t] = float(ll);
        u32[t] = float(uu);
    }
    if (t < m) {
        double d = dr[t];
        double a = rl[t] * d, b = ru[t] * d;
        rl64[t] = a;
        ru64[t] = b;
        rl32[t] = float(a);
        ru32[t] = float(b);
    }
}

// ---------------------------------------------------------------- power iteration

// Deterministic pseudo-random start in [0.5, 1.5) (splitmix64 of the index).
__device__ __forceinline__ double power_start_value(unsigned long long j) {
    unsigned long long z = j * 0x9e3779b97f4a7c15ULL + 0x632be59bd9b4e019ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    z ^= z >> 31;
    return 0.5 + double(z >> 11) * 0x1.0p-53;
}

__global__ void k_power_start(int n, double* __restrict__ u) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    u[j] = power_start_value(j);
}

// Batch start: each instance's columns from its own index 0, so an
// instance's estimate does not depend on the batch around it.
__global__ void k_power_start_batch(int n, const int* __restrict__ col_inst, const int* __restrict__ col_off,
                                    double* __restrict__ u) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    u[j] = power_start_value(j - col_off[col_inst[j]]);
}

// One warp per row FP64 SpMV (setup only).
__global__ void k_spmv_warp64(int rows, const int* __restrict__ rp, const int* __restrict__ ci,
                              const double* __restrict__ v, const double* __restrict__ x, double* __restrict__ y) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= rows) return;
    double acc = 0.0;
    for (int k = rp[warp] + lane; k < rp[warp + 1]; k += 32) acc += v[k] * x[ci[k]];
    acc = warp_sum(acc);
    if (lane == 0) y[warp] = acc;
}

// Per-block partial sums of squares.
__global__ void k_sumsq_partials(int n, const double* __restrict__ w, double* __restrict__ part) {
    __shared__ double sh[kWarps];
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    double v = (j < n) ? w[j] * w[j] : 0.0;
    v = block_sum(v, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = v;
}

// norm = sqrt(sum part); stores it in st->ref_norm_est; the estimate of
// ||A||_2 after the round is sqrt(norm) for a unit start vector.
__global__ void k_norm_finalize(const double* __restrict__ part, int nblk, DevState* st) {
    __shared__ double sh[kWarps];
    double s = block_sum_array(part, nblk, sh);
    if (threadIdx.x == 0) st->ref_norm_est = sqrt(s);
}

__global__ void k_scale_by_inv_norm(int n, double* __restrict__ w, const DevState* __restrict__ st) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    double nrm = st->ref_norm_est;
    w[j] = nrm > 0.0 ? w[j] / nrm : 0.0;
}

// ---------------------------------------------------------------- iterate setup

// x^ = clamp(x_init / dc (or 0), l^, u^); y^ = y_init / dr (or 0); both
// also copied into the anchors and converted to FP32.
__global__ void k_init_iterates(int n, int m, const double* __restrict__ x_in, const double* __restrict__ y_in,
                                const double* __restrict__ dc, const double* __restrict__ dr,
                                const double* __restrict__ l64, const double* __restrict__ u64,
                                double* __restrict__ x64, double* __restrict__ x064, double* __restrict__ y64,
                                double* __restrict__ y064, float* __restrict__ x32, float* __restrict__ x032,
                                float* __restrict__ y32, float* __restrict__ y032, const float* __restrict__ l32,
                                const float* __restrict__ u32) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) {
        double v = x_in ? x_in[t] / dc[t] : 0.0;
        double v64 = clamp_box(v, l64[t], u64[t]);
        x64[t] = v64;
        x064[t] = v64;
        float v32 = clamp_box(float(v), l32[t], u32[t]);
        x32[t] = v32;
        x032[t] = v32;
    }
    if (t < m) {
        double v = y_in ? y_in[t] / dr[t] : 0.0;
        y64[t] = v;
        y064[t] = v;
        y32[t] = float(v);
        y032[t] = float(v);
    }
}

// FP32 -> FP64 hand-over for the polish phase: iterate and anchor become
// the last evaluated point (x+, y+), clamped to the FP64 box.
__global__ void k_promote(int n, int m, const float* __restrict__ xp32, const float* __restrict__ yp32,
                          const double* __restrict__ l64, const double* __restrict__ u64, double* __restrict__ x64,
                          double* __restrict__ x064, double* __restrict__ xp64, double* __restrict__ y64,
                          double* __restrict__ y064, double* __restrict__ yp64) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) {
        double v = clamp_box(double(xp32[t]), l64[t], u64[t]);
        x64[t] = v;
        x064[t] = v;
        xp64[t] = v;
    }
    if (t < m) {
        double v = double(yp32[t]);
        y64[t] = v;
        y064[t] = v;
        yp64[t] = v;
    }
}

// Fresh start of the FP64 polish at the last evaluated point: iterate and
// anchor become (x+, y+).
__global__ void k_restart_at(int n, int m, const double* __restrict__ xp, const double* __restrict__ yp,
                             double* __restrict__ x, double* __restrict__ x0, double* __restrict__ y,
                             double* __restrict__ y0) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) {
        x[t] = xp[t];
        x0[t] = xp[t];
    }
    if (t < m) {
        y[t] = yp[t];
        y0[t] = yp[t];
    }
}

// Original-space output: x = dc * x^, y = dr * y^.
template <typename T>
__global__ void k_unscale_out(int n, int m, const T* __restrict__ xp, const T* __restrict__ yp,
                              const double* __restrict__ dc, const double* __restrict__ dr, double* __restrict__ xo,
                              double* __restrict__ yo) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) xo[t] = double(xp[t]) * dc[t];
    if (t < m) yo[t] = double(yp[t]) * dr[t];
}

__global__ void k_to_float(long long n, const double* __restrict__ a, float* __restrict__ b) {
    long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (k < n) b[k] = float(a[k]);
}

__global__ void k_to_double(long long n, const float* __restrict__ a, double* __restrict__ b) {
    long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (k < n) b[k] = double(a[k]);
}

__global__ void k_fill(long long n, double v, double* __restrict__ a) {
    long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (k < n) a[k] = v;
}

// Compact status record written to host-mapped memory at the end of
// every launch chunk, read by the host after the chunk's event.
struct HostSnap {
    long long seq;
    long long iter;
    int done, status, phase, restarts;
    double kkt, kp, kd, kg, pobj, dobj, max_rel_row, omega, res;
    long long ref_iterations;
    int ref_stopped, pad;
};

constexpr int kSnapRing = 64;

__global__ void k_snap(const DevState* __restrict__ st, HostSnap* __restrict__ ring, long long* __restrict__ seq) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    long long s = *seq + 1;
    *seq = s;
    HostSnap h;
    h.seq = s;
    h.iter = st->iter;
    h.done = st->done;
    h.status = st->status;
    h.phase = st->phase;
    h.restarts = st->restarts;
    h.kkt = st->kkt;
    h.kp = st->kp;
    h.kd = st->kd;
    h.kg = st->kg;
    h.pobj = st->pobj;
    h.dobj = st->dobj;
    h.max_rel_row = st->max_rel_row;
    h.omega = st->omega;
    h.res = st->res;
    h.ref_iterations = st->ref_iterations;
    h.ref_stopped = st->ref_stopped;
    h.pad = 0;
    ring[s % kSnapRing] = h;
    __threadfence_system();
}

}  // namespace nir
