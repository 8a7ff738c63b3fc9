// The double-double solution check on the device.
//
// verify_solution (src/io/sol_io.hpp:25-106, with Model::eval_objective,
// src/model/model.hpp:73-98) for the instances resident in a PDHG handle or
// batch, reporting exactly what nir_verify_solution (include/nir_sol.h)
// reports on the host for the same LP and point, bit for bit:
//   - every column's bound (and integrality) violation, scaled by
//     1 + |bound|, with the first maximum kept;
//   - every row's activity as a double-double sum of a_ij * x_j over the
//     row's entries in ascending column order, skipping x_j == 0 (the order
//     of the reference's column loop), then its scaled bound violation;
//   - the objective as the double-double sum of c_j * x_j in column order
//     from the objective offset;
//   - the report's verdict and worst item by the reference's rules.
// A double-double sum depends on the order of its terms, so each row (and
// each instance's objective) is summed by one thread in that order; only the
// maxima, which do not depend on order, are reduced in parallel.
//
// The per-element steps are __host__ __device__ functions: a host program
// compiled from this header runs the same arithmetic.  On the device every
// operation is an explicitly rounded intrinsic, so nothing is contracted
// into a fused multiply-add that the host check does not perform.
#pragma once

#include <stdint.h>

#include "nir_sol.h"

#if defined(__CUDACC__)
#define NIR_VHD __host__ __device__ __forceinline__
#else
#include <cmath>
#define NIR_VHD inline
#endif

namespace nir {
namespace vfy {

NIR_VHD double add(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
NIR_VHD double sub(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}
NIR_VHD double mul(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
NIR_VHD double fmad(double a, double b, double c) {
#ifdef __CUDA_ARCH__
    return __fma_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}
NIR_VHD double div(double a, double b) {
#ifdef __CUDA_ARCH__
    return __ddiv_rn(a, b);
#else
    return a / b;
#endif
}
NIR_VHD double absv(double a) {
#ifdef __CUDA_ARCH__
    return fabs(a);
#else
    return std::fabs(a);
#endif
}
NIR_VHD bool finite(double a) {
#ifdef __CUDA_ARCH__
    return isfinite(a);
#else
    return std::isfinite(a);
#endif
}
NIR_VHD double round_half_away(double a) {
#ifdef __CUDA_ARCH__
    return round(a);
#else
    return std::round(a);
#endif
}

// is_finite_bound (src/core/types.hpp:49-51): |b| < 1e20 and finite.
NIR_VHD bool fin_bound(double b) { return finite(b) && absv(b) < 1e20; }

// std::max(0.0, d), which is (0.0 < d) ? d : 0.0 (a NaN gives 0.0).
NIR_VHD double pos_part(double d) { return (0.0 < d) ? d : 0.0; }

// ---- double-double accumulation, the reference's dd_real steps
// (src/core/dd_real.hpp): two_sum, quick_two_sum, dd + dd, and an exact
// product a*b = p + e added as a double-double.
struct DD {
    double hi, lo;
};

NIR_VHD void two_sum(double a, double b, double& s, double& e) {
    s = add(a, b);
    const double bb = sub(s, a);
    e = add(sub(a, sub(s, bb)), sub(b, bb));
}

NIR_VHD void quick_two_sum(double a, double b, double& s, double& e) {
    s = add(a, b);
    e = sub(b, sub(s, a));
}

NIR_VHD void add_dd(DD& d, double bhi, double blo) {
    double s1, s2, t1, t2;
    two_sum(d.hi, bhi, s1, s2);
    two_sum(d.lo, blo, t1, t2);
    s2 = add(s2, t1);
    quick_two_sum(s1, s2, s1, s2);
    s2 = add(s2, t2);
    quick_two_sum(s1, s2, d.hi, d.lo);
}

NIR_VHD void add_prod(DD& d, double a, double b) {
    const double p = mul(a, b);
    const double e = fmad(a, b, -p);
    add_dd(d, p, e);
}

// ---- records: a violation and the position of the check that first
// reached it (columns: 3j lower bound, 3j+1 upper bound, 3j+2 integrality;
// rows: 2i lower, 2i+1 upper).  A record holds only values above zero.
struct Rec {
    double v;
    long long pos;
};

NIR_VHD Rec rec0() { return Rec{0.0, -1}; }

// One check, in position order: a new maximum replaces the record.
NIR_VHD void see(Rec& r, double x, long long p) {
    if (x > r.v) {
        r.v = x;
        r.pos = p;
    }
}

// The first maximum of the union of two records' checks: the larger value,
// the earlier position on a tie.  Associative and commutative, so any
// reduction tree gives the record a loop in position order gives.  The
// values are never NaN (pos_part removes them), so the order is total.
NIR_VHD Rec best(const Rec& a, const Rec& b) {
    if (b.v > a.v || (b.v == a.v && b.pos < a.pos)) return b;
    return a;
}

// Column j of an instance (sanitised bounds: +-inf where not finite).
NIR_VHD void col_check(double xv, double lo, double up, int8_t vt, long long j, Rec& B, Rec& G) {
    if (fin_bound(lo)) see(B, div(pos_part(sub(lo, xv)), add(1.0, absv(lo))), 3 * j);
    if (fin_bound(up)) see(B, div(pos_part(sub(xv, up)), add(1.0, absv(up))), 3 * j + 1);
    if (vt == 1 || vt == 2) see(G, absv(sub(xv, round_half_away(xv))), 3 * j + 2);
}

// Row r (i its index in its instance): the double-double activity over the
// row's entries [q0, q1) of a row-major copy of A that keeps each row's
// entries in ascending column order, then the row's record.
NIR_VHD Rec row_check(long long i, long long q0, long long q1, const int* ci, const double* val, const double* x,
                      double lo, double up) {
    DD act{0.0, 0.0};
    for (long long q = q0; q < q1; ++q) {
        const double xv = x[ci[q]];
        if (xv != 0.0) add_prod(act, val[q], xv);
    }
    const double a = add(act.hi, act.lo);
    Rec R = rec0();
    if (fin_bound(lo)) see(R, div(pos_part(sub(lo, a)), add(1.0, absv(lo))), 2 * i);
    if (fin_bound(up)) see(R, div(pos_part(sub(a, up)), add(1.0, absv(up))), 2 * i + 1);
    return R;
}

// Model::eval_objective for an LP: offset + sum of c_j x_j over [c0, c1).
NIR_VHD double objective(double offset, long long c0, long long c1, const double* c, const double* x) {
    DD s{offset, 0.0};
    for (long long j = c0; j < c1; ++j)
        if (c[j] != 0.0 && x[j] != 0.0) add_prod(s, c[j], x[j]);
    return add(s.hi, s.lo);
}

// The report of one instance of n columns, from its first non-finite
// column fb (n when none), its column records, its row record and its
// objective.  The worst item is the one the reference's loops name last:
// the later of the column categories' records above tol, then the rows'.
NIR_VHD nir_verify_report assemble(long long fb, long long n, const Rec& B, const Rec& G, const Rec& R, double obj,
                                   double claimed, double tol) {
    nir_verify_report rep;
    rep.passed = 1;
    rep.worst_kind = 0;
    rep.worst_index = -1;
    rep.max_bound_viol = B.v;
    rep.max_row_viol = 0.0;
    rep.max_int_viol = G.v;
    rep.computed_obj = 0.0;
    rep.obj_rel_err = 0.0;
    const Rec* w = nullptr;
    if (B.v > tol) w = &B;
    if (G.v > tol && (!w || G.pos > w->pos)) w = &G;
    if (w) {
        rep.worst_kind = int32_t(3 + w->pos % 3);
        rep.worst_index = w->pos / 3;
    }
    if (fb < n) {
        rep.passed = 0;
        rep.worst_kind = 2;
        rep.worst_index = fb;
        return rep;
    }
    rep.max_row_viol = R.v;
    if (R.v > tol) {
        rep.worst_kind = int32_t(6 + (R.pos & 1));
        rep.worst_index = R.pos / 2;
    }
    rep.computed_obj = obj;
    if (finite(claimed)) rep.obj_rel_err = div(absv(sub(obj, claimed)), add(1.0, absv(obj)));
    if (rep.max_bound_viol > tol || rep.max_row_viol > tol || rep.max_int_viol > tol || rep.obj_rel_err > 1e-5)
        rep.passed = 0;
    return rep;
}

// ---- kernels

#if defined(__CUDACC__)

constexpr int kVfyBlock = 256;

__device__ __forceinline__ Rec warp_best(Rec r) {
    for (int o = 16; o > 0; o >>= 1) {
        Rec t;
        t.v = __shfl_down_sync(0xffffffffu, r.v, o);
        t.pos = __shfl_down_sync(0xffffffffu, r.pos, o);
        r = best(r, t);
    }
    return r;
}

// The block's best record, returned to every thread.  Every thread of the
// block calls it; blockDim.x is kVfyBlock.
__device__ Rec block_best(Rec r) {
    __shared__ Rec part[kVfyBlock / 32];
    __shared__ Rec out;
    r = warp_best(r);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) part[w] = r;
    __syncthreads();
    if (w == 0) {
        r = lane < kVfyBlock / 32 ? part[lane] : rec0();
        r = warp_best(r);
        if (lane == 0) out = r;
    }
    __syncthreads();
    r = out;
    __syncthreads();  // part and out may be reused by the next call
    return r;
}

// The smallest value over the block, returned to every thread.
__device__ long long block_min(long long v) {
    __shared__ long long part[kVfyBlock / 32];
    __shared__ long long out;
    for (int o = 16; o > 0; o >>= 1) v = min(v, (long long)__shfl_down_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) part[w] = v;
    __syncthreads();
    if (w == 0) {
        long long u = lane < kVfyBlock / 32 ? part[lane] : v;
        for (int o = 16; o > 0; o >>= 1) u = min(u, (long long)__shfl_down_sync(0xffffffffu, u, o));
        if (lane == 0) out = u;
    }
    __syncthreads();
    v = out;
    __syncthreads();
    return v;
}

// One block per instance k: the first column with a non-finite value, then
// the bound and integrality records over the columns before it.  vt may be
// null (no integer columns).
__global__ void __launch_bounds__(kVfyBlock) k_vfy_cols(const int* __restrict__ col_off, const double* __restrict__ x,
                                                        const double* __restrict__ lo, const double* __restrict__ up,
                                                        const int8_t* __restrict__ vt, long long* __restrict__ fb_out,
                                                        Rec* __restrict__ b_out, Rec* __restrict__ g_out) {
    const int k = blockIdx.x;
    const long long c0 = col_off[k], n = col_off[k + 1] - c0;
    long long fb = n;
    for (long long j = threadIdx.x; j < n; j += kVfyBlock)
        if (!finite(x[c0 + j])) {
            fb = j;  // the first of this thread's columns; the block takes the least
            break;
        }
    fb = block_min(fb);
    Rec B = rec0(), G = rec0();
    for (long long j = threadIdx.x; j < fb; j += kVfyBlock)
        col_check(x[c0 + j], lo[c0 + j], up[c0 + j], vt ? vt[c0 + j] : int8_t(0), j, B, G);
    B = block_best(B);
    G = block_best(G);
    if (threadIdx.x == 0) {
        fb_out[k] = fb;
        b_out[k] = B;
        g_out[k] = G;
    }
}

// Threads [0, count): the objective of instance t, one thread each (a
// sequential double-double sum).  Threads [count, count + m): row
// t - count, its record's value and side (0 lower, 1 upper).  Rows of an
// instance with a non-finite column are skipped (the host check stops
// before the rows there).  row_inst null: one instance.  row_orig (null:
// the identity) is the caller's index of each row, where its record goes:
// a handle holds its rows in its own order, and the report's reduction
// runs in the caller's.
__global__ void __launch_bounds__(kVfyBlock) k_vfy_rows(
    int count, long long m, const int* __restrict__ row_off, const int* __restrict__ col_off,
    const int* __restrict__ row_inst, const int* __restrict__ rp, const int* __restrict__ ci,
    const double* __restrict__ val, const double* __restrict__ x, const double* __restrict__ rl,
    const double* __restrict__ ru, const double* __restrict__ c, const double* __restrict__ offset,
    const long long* __restrict__ fb, const int* __restrict__ row_orig, double* __restrict__ rv,
    int8_t* __restrict__ rs, double* __restrict__ obj) {
    const long long t = blockIdx.x * (long long)kVfyBlock + threadIdx.x;
    if (t < count) {
        const int k = int(t);
        const long long c0 = col_off[k], c1 = col_off[k + 1];
        obj[k] = fb[k] < c1 - c0 ? 0.0 : objective(offset[k], c0, c1, c, x);
        return;
    }
    const long long r = t - count;
    if (r >= m) return;
    const int k = row_inst ? row_inst[r] : 0;
    const long long ro = row_orig ? (long long)row_orig[r] : r;
    if (fb[k] < (long long)(col_off[k + 1] - col_off[k])) {
        rv[ro] = 0.0;
        rs[ro] = 0;
        return;
    }
    const Rec R = row_check(ro - row_off[k], rp[r], rp[r + 1], ci, val, x, rl[r], ru[r]);
    rv[ro] = R.v;
    rs[ro] = R.pos >= 0 ? int8_t(R.pos & 1) : int8_t(0);
}

// One block per instance: the row record over the instance's rows, then
// the report.
__global__ void __launch_bounds__(kVfyBlock) k_vfy_report(
    const int* __restrict__ row_off, const int* __restrict__ col_off, const double* __restrict__ rv,
    const int8_t* __restrict__ rs, const long long* __restrict__ fb, const Rec* __restrict__ b, const Rec* __restrict__ g,
    const double* __restrict__ obj, const double* __restrict__ claimed, double tol, nir_verify_report* __restrict__ out) {
    const int k = blockIdx.x;
    const long long r0 = row_off[k], mk = row_off[k + 1] - r0;
    Rec R = rec0();
    for (long long i = threadIdx.x; i < mk; i += kVfyBlock) see(R, rv[r0 + i], 2 * i + rs[r0 + i]);
    R = block_best(R);
    if (threadIdx.x == 0)
        out[k] = assemble(fb[k], col_off[k + 1] - col_off[k], b[k], g[k], R, obj[k], claimed[k], tol);
}

#endif  // __CUDACC__

}  // namespace vfy
}  // namespace nir
