// CTA-level CSR SpMV with a segmented reduction, the core of the
// iteration kernels (CSR of A for A x, the stored CSR of A' for A' y).
//
// A matrix orientation is cut into CTA blocks (row_blocks.hpp,
// build_cta_blocks): consecutive rows holding at most cap = 256 * E
// nonzeros and at most 256 rows, or one longer row.  The block's nonzeros
// lie in a padded copy of the stream starting at a multiple of 4 entries,
// so thread t reads its run of E consecutive entries [E t, E t + E) with
// aligned 128-bit loads (int4 indices, double2 / float4 values), gathers
// the E vector entries at once and forms the products in registers.  Rows
// are then summed without any serial walk over a long row:
//   1. each thread sums the part of its run that belongs to the row still
//      open at its end (tsum) and notes whether a row starts in its run;
//   2. a segmented inclusive scan of (flag, tsum) over the CTA (shuffles in
//      each warp, then the warp totals in order) gives every thread the
//      partial sum of the row open at its run's start;
//   3. each thread closes the rows whose last entry is in its run and puts
//      the sums in shared memory; thread j then runs the epilogue of row j.
// A row longer than cap is streamed by the whole CTA in rounds of cap and
// reduced by the fixed block tree.  The summation order of every row
// depends only on the layout (E and the block boundaries), never on the
// grid or timing, and no atomics are used: results are deterministic.
//
// Reference correspondence: the sums are src/core/csc_matrix.hpp:99-120
// (A x and A' y); the epilogues are those of k_adaptive.cuh.
#pragma once

#include "dev_common.cuh"
#include "row_blocks.hpp"

namespace nir {

// ---------------------------------------------------------------- aligned run loads

// Loads of the matrix stream are streaming (evict-first), so the stream
// does not push the gathered vector out of L1/L2.
__device__ __forceinline__ int4 lds_i4(const int* p) { return __ldcs(reinterpret_cast<const int4*>(p)); }
__device__ __forceinline__ int2 lds_i2(const int* p) { return __ldcs(reinterpret_cast<const int2*>(p)); }
__device__ __forceinline__ double2 lds_d2(const double* p) { return __ldcs(reinterpret_cast<const double2*>(p)); }
__device__ __forceinline__ float4 lds_f4(const float* p) { return __ldcs(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ float2 lds_f2(const float* p) { return __ldcs(reinterpret_cast<const float2*>(p)); }

// E indices at p[pos..pos+E) (pos a multiple of E, p + pos 4E-byte aligned
// for E <= 4, 16-byte aligned for E = 8).  A vector is loaded only when it
// starts below lim; the rest is 0.
template <int E>
__device__ __forceinline__ void ld_idx(const int* __restrict__ p, int pos, int lim, int (&c)[E]) {
    if constexpr (E >= 4) {
#pragma unroll
        for (int k = 0; k < E / 4; ++k) {
            int4 q = make_int4(0, 0, 0, 0);
            if (pos + 4 * k < lim) q = lds_i4(p + pos + 4 * k);
            c[4 * k] = q.x;
            c[4 * k + 1] = q.y;
            c[4 * k + 2] = q.z;
            c[4 * k + 3] = q.w;
        }
    } else if constexpr (E == 2) {
        int2 q = make_int2(0, 0);
        if (pos < lim) q = lds_i2(p + pos);
        c[0] = q.x;
        c[1] = q.y;
    } else {
        c[0] = (pos < lim) ? __ldcs(p + pos) : 0;
    }
}

template <int E>
__device__ __forceinline__ void ld_val(const double* __restrict__ p, int pos, int lim, double (&v)[E]) {
    if constexpr (E >= 2) {
#pragma unroll
        for (int k = 0; k < E / 2; ++k) {
            double2 q = make_double2(0.0, 0.0);
            if (pos + 2 * k < lim) q = lds_d2(p + pos + 2 * k);
            v[2 * k] = q.x;
            v[2 * k + 1] = q.y;
        }
    } else {
        v[0] = (pos < lim) ? __ldcs(p + pos) : 0.0;
    }
}

template <int E>
__device__ __forceinline__ void ld_val(const float* __restrict__ p, int pos, int lim, float (&v)[E]) {
    if constexpr (E >= 4) {
#pragma unroll
        for (int k = 0; k < E / 4; ++k) {
            float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
            if (pos + 4 * k < lim) q = lds_f4(p + pos + 4 * k);
            v[4 * k] = q.x;
            v[4 * k + 1] = q.y;
            v[4 * k + 2] = q.z;
            v[4 * k + 3] = q.w;
        }
    } else if constexpr (E == 2) {
        float2 q = make_float2(0.f, 0.f);
        if (pos < lim) q = lds_f2(p + pos);
        v[0] = q.x;
        v[1] = q.y;
    } else {
        v[0] = (pos < lim) ? __ldcs(p + pos) : 0.f;
    }
}

// Gathers of the multiplied vector: the read-only path, or L2 (coherent)
// for a kernel that rewrites the vector between grid barriers.
template <bool COH, typename T>
__device__ __forceinline__ T cta_gather(const T* p) {
    if (COH) return __ldcg(p);
    return __ldg(p);
}

// ---------------------------------------------------------------- block state

template <typename TA>
struct CtaShared {
    int off[kCtaRowsMax + 1];  // row starts within the block, off[nrows] = block nonzeros
    TA rowsum[kCtaRowsMax];
    TA wc[kWarps];             // warp totals of the segmented scan
    int wf[kWarps];
    TA red[kWarps];            // block reduction of a long row
};

// Resident CTAs per SM the kernels are compiled for, by run length and
// accumulator width (register budget 65536 / (256 * n)).
template <typename TA, int E>
constexpr int cta_min_blocks() {
    return (E >= 8) ? (sizeof(TA) == 8 ? 3 : 4) : (E >= 4 ? 4 : 5);
}

// One CTA block.  d0 = (r0, p0, q0, -), d1 = the next descriptor.
template <typename TA, typename TV, typename TX, int E, class Epi, bool COH>
__device__ __forceinline__ void cta_block(const int4 d0, const int4 d1, const int* __restrict__ rp,
                                          const int* __restrict__ ci, const TV* __restrict__ val,
                                          const TX* __restrict__ x, Epi& epi, CtaShared<TA>& sm) {
    constexpr int CAP = kBlock * E;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int r0 = d0.x, p0 = d0.y, q0 = d0.z;
    const int nrows = d1.x - r0, nnzb = d1.y - p0;
    const int* __restrict__ cb = ci + q0;
    const TV* __restrict__ vb = val + q0;
    typename Epi::Pre pre{};
    if (nnzb > CAP) {
        // one long row, streamed by the whole CTA in rounds of CAP
        if (t == 0) pre = epi.prefetch(r0);
        TA acc = TA(0);
        for (int base = 0; base < nnzb; base += CAP) {
            const int a = base + t * E;
            int c[E];
            TV v[E];
            TX xv[E];
            ld_idx<E>(cb, a, nnzb, c);
            ld_val<E>(vb, a, nnzb, v);
#pragma unroll
            for (int i = 0; i < E; ++i) xv[i] = (a + i < nnzb) ? cta_gather<COH>(x + c[i]) : TX(0);
#pragma unroll
            for (int i = 0; i < E; ++i) acc += TA(v[i]) * TA(xv[i]);
        }
        acc = block_sum(acc, sm.red);
        if (t == 0) epi.row(r0, acc, pre);
        return;
    }
    // packed rows: nrows <= kCtaRowsMax, nnzb <= CAP
    for (int j = t; j <= nrows; j += kBlock) sm.off[j] = (j < nrows) ? __ldg(rp + r0 + j) - p0 : nnzb;
    if (t < nrows) pre = epi.prefetch(r0 + t);
    const int a = t * E;
    const bool active = a < nnzb;
    TA p[E];
    {
        int c[E];
        TV v[E];
        TX xv[E];
        ld_idx<E>(cb, a, nnzb, c);
        ld_val<E>(vb, a, nnzb, v);
#pragma unroll
        for (int i = 0; i < E; ++i) xv[i] = (a + i < nnzb) ? cta_gather<COH>(x + c[i]) : TX(0);
#pragma unroll
        for (int i = 0; i < E; ++i) p[i] = TA(v[i]) * TA(xv[i]);
    }
    __syncthreads();  // off[] is complete
    // the row open at a, the sum of the run's last segment, and whether a
    // row starts in the run
    int row = 0;
    bool head = false;
    TA tsum = TA(0);
    int flag = 0;
    if (active) {
        int lo = 0, hi = nrows - 1;  // largest j with off[j] <= a: a non-empty row containing a
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (sm.off[mid] <= a) lo = mid;
            else hi = mid - 1;
        }
        row = lo;
        head = sm.off[row] < a;
        flag = head ? 0 : 1;
        int r = row, e = sm.off[row + 1];
#pragma unroll
        for (int i = 0; i < E; ++i) {
            const int pos = a + i;
            if (pos < nnzb) {
                while (pos >= e) {
                    ++r;
                    e = sm.off[r + 1];
                    flag = 1;
                    tsum = TA(0);
                }
                tsum += p[i];
            }
        }
    }
    // segmented inclusive scan of (flag, tsum) within the warp
    TA cs = tsum;
    int fs = flag;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const TA cu = __shfl_up_sync(0xffffffffu, cs, d);
        const int fu = __shfl_up_sync(0xffffffffu, fs, d);
        if (lane >= d) {
            if (!fs) cs = cu + cs;
            fs |= fu;
        }
    }
    if (lane == 31) {
        sm.wc[w] = cs;
        sm.wf[w] = fs;
    }
    TA ce = __shfl_up_sync(0xffffffffu, cs, 1);
    int fe = __shfl_up_sync(0xffffffffu, fs, 1);
    if (lane == 0) {
        ce = TA(0);
        fe = 0;
    }
    __syncthreads();  // warp totals are complete
    if (active) {
        TA acc = TA(0);
        if (head) {
            // the part of the row open at a that lies before a: the warps
            // before this one, then the lanes before this one
            TA cw = TA(0);
            for (int k = 0; k < w; ++k) cw = sm.wf[k] ? sm.wc[k] : cw + sm.wc[k];
            acc = fe ? ce : cw + ce;
        }
        int r = row, e = sm.off[row + 1];
#pragma unroll
        for (int i = 0; i < E; ++i) {
            const int pos = a + i;
            if (pos < nnzb) {
                while (pos >= e) {
                    ++r;
                    e = sm.off[r + 1];
                }
                acc += p[i];
                if (pos + 1 == e) {
                    sm.rowsum[r] = acc;
                    acc = TA(0);
                }
            }
        }
    }
    __syncthreads();  // row sums are complete
    if (t < nrows) epi.row(r0 + t, (sm.off[t] == sm.off[t + 1]) ? TA(0) : sm.rowsum[t], pre);
}

// Persistent CTAs: CTA c takes blocks c, c + G, c + 2G, ...  Consecutive
// blocks alternate between two shared-memory sets, so the next block's
// row starts can be written while the last epilogue still reads the
// other set.
template <typename TA, typename TV, typename TX, int E, class Epi, bool COH = false>
__device__ __forceinline__ void cta_spmv(const int4* __restrict__ blk, int nblk, const int* __restrict__ rp,
                                         const int* __restrict__ ci, const TV* __restrict__ val,
                                         const TX* __restrict__ x, Epi& epi, CtaShared<TA>* sm) {
    int k = 0;
    for (int b = blockIdx.x; b < nblk; b += gridDim.x, ++k) {
        const int4 d0 = __ldg(blk + b), d1 = __ldg(blk + b + 1);
        cta_block<TA, TV, TX, E, Epi, COH>(d0, d1, rp, ci, val, x, epi, sm[k & 1]);
    }
}

// ---------------------------------------------------------------- plain SpMV

template <typename TA>
struct CtaPlainEpi {
    static constexpr int NQ = 0;
    static constexpr bool kLastIsMax = false;
    struct Pre {};
    double q[1];
    TA* y;
    __device__ Pre prefetch(int) const { return Pre{}; }
    __device__ void row(int r, TA s, const Pre&) { y[r] = s; }
};

template <typename TA, typename TV, typename TX, int E>
__global__ void __launch_bounds__(kBlock, cta_min_blocks<TA, E>())
    k_spmv_cta(const int4* __restrict__ blk, int nblk, const int* __restrict__ rp, const int* __restrict__ ci,
               const TV* __restrict__ val, const TX* __restrict__ x, TA* __restrict__ y) {
    __shared__ CtaShared<TA> sm[2];
    CtaPlainEpi<TA> epi;
    epi.y = y;
    cta_spmv<TA, TV, TX, E>(blk, nblk, rp, ci, val, x, epi, sm);
}

// ---------------------------------------------------------------- ceilings

// The row-less SpMV: each thread streams groups of 8 consecutive nonzeros
// of the stream with aligned 128-bit loads, gathers x for them (GATHER) or
// only adds the stream (no gathers), and keeps one running sum.  Every
// row-structured SpMV over the same stream and the same gathers does at
// least this work, so its time is the ceiling the iteration kernels are
// measured against.  ngroups = nonzeros / 8 (the tail is left out).
template <typename TA, typename TV, typename TX, bool GATHER>
__global__ void __launch_bounds__(kBlock) k_stream_ceiling(int ngroups, const int* __restrict__ ci,
                                                           const TV* __restrict__ val, const TX* __restrict__ x,
                                                           TA* __restrict__ out) {
    TA acc = TA(0);
    for (int g = blockIdx.x * kBlock + threadIdx.x; g < ngroups; g += gridDim.x * kBlock) {
        int c[8];
        TV v[8];
        ld_idx<8>(ci, 8 * g, 8 * g + 8, c);
        ld_val<8>(val, 8 * g, 8 * g + 8, v);
        if (GATHER) {
            TX xv[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) xv[i] = __ldg(x + c[i]);
#pragma unroll
            for (int i = 0; i < 8; ++i) acc += TA(v[i]) * TA(xv[i]);
        } else {
#pragma unroll
            for (int i = 0; i < 8; ++i) acc += TA(v[i]) + TA(c[i]);
        }
    }
    out[blockIdx.x * kBlock + threadIdx.x] = acc;
}

// Copies each CTA block's nonzeros from the CSR arrays into the padded
// stream (zeros in the padding); ci_p may be null (values only).  One CTA
// per block at a time.
template <typename TV>
__global__ void k_pad_stream(const int4* __restrict__ blk, int nblk, const int* __restrict__ ci,
                             const TV* __restrict__ val, int* __restrict__ ci_p, TV* __restrict__ val_p) {
    for (int b = blockIdx.x; b < nblk; b += gridDim.x) {
        const int4 d0 = blk[b], d1 = blk[b + 1];
        const int p0 = d0.y, q0 = d0.z, n = d1.y - d0.y, q1 = d1.z;
        for (int k = threadIdx.x; k < q1 - q0; k += blockDim.x) {
            const bool in = k < n;
            if (ci_p) ci_p[q0 + k] = in ? ci[p0 + k] : 0;
            val_p[q0 + k] = in ? val[p0 + k] : TV(0);
        }
    }
}

}  // namespace nir
