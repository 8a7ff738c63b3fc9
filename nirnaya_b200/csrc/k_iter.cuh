// The PDHG iteration kernels: one launch per half-iteration, A' y fused with
// the primal step and A x-bar fused with the dual step (epilogues in
// k_adaptive.cuh), plus the FP64 KKT passes of a check.
//
// Two layouts of a matrix orientation carry the SpMV, and the autotuner
// picks one per orientation (template parameter LAY):
//   kLayWarp  warp row blocks (k_adaptive.cuh): a warp per block of <= 32
//             rows and <= cap nonzeros, register double buffering, no block
//             barrier; best on short rows;
//   kLayCta   CTA blocks of 256 x 4 nonzeros with a segmented reduction
//             (k_cta.cuh): 128-bit loads of a padded stream, a long row
//             taken by a whole CTA at once; best on medium rows.
// Measured on B200 (CUDA events, cold L2, FP64): on the 200,000 x 500,000
// power-law LP the warp layout takes 32.8 us for A' y (its row-less gather
// ceiling: 30.8 us) against 45 us for the CTA layout, and both ~48 us for
// A x (ceiling 34.8 us); on a 20,000 x 50,000 multiperiod LP the CTA layout
// takes 11.4 us against 14.4 us.
//
// Precisions: TV is the type of the matrix values, TX the type of the
// iterates and of the accumulation.  The engine runs (double, double) for
// FP64; (float, double) -- FP32 values with FP64 iterates, 8 instead of 12
// bytes per nonzero -- for the first phase of the mixed precision; and
// (float, float) for FP32 throughout.
#pragma once

#include "k_adaptive.cuh"
#include "k_cta.cuh"

namespace nir {

constexpr int kLayWarp = 0;
constexpr int kLayCta = 4;  // CTA blocks with a run of 4 nonzeros per thread

// Resident CTAs per SM an iteration kernel is compiled for: by the
// accumulator width in the warp layout, by the run length in the CTA
// layout.  BATCH: the batched kernels, whose FP32-value / FP64-iterate warp
// kernels get one CTA more (80 instead of 110-128 registers).  Their
// instances are medium LPs with short rows, where the extra resident warps
// pay: the 256-instance multiperiod batch solved in 2.99 s against 3.85 s.
// The single-LP kernels keep 2: on the power-law LP the long rows' overlapped
// rounds need the registers, and A x was 12 % slower with 3.
template <int LAY, typename TV, typename TX, bool BATCH = false>
constexpr int lay_min_blocks() {
    if constexpr (LAY == kLayWarp) {
        if constexpr (BATCH && sizeof(TV) == 4 && sizeof(TX) == 8) return iter_min_blocks<TX>() + 1;
        return iter_min_blocks<TX>();
    } else {
        return cta_min_blocks<TX, LAY>();
    }
}

// One orientation's layout as the kernels see it.
struct Lay {
    const void* blk;  // int2 (warp) or int4 (CTA) descriptors, nblk + 1
    int nblk;
    int cap;          // warp row-block capacity (kLayWarp)
    const int* rp;    // CSR row pointers
    const int* ci;    // column indices: the CSR's (kLayWarp) or the padded stream's (kLayCta)
};

// The SpMV of one orientation over its layout with epilogue epi.  The warp
// layout uses the kernel's dynamic shared memory (warp_smem_bytes<TA>).
template <int LAY, typename TA, typename TV, typename TX, class Epi, bool COH>
__device__ __forceinline__ void lay_spmv(const Lay& L, const TV* __restrict__ val, const TX* __restrict__ x,
                                         Epi& epi) {
    if constexpr (LAY == kLayWarp) {
        rowblock_spmv<TA, TV, TX, Epi, COH>(static_cast<const int2*>(L.blk), L.nblk, L.cap, L.rp, L.ci, val, x, epi,
                                            nullptr);
    } else {
        __shared__ CtaShared<TA> sm[2];
        cta_spmv<TA, TV, TX, LAY, Epi, COH>(static_cast<const int4*>(L.blk), L.nblk, L.rp, L.ci, val, x, epi, sm);
    }
}

// Layout of one orientation plus the per-launch scalars.
struct IterArgs {
    Lay lay;
    double* part;     // CHECK launches: per-CTA partial sums
    const DevState* st;
    int i_in_chunk;
    int halpern;
    int phase;        // the kernel runs only while st->phase == phase
    double rho;
};

template <int LAY, typename TV, typename TX, bool CHECK, bool COH>
__device__ __forceinline__ void primal_phase(const IterArgs& a, const TV* __restrict__ val, const TX* __restrict__ y,
                                             TX* __restrict__ x, TX* __restrict__ xbar, TX* __restrict__ xplus,
                                             const TX* __restrict__ c, const TX* __restrict__ lo,
                                             const TX* __restrict__ up, const TX* __restrict__ x0, double* s_red) {
    PrimalEpi<TX, CHECK> epi;
    epi.x = x;
    epi.xbar = xbar;
    epi.xplus = xplus;
    epi.c = c;
    epi.lo = lo;
    epi.up = up;
    epi.x0 = x0;
    epi.s = step_scalars<TX>(a.st, a.i_in_chunk, a.halpern, a.rho);
    epi.halpern = a.halpern;
    lay_spmv<LAY, TX, TV, TX, PrimalEpi<TX, CHECK>, COH>(a.lay, val, y, epi);
    if (CHECK) write_partials(epi, a.part, s_red);
}

template <int LAY, typename TV, typename TX, bool CHECK, bool COH>
__device__ __forceinline__ void dual_phase(const IterArgs& a, const TV* __restrict__ val, const TX* __restrict__ xbar,
                                           TX* __restrict__ y, TX* __restrict__ yplus, const TX* __restrict__ rl,
                                           const TX* __restrict__ ru, const TX* __restrict__ y0, double* s_red) {
    DualEpi<TX, CHECK> epi;
    epi.y = y;
    epi.yplus = yplus;
    epi.rl = rl;
    epi.ru = ru;
    epi.y0 = y0;
    epi.s = step_scalars<TX>(a.st, a.i_in_chunk, a.halpern, a.rho);
    epi.halpern = a.halpern;
    lay_spmv<LAY, TX, TV, TX, DualEpi<TX, CHECK>, COH>(a.lay, val, xbar, epi);
    if (CHECK) write_partials(epi, a.part, s_red);
}

template <int LAY, typename TV, typename TX, bool CHECK>
__global__ void __launch_bounds__(kBlock, (lay_min_blocks<LAY, TV, TX>()))
    k_primal(IterArgs a, const TV* __restrict__ val, const TX* __restrict__ y, TX* __restrict__ x,
             TX* __restrict__ xbar, TX* __restrict__ xplus, const TX* __restrict__ c, const TX* __restrict__ lo,
             const TX* __restrict__ up, const TX* __restrict__ x0) {
    __shared__ double s_red[kWarps];
    if (a.st->done || a.st->phase != a.phase) return;
    primal_phase<LAY, TV, TX, CHECK, false>(a, val, y, x, xbar, xplus, c, lo, up, x0, s_red);
}

template <int LAY, typename TV, typename TX, bool CHECK>
__global__ void __launch_bounds__(kBlock, (lay_min_blocks<LAY, TV, TX>()))
    k_dual(IterArgs a, const TV* __restrict__ val, const TX* __restrict__ xbar, TX* __restrict__ y,
           TX* __restrict__ yplus, const TX* __restrict__ rl, const TX* __restrict__ ru, const TX* __restrict__ y0) {
    __shared__ double s_red[kWarps];
    if (a.st->done || a.st->phase != a.phase) return;
    dual_phase<LAY, TV, TX, CHECK, false>(a, val, xbar, y, yplus, rl, ru, y0, s_red);
}

// ---------------------------------------------------------------- KKT (FP64)

struct KktArgs {
    Lay lay;
    const double* val;   // scaled FP64 values in the layout's stream
    double* part;
    const DevState* st;
    int phase;
};

template <int LAY, typename TX>
__global__ void __launch_bounds__(kBlock)
    k_kkt_rows(KktArgs a, const TX* __restrict__ xplus, const TX* __restrict__ yplus, const double* __restrict__ dr,
               const double* __restrict__ rl, const double* __restrict__ ru) {
    __shared__ double s_red[kWarps];
    if (a.st->done || a.st->phase != a.phase) return;
    KktRowEpi<TX> epi;
    epi.dr = dr;
    epi.rl = rl;
    epi.ru = ru;
    epi.yplus = yplus;
    lay_spmv<LAY, double, double, TX, KktRowEpi<TX>, false>(a.lay, a.val, xplus, epi);
    write_partials(epi, a.part, s_red);
}

template <int LAY, typename TX>
__global__ void __launch_bounds__(kBlock)
    k_kkt_cols(KktArgs a, const TX* __restrict__ xplus, const TX* __restrict__ yplus, const double* __restrict__ dc,
               const double* __restrict__ c, const double* __restrict__ l, const double* __restrict__ u) {
    __shared__ double s_red[kWarps];
    if (a.st->done || a.st->phase != a.phase) return;
    KktColEpi<TX> epi;
    epi.dc = dc;
    epi.c = c;
    epi.l = l;
    epi.u = u;
    epi.xplus = xplus;
    lay_spmv<LAY, double, double, TX, KktColEpi<TX>, false>(a.lay, a.val, yplus, epi);
    write_partials(epi, a.part, s_red);
}

}  // namespace nir
