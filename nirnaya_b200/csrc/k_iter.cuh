// The PDHG iteration kernels on the CTA-block SpMV (k_cta.cuh): one launch
// per half-iteration, A' y fused with the primal step and A x-bar fused with
// the dual step (epilogues in k_adaptive.cuh), plus the FP64 KKT passes of a
// check.
//
// Precisions: TV is the type of the matrix values in the stream, TX the type
// of the iterates and of the accumulation.  The engine runs
//   (double, double)  FP64;
//   (float,  double)  FP32 matrix with FP64 iterates: 8 instead of 12 bytes
//                     per nonzero, the first phase of the mixed precision;
//   (float,  float)   everything in FP32.
// E (1, 2, 4 or 8) is the run length of a thread, so a CTA block holds up to
// 256 E nonzeros; the autotuner picks it per matrix.
#pragma once

#include "k_adaptive.cuh"
#include "k_cta.cuh"

namespace nir {

// Layout of one orientation plus the per-launch scalars.
struct IterArgs {
    const int4* blk;  // CTA-block descriptors (nblk + 1)
    int nblk;
    const int* rp;    // CSR row pointers
    const int* ci;    // padded column indices
    double* part;     // CHECK launches: per-CTA partial sums
    const DevState* st;
    int i_in_chunk;
    int halpern;
    int phase;        // the kernel runs only while st->phase == phase
    double rho;
};

template <typename TV, typename TX, int E, bool CHECK, bool COH>
__device__ __forceinline__ void primal_phase(const IterArgs& a, const TV* __restrict__ val, const TX* __restrict__ y,
                                             TX* __restrict__ x, TX* __restrict__ xbar, TX* __restrict__ xplus,
                                             const TX* __restrict__ c, const TX* __restrict__ lo,
                                             const TX* __restrict__ up, const TX* __restrict__ x0,
                                             CtaShared<TX>* sm, double* s_red) {
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
    cta_spmv<TX, TV, TX, E, PrimalEpi<TX, CHECK>, COH>(a.blk, a.nblk, a.rp, a.ci, val, y, epi, sm);
    if (CHECK) write_partials(epi, a.part, s_red);
}

template <typename TV, typename TX, int E, bool CHECK, bool COH>
__device__ __forceinline__ void dual_phase(const IterArgs& a, const TV* __restrict__ val, const TX* __restrict__ xbar,
                                           TX* __restrict__ y, TX* __restrict__ yplus, const TX* __restrict__ rl,
                                           const TX* __restrict__ ru, const TX* __restrict__ y0, CtaShared<TX>* sm,
                                           double* s_red) {
    DualEpi<TX, CHECK> epi;
    epi.y = y;
    epi.yplus = yplus;
    epi.rl = rl;
    epi.ru = ru;
    epi.y0 = y0;
    epi.s = step_scalars<TX>(a.st, a.i_in_chunk, a.halpern, a.rho);
    epi.halpern = a.halpern;
    cta_spmv<TX, TV, TX, E, DualEpi<TX, CHECK>, COH>(a.blk, a.nblk, a.rp, a.ci, val, xbar, epi, sm);
    if (CHECK) write_partials(epi, a.part, s_red);
}

template <typename TV, typename TX, int E, bool CHECK>
__global__ void __launch_bounds__(kBlock, cta_min_blocks<TX, E>())
    k_primal(IterArgs a, const TV* __restrict__ val, const TX* __restrict__ y, TX* __restrict__ x,
             TX* __restrict__ xbar, TX* __restrict__ xplus, const TX* __restrict__ c, const TX* __restrict__ lo,
             const TX* __restrict__ up, const TX* __restrict__ x0) {
    __shared__ CtaShared<TX> sm[2];
    __shared__ double s_red[kWarps];
    if (a.st->done || a.st->phase != a.phase) return;
    primal_phase<TV, TX, E, CHECK, false>(a, val, y, x, xbar, xplus, c, lo, up, x0, sm, s_red);
}

template <typename TV, typename TX, int E, bool CHECK>
__global__ void __launch_bounds__(kBlock, cta_min_blocks<TX, E>())
    k_dual(IterArgs a, const TV* __restrict__ val, const TX* __restrict__ xbar, TX* __restrict__ y,
           TX* __restrict__ yplus, const TX* __restrict__ rl, const TX* __restrict__ ru, const TX* __restrict__ y0) {
    __shared__ CtaShared<TX> sm[2];
    __shared__ double s_red[kWarps];
    if (a.st->done || a.st->phase != a.phase) return;
    dual_phase<TV, TX, E, CHECK, false>(a, val, xbar, y, yplus, rl, ru, y0, sm, s_red);
}

// ---------------------------------------------------------------- KKT (FP64)

struct KktArgs {
    const int4* blk;
    int nblk;
    const int* rp;
    const int* ci;       // padded column indices
    const double* val;   // padded scaled FP64 values
    double* part;
    const DevState* st;
    int phase;
};

template <typename TX, int E>
__global__ void __launch_bounds__(kBlock, cta_min_blocks<double, E>())
    k_kkt_rows(KktArgs a, const TX* __restrict__ xplus, const TX* __restrict__ yplus, const double* __restrict__ dr,
               const double* __restrict__ rl, const double* __restrict__ ru) {
    __shared__ CtaShared<double> sm[2];
    __shared__ double s_red[kWarps];
    if (a.st->done || a.st->phase != a.phase) return;
    KktRowEpi<TX> epi;
    epi.dr = dr;
    epi.rl = rl;
    epi.ru = ru;
    epi.yplus = yplus;
    cta_spmv<double, double, TX, E>(a.blk, a.nblk, a.rp, a.ci, a.val, xplus, epi, sm);
    write_partials(epi, a.part, s_red);
}

template <typename TX, int E>
__global__ void __launch_bounds__(kBlock, cta_min_blocks<double, E>())
    k_kkt_cols(KktArgs a, const TX* __restrict__ xplus, const TX* __restrict__ yplus, const double* __restrict__ dc,
               const double* __restrict__ c, const double* __restrict__ l, const double* __restrict__ u) {
    __shared__ CtaShared<double> sm[2];
    __shared__ double s_red[kWarps];
    if (a.st->done || a.st->phase != a.phase) return;
    KktColEpi<TX> epi;
    epi.dc = dc;
    epi.c = c;
    epi.l = l;
    epi.u = u;
    epi.xplus = xplus;
    cta_spmv<double, double, TX, E>(a.blk, a.nblk, a.rp, a.ci, a.val, yplus, epi, sm);
    write_partials(epi, a.part, s_red);
}

}  // namespace nir
