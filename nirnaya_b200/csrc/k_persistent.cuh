// Persistent chunk kernel (nir_pdhg_params.persistent = 1).
//
// Measured on B200 it is slower than the default path (one kernel per
// half-iteration, chunks captured in CUDA graphs): two grid barriers per
// iteration cost more than two graph-launched kernels, 9.8 vs 6.7 us per
// iteration on a 40k-nonzero LP and 18.6 vs 14.7 us at 500k.  It stays as
// an option because its iterates are bit-identical and its bounded waits
// are tested.
//
// One cooperative launch runs the non-check iterations of a chunk: the
// primal phase over all blocks of A', a grid barrier, the dual phase over A,
// a grid barrier, and so on.  The block code and the per-row summation
// order are those of k_primal / k_dual, so the iterates are bit-identical
// to the two-kernel path; the gathers go through L2 because the gathered
// vectors change inside the launch.  Every warp (warp layout) or CTA (CTA
// layout) keeps the same blocks in every iteration, so a row's own x / y
// entries are read back only by the one that wrote them.
//
// The barrier is a counter and a generation word in global memory.  A
// cooperative launch makes every CTA co-resident, so it always completes;
// its waits are still bounded (limit_cycles of the SM clock), after which
// the CTA raises the error word, every other waiting CTA sees it and
// leaves, and the kernel marks the solve done with NIR_STATUS_INTERNAL_ERROR.
#pragma once

#include "k_batch.cuh"
#include "k_iter.cuh"

namespace nir {

struct GridSync {
    unsigned* count;
    unsigned* gen;
    int* err;
    unsigned nblocks;        // CTAs that must arrive
    long long limit_cycles;  // bound on one wait
};

__device__ __forceinline__ bool grid_sync(const GridSync& g) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* vgen = g.gen;
        volatile int* verr = g.err;
        const unsigned my = *vgen;
        __threadfence();
        if (atomicAdd(g.count, 1u) + 1u == g.nblocks) {
            atomicExch(g.count, 0u);
            __threadfence();
            atomicAdd(g.gen, 1u);
        } else {
            const long long t0 = clock64();
            while (*vgen == my) {
                if (*verr) break;
                if (clock64() - t0 > g.limit_cycles) {
                    atomicExch(g.err, 1);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __shared__ int ok;
    if (threadIdx.x == 0) ok = (*(volatile int*)g.err == 0);
    __syncthreads();
    const bool r = ok != 0;
    __syncthreads();  // ok is rewritten by the next barrier
    return r;
}

template <typename TV, typename TX>
struct ChunkPtrs {
    const TV *valAt, *valA;
    TX *x, *xb, *xp, *y, *yp;
    const TX *c, *l, *u, *x0, *rl, *ru, *y0;
};

// LP / LD: layouts of A' (primal phase) and A (dual phase).  A kernel that
// mixes the layouts needs both kinds of shared memory; its dynamic part is
// the warp layout's.
template <int LP, int LD, typename TV, typename TX>
__global__ void __launch_bounds__(kBlock, (lay_min_blocks<LP, TV, TX>() < lay_min_blocks<LD, TV, TX>() ? lay_min_blocks<LP, TV, TX>()
                                                                                                : lay_min_blocks<LD, TV, TX>()))
    k_chunk(IterArgs ap, IterArgs ad, ChunkPtrs<TV, TX> v, int i0, int iters, GridSync gs, DevState* st) {
    __shared__ double s_red[kWarps];
    // no kernel changes the state during a chunk: every CTA decides alike
    if (ap.st->done || ap.st->phase != ap.phase) return;
    for (int i = i0; i < i0 + iters; ++i) {
        ap.i_in_chunk = i;
        ad.i_in_chunk = i;
        primal_phase<LP, TV, TX, false, true>(ap, v.valAt, v.y, v.x, v.xb, v.xp, v.c, v.l, v.u, v.x0, s_red);
        if (!grid_sync(gs)) break;
        dual_phase<LD, TV, TX, false, true>(ad, v.valA, v.xb, v.y, v.yp, v.rl, v.ru, v.y0, s_red);
        if (!grid_sync(gs)) break;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && *(volatile int*)gs.err) {
        st->done = 1;
        st->status = 14;  // NIR_STATUS_INTERNAL_ERROR
    }
}

// The batched chunk: the same loop over the batch's blocks (k_batch.cuh),
// each block running only while its instance is active.  No kernel changes
// an instance's state inside the launch, so every CTA skips the same
// blocks.  On a barrier that gave up, every instance still running ends
// with NIR_STATUS_INTERNAL_ERROR.
template <int LP, int LD, typename TV, typename TX>
__global__ void __launch_bounds__(kBlock, (lay_min_blocks<LP, TV, TX, true>() < lay_min_blocks<LD, TV, TX, true>() ? lay_min_blocks<LP, TV, TX, true>()
                                                                                                : lay_min_blocks<LD, TV, TX, true>()))
    k_bchunk(BatchArgs ap, BatchArgs ad, ChunkPtrs<TV, TX> v, int i0, int iters, GridSync gs, DevState* insts,
             int count) {
    __shared__ double s_red[kWarps];
    for (int i = i0; i < i0 + iters; ++i) {
        ap.i_in_chunk = i;
        ad.i_in_chunk = i;
        PrimalEpi<TX, false> pe;
        pe.x = v.x;
        pe.xbar = v.xb;
        pe.xplus = v.xp;
        pe.c = v.c;
        pe.lo = v.l;
        pe.up = v.u;
        pe.x0 = v.x0;
        pe.halpern = ap.halpern;
        lay_spmv_batch<LP, TX, TV, TX, PrimalEpi<TX, false>, true>(
            ap, v.valAt, v.y, pe,
            [&](PrimalEpi<TX, false>& e, const DevState& s) { e.s = step_scalars<TX>(&s, ap.i_in_chunk, ap.halpern, ap.rho); },
            s_red);
        if (!grid_sync(gs)) break;
        DualEpi<TX, false> de;
        de.y = v.y;
        de.yplus = v.yp;
        de.rl = v.rl;
        de.ru = v.ru;
        de.y0 = v.y0;
        de.halpern = ad.halpern;
        lay_spmv_batch<LD, TX, TV, TX, DualEpi<TX, false>, true>(
            ad, v.valA, v.xb, de,
            [&](DualEpi<TX, false>& e, const DevState& s) { e.s = step_scalars<TX>(&s, ad.i_in_chunk, ad.halpern, ad.rho); },
            s_red);
        if (!grid_sync(gs)) break;
    }
    if (blockIdx.x == 0 && *(volatile int*)gs.err) {
        for (int k = threadIdx.x; k < count; k += kBlock) {
            DevState& s = insts[k];
            if (!s.done) {
                s.done = 1;
                s.status = 14;  // NIR_STATUS_INTERNAL_ERROR
            }
        }
    }
}

}  // namespace nir
