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
// primal phase over all warp row blocks of A', a grid barrier, the dual
// phase over A, a grid barrier, and so on.  The row-block code and the
// per-row summation order are those of k_primal / k_dual, so the iterates
// are bit-identical to the two-kernel path; the gathers go through L2
// (gather_ld<true>) because the gathered vectors change inside the launch.
// Every warp keeps the same row blocks in every iteration, so a row's own
// x / y entries are read back only by the warp that wrote them.
//
// The barrier is a counter and a generation word in global memory.  A
// cooperative launch makes every CTA co-resident, so it always completes;
// its waits are still bounded (limit_cycles of the SM clock), after which
// the CTA raises the error word, every other waiting CTA sees it and
// leaves, and the kernel marks the solve done with NIR_STATUS_INTERNAL_ERROR.
#pragma once

#include "k_adaptive.cuh"

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

template <typename T>
struct ChunkPtrs {
    const T *valAt, *valA;
    T *x, *xb, *xp, *y, *yp;
    const T *c, *l, *u, *x0, *rl, *ru, *y0;
};

template <typename T>
__global__ void __launch_bounds__(kBlock, iter_min_blocks<T>()) k_chunk(IterArgs ap, IterArgs ad, ChunkPtrs<T> v,
                                                                        int i0, int iters, GridSync gs, DevState* st) {
    __shared__ double s_red[kWarps];
    // no kernel changes the state during a chunk: every CTA decides alike
    if (ap.st->done || ap.st->phase != ap.phase) return;
    for (int i = i0; i < i0 + iters; ++i) {
        ap.i_in_chunk = i;
        ad.i_in_chunk = i;
        primal_phase<T, false, true>(ap, v.valAt, v.y, v.x, v.xb, v.xp, v.c, v.l, v.u, v.x0, s_red);
        if (!grid_sync(gs)) break;
        dual_phase<T, false, true>(ad, v.valA, v.xb, v.y, v.yp, v.rl, v.ru, v.y0, s_red);
        if (!grid_sync(gs)) break;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && *(volatile int*)gs.err) {
        st->done = 1;
        st->status = 14;  // NIR_STATUS_INTERNAL_ERROR
    }
}

}  // namespace nir
