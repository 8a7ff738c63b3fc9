/*
 * nir_lpgen.h -- seeded synthetic LP instances for the PDHG path.
 *
 * Every instance is an LP in the layout of the reference's `sov::Model`
 * (src/model/model.hpp:21-40): a CSC constraint matrix with int64 column
 * starts, int32 row indices and double values (src/core/csc_matrix.hpp:18-23),
 * column bounds collo/colup, row bounds rowlo/rowup (+-inf = no bound) and a
 * cost vector.  Instances are feasible and bounded by construction: a point
 * x0 inside the column box fixes the row bounds (b = A*x0 for equality rows)
 * and a dual guess y0 plus a slack s >= 0 fixes c = A^T*y0 + s.
 *
 * Kinds (sizes in brackets are the defaults, i.e. the full workloads):
 *   NIR_GEN_RANDOM_EQ     random sparse LP, Ax=b, 0<=x<=10, k distinct
 *                         N(0,1) entries per column     [m=2000 n=5000 k=8]
 *   NIR_GEN_ZIPF          power-law rows (Zipf 1.5, cap 2000), log-uniform
 *                         |a| in [1e-2,1e2] with random sign, 0<=x<=U,
 *                         U~U[1,100], Ax=b   [m=200000 n=500000 nnz~5e6]
 *   NIR_GEN_MULTIPERIOD   block-angular multi-period blending: 12 period
 *                         blocks, 10 U[0.5,2] entries per column inside its
 *                         block, +-1 inventory links between consecutive
 *                         periods, alternating =/<= rows   [m given, n=2.5m]
 *   NIR_GEN_BLEND_FAMILY  fixed blending matrix (from family_seed) with
 *                         demand rows (>=), quality and capacity rows (<=);
 *                         the instance seed perturbs demand b by
 *                         (1+0.2 N(0,1)) and c by (1+0.1 N(0,1))
 *                                                [m=20000 n=50000 nnz=400000]
 *   NIR_GEN_BADLY_SCALED  row and column scales 10^U[-d,d], half the
 *                         columns duplicated with a 1e-9 relative
 *                         perturbation, Ax=b, 0<=x<=10
 *                                              [m=50000 n=120000 nnz~1e6 d=4]
 *
 * All randomness comes from xoshiro256** seeded through splitmix64, so the
 * same (kind, seed, options) gives bit-identical arrays on every x86-64 host.
 */
#ifndef NIR_LPGEN_H
#define NIR_LPGEN_H

#include <stdint.h>
#include "nir_lp.h"

#ifdef __cplusplus
extern "C" {
#endif

enum {
    NIR_GEN_RANDOM_EQ = 1,
    NIR_GEN_ZIPF = 2,
    NIR_GEN_MULTIPERIOD = 3,
    NIR_GEN_BLEND_FAMILY = 4,
    NIR_GEN_BADLY_SCALED = 5
};

typedef struct nir_lpgen_opts {
    int32_t m;              /* rows; 0 = the kind's default                         */
    int32_t n;              /* columns; 0 = the kind's default                      */
    int64_t target_nnz;     /* ZIPF: total row length after rescaling; BLEND and
                               BADLY_SCALED: approximate nonzeros; 0 = default       */
    int32_t per_col;        /* RANDOM_EQ: entries per column; 0 = default           */
    int32_t zipf_cap;       /* ZIPF: longest row; 0 = 2000                          */
    uint64_t family_seed;   /* BLEND_FAMILY: seed of the fixed matrix (default 0)   */
    double scale_decades;   /* BADLY_SCALED: scales are 10^U[-d,d]; 0 = 4           */
} nir_lpgen_opts;

typedef struct nir_lpgen nir_lpgen;

/* Builds one instance.  Returns 0 on success, nonzero on bad arguments or
 * allocation failure (message via nir_lpgen_last_error). */
int nir_lpgen_create(int kind, uint64_t seed, const nir_lpgen_opts* opts, nir_lpgen** out);

/* Views into generator-owned arrays; valid until nir_lpgen_free. */
int nir_lpgen_view(const nir_lpgen* g, nir_lp_view* out);

/* The interior point x0 (ncol doubles) the instance was built around. */
const double* nir_lpgen_x0(const nir_lpgen* g);

/* Demand-row / cost perturbation factors of a BLEND_FAMILY instance
 * (the learned warm start's features); NULL for other kinds.
 * n_demand receives the number of demand rows (the first n_demand rows). */
const double* nir_lpgen_demand_factors(const nir_lpgen* g, int32_t* n_demand);
const double* nir_lpgen_cost_factors(const nir_lpgen* g);

void nir_lpgen_free(nir_lpgen* g);
const char* nir_lpgen_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
