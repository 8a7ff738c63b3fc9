/*
 * nir_oracle.h -- CPU oracle for the NIRNAYA PDHG path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA engine is compared
 * against: only the tests, the smoke check and the benchmark's CPU-baseline
 * leg may load it.  Nothing in the product (libnir_pdhg.so, the drop-in
 * header, the Python package) links, imports or calls it.
 *
 * Every function restates one piece of the reference in plain C99, with the
 * reference's own arithmetic order and no fused multiply-add (compile with
 * -ffp-contract=off), so results are bit-identical to the reference's:
 *   or_spmv / or_spmv_t       src/core/csc_matrix.hpp:99-120
 *   or_csc_from_triplets      src/core/csc_matrix.hpp:30-96
 *   or_ref_pdhg               src/gpu/pdhg_solver.hpp:25-107
 *   or_eval_objective         src/model/model.hpp:73-98 (LP part)
 *   or_verify                 src/io/sol_io.hpp:25-106
 *   or_dd_*                   src/core/dd_real.hpp:8-104
 * or_rel_kkt is the relative KKT error the engine stops on (the reference
 * has none); it is computed here with double-double accumulation.
 * Parity pinned by: tests/test_oracle.py against the reference's own known
 * answers (tests/unit_tests.cpp:29-76, :316-331; tools/bench_runner.cpp:24-39;
 * data/refinery/MRPL_Crude_Blending_LP.sol) and against the reference
 * compiled from source (oracle/Makefile -> oracle/_ref).
 */
#ifndef NIR_ORACLE_H
#define NIR_ORACLE_H

#include <stdint.h>
#include "../include/nir_lp.h"

#ifdef __cplusplus
extern "C" {
#endif

/* dd_real cancellation probe: returns (1e16 + 1 - 1e16) accumulated in dd */
double or_dd_cancellation_probe(double a, double b, double c);
double or_neumaier_probe(double a, double b, double c);

void or_spmv(const nir_lp_view* lp, const double* x, double* y);    /* y = A x  (nrow) */
void or_spmv_t(const nir_lp_view* lp, const double* x, double* y);  /* y = A' x (ncol) */

/* Canonical CSC from triplets: out-of-range and zero entries dropped,
 * duplicates summed in ascending-row order, zero sums dropped.
 * start_out has ncol+1 entries; index_out/value_out hold ntrip entries.
 * Returns nnz. */
int64_t or_csc_from_triplets(int32_t nrow, int32_t ncol, int64_t ntrip, const int32_t* trow,
                             const int32_t* tcol, const double* tval, int64_t* start_out,
                             int32_t* index_out, double* value_out);

typedef struct or_pdhg_out {
    int64_t iterations;     /* PdhgResult::iterations                                 */
    int32_t stopped;        /* 1 = the row-violation stop test fired, 0 = hit max_iters */
    double objective;       /* eval_objective(x) in double-double                     */
    double tau, sigma;      /* the fixed steps from the power iteration               */
    int64_t first_hit;      /* first probed iteration with rel KKT <= probe_tol, or -1 */
    double last_kkt;        /* rel KKT at the last probe (or NaN)                     */
} or_pdhg_out;

/* The reference PDHG loop.  max_iters is what the reference derives from
 * its options (max(5000, simplex_iter_limit/10)).  If probe_every > 0 the
 * relative KKT error of (x, y) is evaluated after every probe_every-th
 * iteration; with stop_at_probe != 0 the loop ends at the first probe that
 * reaches probe_tol.  x (ncol) and y (nrow) receive the final iterates. */
void or_ref_pdhg(const nir_lp_view* lp, int64_t max_iters, int64_t probe_every, double probe_tol,
                 int stop_at_probe, double* x, double* y, or_pdhg_out* out);

/* Model::eval_objective for an LP: offset + sum c_j x_j in double-double. */
double or_eval_objective(const nir_lp_view* lp, const double* x);

typedef struct or_verify_report {
    int32_t passed;
    double max_bound_viol;
    double max_row_viol;
    double computed_obj;
    double obj_rel_err;
} or_verify_report;

/* verify_solution: relative bound and row violations (rows in
 * double-double), objective recomputed in double-double. */
void or_verify(const nir_lp_view* lp, const double* x, double claimed_obj, double tol,
               or_verify_report* rep);

typedef struct or_kkt {
    double rel_primal;   /* ||A x - proj_[rl,ru](A x)||_2 (+ column box) / (1 + ||rhs||_2) */
    double rel_dual;     /* ||c - A'y - lambda||_2 (+ wrong-sign y) / (1 + ||c||_2)        */
    double rel_gap;      /* |pobj - dobj| / (1 + |pobj| + |dobj|)                          */
    double rel_kkt;      /* max of the three                                                */
    double pobj, dobj;
    double max_rel_row_viol; /* max_i viol_i / (1 + |bound_i|), the checker's row measure  */
} or_kkt;

void or_rel_kkt(const nir_lp_view* lp, const double* x, const double* y, or_kkt* out);

#ifdef __cplusplus
}
#endif
#endif
