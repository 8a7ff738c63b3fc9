/*
 * nir_facade.h -- C ABI of the multi-threaded presolve and scaling that
 * Solver::solve runs before the PDHG path (libnir_facade.so).
 *
 * nir_presolve replaces sov::Presolver::presolve
 * (src/presolve/presolve.hpp:32-345): the same rounds of fixed columns
 * (R4), empty and singleton rows (R1, R3), activity-based infeasibility,
 * redundant and forcing rows and integer bound tightening (R6, R5, R14,
 * R7), and empty columns (R2), with the same tolerances, in the same
 * order.  So the reduced model, the maps, the fixed values, the counters
 * and the status are bit-identical to the reference's.
 * The parallel parts:
 *   - detecting fixed columns, counting row entries, computing every row's
 *     activity bounds and finding empty columns, all over rows or columns;
 *   - applying the reductions in the reference's order on one thread,
 *     recomputing a row's activity there when an earlier reduction in the
 *     same pass touched one of its columns.
 *
 * nir_scale replaces sov::scale_model (src/model/scaling.hpp:56-154):
 * geometric-mean equilibration, rounded to powers of two, computed in
 * parallel.  Its min/max reductions are order-free, so the scales and the
 * scaled arrays are bit-identical.
 *
 * Status codes are sov::Status (src/core/status.hpp:7-24).
 */
#ifndef NIR_FACADE_H
#define NIR_FACADE_H

#include <stdint.h>
#include "nir_lp.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct nir_presolved nir_presolved;

/* Presolves the internal-minimisation model (the reference's presolve
 * level > 0 on a model without a quadratic block; a caller with level <= 0
 * or a QP copies the model, as the reference does).  vartype: ncol bytes,
 * 0 continuous, 1 integer, 2 binary (NULL: all continuous).
 * threads <= 0: all hardware threads.  Returns 0 when the presolve ran;
 * its outcome is read with nir_presolved_status.  12 is returned on a bad
 * argument, 14 on an internal error. */
int nir_presolve(const nir_lp_view* lp, const int8_t* vartype, int32_t max_rounds, int32_t threads,
                 nir_presolved** out);

/* status: 0 (reduced model to solve, or solved in presolve), 1 infeasible,
 * 2 unbounded; counters = {rows_removed, cols_removed, bound_tightenings}. */
int nir_presolved_status(const nir_presolved* r, int32_t* status, int32_t* solved_in_presolve,
                         int32_t* counters3);

/* The reduced model (empty when presolve stopped with infeasible or
 * unbounded) and its variable types; valid until nir_presolved_free. */
int nir_presolved_reduced(const nir_presolved* r, nir_lp_view* reduced, const int8_t** vartype);

/* orig_col_map[ncol_reduced], orig_row_map[nrow_reduced]; fixed_x and
 * is_col_fixed have one entry per original column. */
int nir_presolved_maps(const nir_presolved* r, const int32_t** orig_col_map, const int32_t** orig_row_map,
                       const double** fixed_x, const uint8_t** is_col_fixed);

void nir_presolved_free(nir_presolved* r);

/* scale_model's scales and scaled arrays.  Outputs: R[nrow], C[ncol],
 * *active; cost, collo, colup, rowlo, rowup (the size of the inputs) and
 * value[nnz] scaled; q_value[qnnz] scaled when qnnz > 0.  When scaling is
 * off or not needed (*active = 0) the outputs are copies of the inputs and
 * the scales are 1. */
int nir_scale(const nir_lp_view* lp, const int8_t* vartype, int32_t enable, int64_t qnnz, const int64_t* q_start,
              const int32_t* q_index, const double* q_value, int32_t threads, double* R, double* C,
              int32_t* active, double* cost, double* collo, double* colup, double* value, double* rowlo,
              double* rowup, double* q_value_out);

const char* nir_facade_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* NIR_FACADE_H */
