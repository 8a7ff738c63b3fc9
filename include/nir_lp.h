/*
 * nir_lp.h -- the LP as it crosses the C ABI.
 *
 * Mirrors the reference's internal minimisation `sov::Model` for a
 * continuous LP (src/model/model.hpp:21-40): cost, collo/colup, rowlo/rowup
 * and the CSC matrix A of `sov::CscMatrix` (src/core/csc_matrix.hpp:18-23:
 * `std::vector<Off> start` with Off=int64, `std::vector<Idx> index` with
 * Idx=int32, `std::vector<double> value`; src/core/types.hpp:12-13).
 * A bound whose magnitude is >= 1e20 or that is not finite is "no bound",
 * as `is_finite_bound` decides (src/core/types.hpp:49-51).
 * All pointers are caller-owned host memory and are only read.
 */
#ifndef NIR_LP_H
#define NIR_LP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct nir_lp_view {
    int32_t nrow;
    int32_t ncol;
    int64_t nnz;
    const int64_t* col_start;  /* ncol+1, col_start[0]=0, nondecreasing        */
    const int32_t* row_index;  /* nnz, strictly ascending inside each column   */
    const double* value;       /* nnz, finite, nonzero                         */
    const double* cost;        /* ncol                                         */
    const double* collo;       /* ncol                                         */
    const double* colup;       /* ncol                                         */
    const double* rowlo;       /* nrow                                         */
    const double* rowup;       /* nrow                                         */
    double obj_offset;
} nir_lp_view;

#ifdef __cplusplus
}
#endif
#endif
