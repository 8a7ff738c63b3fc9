/*
 * nir_mps.h -- C ABI of the multi-threaded MPS reader (libnir_mps.so).
 *
 * Replaces sov::MpsReader::read (src/io/mps_reader.hpp:15-304), the step
 * before the PDHG path on the CLI (`sovsolve model.mps --method pdhg`):
 * the same sections, conventions and model (first N row = objective,
 * further N rows dropped, MARKER INTORG/INTEND, RHS on the objective =
 * minus the offset, RANGES by row type, the negative-UP rule, BV/LI/UI/
 * FR/MI/PL/FX bounds, QUADOBJ/QMATRIX), the same duplicate merging
 * (CscMatrix::from_triplets, src/core/csc_matrix.hpp:30-96) and the same
 * validation and repair (Model::validate, src/model/model.hpp:117-178).
 * Numbers are converted exactly as std::stod does (D exponents allowed), so
 * the arrays are bit-identical to the reference's -- except that where one
 * (row, column) pair is given three or more times the summation order of
 * its duplicates may differ (the reference sorts them with an unstable
 * sort).
 *
 * The COLUMNS section is tokenised and converted by `threads` threads in
 * parallel and replayed in file order; the CSC is built in parallel.
 * Status codes are sov::Status (src/core/status.hpp:7-24): 0 valid,
 * 1 infeasible bounds (as Model::validate), 12 input error, 14 internal
 * (allocation) error.  Where the reference lets std::stod's exception
 * escape (a token that is not a number, or out of double range), this
 * reader returns 12 and names the token and its line.
 */
#ifndef NIR_MPS_H
#define NIR_MPS_H

#include <stdint.h>
#include "nir_lp.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct nir_mps nir_mps;

/* Parses `path` with `threads` threads (<= 0: all hardware threads).
 * On success *out owns the model; on failure *out is NULL and
 * nir_mps_last_error() says why. */
int nir_mps_read(const char* path, int32_t threads, nir_mps** out);

/* The model as read (after validation): matrix, cost, bounds and offset in
 * the file's own objective sense; *sense = 1 for MIN, -1 for MAX.  The
 * arrays stay valid until nir_mps_free. */
int nir_mps_view(const nir_mps* m, nir_lp_view* view, int32_t* sense);

/* Variable types, ncol bytes: 0 continuous, 1 integer, 2 binary
 * (sov::VarType). */
const int8_t* nir_mps_vartypes(const nir_mps* m);

/* The NAME line's model name ("mps_model" when there is none). */
const char* nir_mps_model_name(const nir_mps* m);

/* Column (of_rows = 0) or row (of_rows = 1) names, packed: name i is the
 * bytes [offsets[i], offsets[i+1]) of chars (not NUL-terminated). */
int nir_mps_names(const nir_mps* m, int32_t of_rows, const char** chars, const int64_t** offsets);

/* The quadratic objective block (QUADOBJ / QMATRIX) as an ncol x ncol CSC
 * (upper triangle as the reference stores it); *nnz = 0 for an LP. */
int nir_mps_quadratic(const nir_mps* m, int64_t* nnz, const int64_t** col_start, const int32_t** row_index,
                      const double** value);

/* Seconds spent per phase of the last successful read on this thread:
 * [0] file read, [1] line scan, [2] parallel COLUMNS parse, [3] ordered
 * replay, [4] CSC build, [5] other sections and validation. */
int nir_mps_timings(double* out6);

void nir_mps_free(nir_mps* m);

/* Writes an MPS file byte for byte as sov::MpsReader::write
 * (src/io/mps_reader.hpp:306-412) writes the same model: `sense` 1 / -1,
 * `vartype` (ncol bytes, may be NULL: all continuous), names NUL-terminated
 * (NULL: the reference's generated C<j> / R<i>), the quadratic block as an
 * upper-triangle CSC (qnnz = 0: none).  Formatting runs on `threads`
 * threads (<= 0: all).  Returns 0, 12 on a bad argument, 14 when the file
 * cannot be written. */
int nir_mps_write(const nir_lp_view* lp, const int8_t* vartype, int32_t sense, const char* model_name,
                  const char* const* col_names, const char* const* row_names, int64_t qnnz, const int64_t* q_start,
                  const int32_t* q_index, const double* q_value, int32_t threads, const char* path);

/* The message of the last failed call on this thread. */
const char* nir_mps_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* NIR_MPS_H */
