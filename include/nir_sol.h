/*
 * nir_sol.h -- C ABI of the SOL file I/O and the double-double solution
 * check (in libnir_mps.so).
 *
 * Replaces SolIo::write_sol / read_sol (src/io/sol_io.hpp:108-170) and
 * verify_solution (:25-106), which the CLI runs after the PDHG path
 * (include/sov/solver.hpp:262-313) and tools/checker.cpp runs on a file.
 * The outputs equal the reference's:
 *   - write: the same bytes;
 *   - read: the same x and objective.  Values are taken as `istream >>
 *     double` takes them (C locale: the longest prefix of sign, digits,
 *     point, exponent; a prefix that does not convert fully, or overflows,
 *     leaves the line unused).  The objective is taken as std::stod takes
 *     it;
 *   - verify: the same report, bit for bit.  The row activities are
 *     double-double sums in the reference's order (columns ascending within
 *     each row), computed in parallel over rows.  Where several items
 *     exceed the tolerance, the item named is the one the reference's loop
 *     names last.
 */
#ifndef NIR_SOL_H
#define NIR_SOL_H

#include <stdint.h>
#include "nir_lp.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Writes "# status <status_text>", "# objective %.17g", "# gap %.6e" and one
 * "<name> %.17g" line per column j < min(ncol, nx).  Names: col_names[j] for
 * j < n_names, else "C<j>".  Returns 0, or 14 when the file cannot be
 * opened. */
int nir_sol_write(const char* path, const char* status_text, double objective, double gap, int32_t ncol,
                  const double* x, int64_t nx, const char* const* col_names, int64_t n_names, int32_t threads);

/* Reads a solution file for a model with `ncol` named columns: x_out[ncol]
 * (0 where no line names the column; the last line for a name wins; where
 * two columns share a name, the later column gets the value).
 * *objective = the last "# objective" line's value (0 when none).
 * *n_objective_lines counts those lines; nir_sol_objective_token returns
 * their value tokens in order.  Returns 0; 14 when the file cannot be
 * opened; 12 when an objective token is not a number std::stod takes
 * (the reference throws there). */
int nir_sol_read(const char* path, int32_t ncol, const char* const* col_names, int32_t threads, double* x_out,
                 double* objective, int32_t* n_objective_lines);
const char* nir_sol_objective_token(int32_t k);

/* Model::eval_objective (src/model/model.hpp:73-98): the double-double
 * objective with offset, and the quadratic block when qnnz > 0. */
double nir_eval_objective(const nir_lp_view* lp, int64_t qnnz, const int64_t* q_start, const int32_t* q_index,
                          const double* q_value, const double* x);

typedef struct nir_verify_report {
    int32_t passed;
    int32_t worst_kind;     /* 0 none, 1 size mismatch, 2 NaN/Inf in variable, 3 lower bound, 4 upper bound,
                               5 integrality, 6 row lower bound, 7 row upper bound */
    int64_t worst_index;    /* the column or row the item names, -1 when none */
    double max_bound_viol;
    double max_row_viol;
    double max_int_viol;
    double computed_obj;
    double obj_rel_err;
} nir_verify_report;

/* verify_solution(model, x, claimed_obj, tol).  vartype: ncol bytes
 * (NULL: all continuous); nx is x's length; the objective is evaluated
 * as nir_eval_objective does. */
int nir_verify_solution(const nir_lp_view* lp, const int8_t* vartype, int64_t qnnz, const int64_t* q_start,
                        const int32_t* q_index, const double* q_value, const double* x, int64_t nx,
                        double claimed_obj, double tol, int32_t threads, nir_verify_report* out);

#ifdef __cplusplus
}
#endif

#endif /* NIR_SOL_H */
