/*
 * nir_pdhg.h -- C ABI of the B200 PDHG / PDLP engine (libnir_pdhg.so).
 *
 * This is the boundary a caller of the reference's PDHG path binds.  It
 * replaces, one for one:
 *
 *   sov::PdhgSolver::solve(const Model&, const Options&, const Deadline&)
 *       src/gpu/pdhg_solver.hpp:25-107         -> nir_pdhg_solve_lp, or
 *                                                 nir_pdhg_create + nir_pdhg_solve
 *   sov::PdhgResult {status, objective, x, y, iterations}
 *       src/gpu/pdhg_solver.hpp:14-20          -> status return, x_out, y_out,
 *                                                 nir_pdhg_info
 *   sov::Deadline::expired() (stop flag, wall clock, work counter)
 *       src/core/timer.hpp:41-46, polled every 256 iterations at
 *       src/gpu/pdhg_solver.hpp:63            -> the poll callback, called on
 *                                                 the host between launch chunks
 *   sov::Options::simplex_iter_limit -> max_iters
 *       src/gpu/pdhg_solver.hpp:60             -> nir_pdhg_params.max_iters
 *   sov::Status (src/core/status.hpp:7-24)     -> NIR_STATUS_* (same values)
 *
 * The LP comes in the reference's layout (nir_lp.h).  All pointers in
 * the signatures are host pointers owned by the caller; device memory is
 * owned by the handle.  No C++ exception crosses this boundary: every entry
 * point returns a status and sets a thread-local message
 * (nir_pdhg_last_error), as src/driver/c_api.cpp:56-59, :136-139 do.
 *
 * There is no CPU fallback: without a usable CUDA device nir_pdhg_create
 * fails with NIR_STATUS_INTERNAL_ERROR.
 */
#ifndef NIR_PDHG_H
#define NIR_PDHG_H

#include <stdint.h>
#include "nir_lp.h"
#include "nir_sol.h" /* nir_verify_report */

#ifdef __cplusplus
extern "C" {
#endif

/* sov::Status values (src/core/status.hpp:7-24). */
enum {
    NIR_STATUS_OPTIMAL = 0,
    NIR_STATUS_TIME_LIMIT = 4,
    NIR_STATUS_ITERATION_LIMIT = 6,
    NIR_STATUS_INTERRUPTED = 10,
    NIR_STATUS_NUMERICAL_TROUBLE = 11,
    NIR_STATUS_INPUT_ERROR = 12,
    NIR_STATUS_INTERNAL_ERROR = 14
};

/* Algorithms.
 *  REFERENCE  the reference loop itself (src/gpu/pdhg_solver.hpp:33-105) in
 *             FP64, reproduced bit for bit: same power iteration, fixed
 *             steps 0.85/||A||, box-midpoint start, its absolute row-violation
 *             stop test every 32 iterations, and the same iteration count.
 *             Unlike the reference it reports NIR_STATUS_ITERATION_LIMIT
 *             (not Optimal) when max_iters is reached without the stop test.
 *  PDHG       the same unrestarted iteration on the fast kernels, stopping on
 *             the relative KKT error (precision selectable).
 *  PDLP       diagonal preconditioning (Ruiz + Pock-Chambolle), reflected
 *             Halpern PDHG with fixed-point-residual restarts, adaptive primal
 *             weight, relative-KKT stop; mixed precision by default. */
enum { NIR_ALGO_REFERENCE = 0, NIR_ALGO_PDHG = 1, NIR_ALGO_PDLP = 2 };

/* Precision of matrix, iterates and SpMV.  KKT residuals, restart
 * criterion, primal weight and objective are always FP64, on the FP64
 * matrix.  FP64: FP64 matrix values and iterates.  MIXED: FP32 matrix
 * values (8 instead of 12 bytes per nonzero streamed) with FP64 iterates and
 * accumulation, then the FP64 values as a polish when the KKT error stops
 * improving (the iterates carry on).  FP32: FP32 values, iterates and
 * accumulation throughout. */
enum { NIR_PREC_FP64 = 0, NIR_PREC_MIXED = 1, NIR_PREC_FP32 = 2 };

typedef struct nir_pdhg_params {
    int32_t algorithm;            /* NIR_ALGO_*                                  (PDLP)  */
    int32_t precision;            /* NIR_PREC_*                                  (MIXED) */
    double tol;                   /* relative KKT target                         (1e-6)  */
    double feas_tol;              /* also require max_i viol_i/(1+|b_i|) <= this (0=off) */
    int64_t max_iters;            /* iteration cap                               (1e6)   */
    double time_limit;            /* seconds of solve time; <= 0 = none          (0)     */
    int32_t check_every;          /* iterations per restart/KKT check            (64)    */
    int32_t ruiz_iters;           /* Ruiz l-inf equilibration passes             (10)    */
    int32_t pock_chambolle;       /* 1 = one Pock-Chambolle (alpha=1) pass        (1)     */
    double reflection;            /* Halpern reflection rho in [0,1]             (1.0)   */
    double restart_sufficient;    /* restart if r <= this * r_anchor             (0.2)   */
    double restart_necessary;     /* ... or r <= this * r_anchor and r grew      (0.8)   */
    double restart_artificial;    /* ... or inner iterations >= this * total     (0.36)  */
    double primal_weight_smoothing; /* theta of the log-space weight update      (0.5)   */
    double step_factor;           /* eta = step_factor / ||A||_2 estimate        (0.998) */
    int32_t power_iters;          /* power-iteration rounds for ||A||_2          (64)    */
    int32_t polish_stall_checks;  /* MIXED: FP64 polish once KKT <= 30 tol has not
                                     improved 0.8x for this many checks and half
                                     of the checks so far                         (40)   */
    double polish_switch_kkt;     /* MIXED: ... or as soon as KKT <= this        (0)     */
    int32_t spmv_block_nnz;       /* SpMV layout of both orientations: 32, 64, 128 or 256 =
                                     warp row blocks of that many nonzeros, 1024 = CTA
                                     blocks with a segmented reduction; 0 = autotuned
                                     per orientation                               (0) */
    int32_t use_graphs;           /* capture launch chunks in CUDA graphs        (1)     */
    int32_t verbose;              /* 1 = one line per check on stderr            (0)     */
    int32_t restart_anchor;       /* residual the restart tests compare with: 0 = first
                                     check after a restart, 1 = at the restart     (1)    */
    int32_t polish_fresh;         /* MIXED hand-over to FP64: 2 = pure change of precision
                                     (iterate, anchor and counters carry on), 1 = fresh
                                     FP64 solve from the last FP32 point with the initial
                                     weight, 0 = as 1 but keeping the weight     (2)    */
    const double* x_init;         /* warm start in original space, ncol, or NULL          */
    const double* y_init;         /* warm start duals, nrow, or NULL.  Either may be host
                                     memory or device memory (unified addressing): a
                                     device-resident start is copied on the device, with
                                     no trip through the host except where the engine
                                     remaps it (its row order, parallel columns); it must
                                     be complete before the call                          */
    double omega_init;            /* warm-start primal weight; <= 0 = default             */
    double primal_weight_decades; /* the weight stays within this many decades of
                                     its initial value                           (1.0)   */
    int32_t persistent;           /* PDHG/PDLP: 1 = run a chunk's non-check iterations in
                                     one cooperative launch with grid barriers (bit-identical
                                     iterates); 0 = one launch per half-iteration inside CUDA
                                     graphs, measured faster on B200 (6.7 vs 9.8 us per
                                     iteration at 40k nonzeros: two grid barriers cost more
                                     than two graph-launched kernels); 2 = test of the
                                     barrier's bounded wait (one CTA too many: the solve
                                     must end with NIR_STATUS_INTERNAL_ERROR in ~0.1 s)  (0) */
    int32_t pad_;
} nir_pdhg_params;

typedef struct nir_pdhg_info {
    int32_t status;               /* NIR_STATUS_*                                        */
    int32_t restarts;
    int64_t iterations;           /* all iterations (FP32 + FP64)                        */
    int64_t iterations_fp64;      /* of which in FP64 (polish, or all for FP64)          */
    double objective;             /* c'x + offset in double-double (eval_objective)      */
    double rel_kkt, rel_primal, rel_dual, rel_gap;  /* at the returned point, FP64       */
    double max_rel_row_viol;      /* max_i viol_i / (1 + |b_i|) at the returned point    */
    double primal_weight, step_size;
    double setup_seconds;         /* preconditioning, norm estimate, graph capture       */
    double solve_seconds;         /* iterations until the returned point                 */
    double time_to_fp64_seconds;  /* when the FP64 polish began (MIXED), else 0          */
    int32_t kernel_launches;      /* engine kernels launched by this solve               */
    int32_t parallel_groups;      /* groups of parallel columns re-expressed for the solve
                                     (each adds one row; 0 = the LP as given)             */
    int64_t iterations_to_tol;    /* NIR_ALGO_REFERENCE with tol > 0: first iteration (a
                                     multiple of 32) whose iterate has rel KKT <= tol,
                                     -1 if none; the iterates are not changed by the probe.
                                     Other algorithms: the iterations when they stopped at
                                     tol, else -1                                         */
} nir_pdhg_info;

typedef struct nir_pdhg nir_pdhg;

/* Fills *p with the defaults shown above. */
int nir_pdhg_default_params(nir_pdhg_params* p);

/* Copies the LP to `device`, builds CSR(A) and CSR(A^T) there.
 * Errors: NIR_STATUS_INPUT_ERROR (malformed LP), NIR_STATUS_INTERNAL_ERROR
 * (no device / out of device memory). */
int nir_pdhg_create(const nir_lp_view* lp, int device, nir_pdhg** out);

/* Groups of parallel columns the handle re-expresses before a PDHG / PDLP
 * solve: column j' joins the group of the earlier column j when both have
 * the same row pattern and A_j' = lambda A_j + eps with max|eps| at most
 * 1e-6 max|A_j'|.  Each group adds one row to the LP the iterations run on
 * (x_j = v - sum lambda x_j' with x_j's bounds) and moves the split of the
 * group out of the matrix, where PDHG cannot resolve it; the result is
 * mapped back and its KKT error evaluated on the LP as given.  Host only,
 * no device needed.  rep_of (ncol, or NULL): each column's representative,
 * -1 for none; lambda (ncol, or NULL): its factor; *groups: the number of
 * groups.  Setting NIR_PDHG_PARALLEL_COLUMNS=0 in the environment turns the
 * re-expression off for handles created afterwards.  No counterpart in the
 * reference (its presolve has no parallel-column rule). */
int nir_pdhg_parallel_groups(const nir_lp_view* lp, int32_t* rep_of, double* lambda, int32_t* groups);

/* Replaces cost, column and row bounds of an existing handle (same
 * matrix); NULL leaves an array unchanged.  Used by families of LPs that
 * share A (warm-start training). */
int nir_pdhg_update_vectors(nir_pdhg* h, const double* cost, const double* collo, const double* colup,
                            const double* rowlo, const double* rowup);

/* Solves.  poll(ctx) is called on the host between launch chunks (at least
 * every 256 iterations); a nonzero return stops the solve with
 * NIR_STATUS_TIME_LIMIT, like Deadline::expired().  x_out (ncol) and y_out
 * (nrow) may be NULL.  y follows the reference's sign convention
 * (y += sigma*(clamp(Ax - y/sigma) - Ax): y > 0 where a row's lower bound
 * binds).  Returns info->status. */
int nir_pdhg_solve(nir_pdhg* h, const nir_pdhg_params* p, int (*poll)(void* ctx), void* poll_ctx,
                   double* x_out, double* y_out, nir_pdhg_info* info);

/* create + solve + free in one call (what the drop-in PdhgSolver uses). */
int nir_pdhg_solve_lp(const nir_lp_view* lp, int device, const nir_pdhg_params* p, int (*poll)(void* ctx),
                      void* poll_ctx, double* x_out, double* y_out, nir_pdhg_info* info);

void nir_pdhg_free(nir_pdhg* h);
const char* nir_pdhg_last_error(void);

/* --- kernel-level entry points (parity tests and the benchmark) --- */

/* One SpMV with the handle's unscaled matrix, host in/out.
 * transpose=0: y = A x (x: ncol, y: nrow); 1: y = A' x.
 * kernel: 0 = reference-order sequential FP64 (bit-identical to
 * CscMatrix::spmv / spmv_transpose), 1 = CSR-adaptive FP64,
 * 2 = CSR-adaptive FP32 (values and x rounded to FP32, FP32 accumulation). */
int nir_pdhg_spmv(nir_pdhg* h, int transpose, int kernel, const double* x, double* y);

/* Times `reps` back-to-back launches of one SpMV kind on device-resident
 * data (optionally flushing L2 before each) and reports the mean duration
 * in microseconds measured with CUDA events on the launching stream. */
int nir_pdhg_time_spmv(nir_pdhg* h, int transpose, int kernel, int reps, int flush_l2, double* usec);

/* The same two, with more kernel kinds and the CTA-block capacity:
 *   0-2  as nir_pdhg_spmv (block_nnz ignored)
 *   3    CTA-block SpMV (segmented reduction, aligned 128-bit stream loads), FP64
 *   4    CTA-block SpMV, FP32 values, x and accumulation
 *   5    CTA-block SpMV, FP32 values with FP64 x and accumulation
 *   6-9  (timing only) the row-less ceilings: the stream of indices and
 *        values with the gathers of x (6 FP64, 7 FP32) or without them
 *        (8 FP64, 9 FP32), with no row structure at all
 * block_nnz: CTA-block capacity for 3-5 (256, 512, 1024 or 2048; 0 = 1024,
 * the capacity of the iteration kernels); nir_pdhg_time_kernel also takes
 * the warp row-block capacity for 1-2 (32, 64, 128 or 256; 0 = the current
 * blocks).
 * No counterpart in the reference: measurement of the SpMV kernels that
 * replace CscMatrix::spmv / spmv_transpose (src/core/csc_matrix.hpp:99-120). */
int nir_pdhg_spmv_kernel(nir_pdhg* h, int transpose, int kernel, int block_nnz, const double* x, double* y);
int nir_pdhg_time_kernel(nir_pdhg* h, int transpose, int kernel, int block_nnz, int reps, int flush_l2,
                         double* usec);

typedef struct nir_pdhg_kernel_time {
    /* index 0: chunks iterating in FP32, index 1: chunks iterating in FP64 */
    double primal_us[2]; /* mean duration of the fused A'y + primal-update kernel */
    double dual_us[2];   /* mean duration of the fused A x + dual-update kernel   */
    double iter_us[2];   /* mean time of one iteration (kernels + check share)    */
    int64_t samples[2];  /* timed chunks                                           */
} nir_pdhg_kernel_time;

/* Event timing of the hot kernels during the last solve (when enabled by
 * nir_pdhg_set_profiling before the solve). */
int nir_pdhg_set_profiling(nir_pdhg* h, int on);
int nir_pdhg_kernel_times(nir_pdhg* h, nir_pdhg_kernel_time* out);

/* Steady-state CUDA-event timing of the two fused iteration kernels (A' y
 * + primal step, A x-bar + dual step) after a PDHG/PDLP solve on this handle:
 * `reps` back-to-back launches of each kernel alone and of the pair, on the
 * last solve's layout and state.  precision: NIR_PREC_FP64 (FP64 values and
 * iterates), NIR_PREC_MIXED (FP32 values, FP64 iterates) or NIR_PREC_FP32.
 * The kernels overwrite the handle's iterates (not x_out / y_out of the
 * solve, nor the point nir_pdhg_verify checks); the next solve starts anew.
 * No counterpart in the reference. */
int nir_pdhg_time_iteration(nir_pdhg* h, int precision, int reps, double* primal_us, double* dual_us,
                            double* pair_us);

/* KKT history of the last PDHG/PDLP solve, one entry per check, oldest
 * first: 8 doubles per entry (iteration, rel KKT, rel primal, rel dual,
 * rel gap, fixed-point residual, primal weight, phase).  Returns the number
 * of entries written (at most max_entries and the last 4096 checks). */
int nir_pdhg_history(nir_pdhg* h, double* out, int max_entries);

/* Matrix and layout facts: nnz, rows, row blocks of each orientation. */
typedef struct nir_pdhg_layout {
    int32_t nrow, ncol;
    int64_t nnz;
    int32_t blocks_a, blocks_at;        /* SpMV blocks of A and A' of the last solve */
    int32_t block_nnz;                  /* nonzeros per block of A: 32..256 for warp row
                                           blocks, 1024 for CTA blocks               */
    int64_t device_bytes;               /* device memory held by the handle    */
    int32_t block_nnz_at;               /* the same for A'                         */
    int32_t pad_;
} nir_pdhg_layout;
int nir_pdhg_get_layout(nir_pdhg* h, nir_pdhg_layout* out);

/* --- batched solves ---
 *
 * Many LPs of uneven sizes in one handle, solved by the PDLP iteration with
 * one launch per half-iteration for the whole batch.  The reference solves
 * one Model per PdhgSolver::solve call (src/gpu/pdhg_solver.hpp:25); a
 * batch replaces `count` such calls.  Every instance keeps its own step
 * sizes, primal weight, restart state, precision phase and convergence flag
 * on the device and stops on its own relative KKT error; converged
 * instances drop out of the work.  In MIXED precision the instances that
 * stall in FP32 continue in FP64 after the FP32 pass. */
typedef struct nir_pdhg_batch nir_pdhg_batch;

/* lps[0..count): the instances (host arrays, copied). */
int nir_pdhg_batch_create(const nir_lp_view* lps, int32_t count, int device, nir_pdhg_batch** out);

/* x_out / y_out receive the instances' primal / dual vectors concatenated in
 * instance order (sum of ncol, sum of nrow doubles; may be NULL); infos[i]
 * (may be NULL) the result of instance i; total the batch (status = the
 * first non-optimal instance status, or OPTIMAL).  params->algorithm must be
 * NIR_ALGO_PDLP; warm starts are not taken. */
int nir_pdhg_batch_solve(nir_pdhg_batch* b, const nir_pdhg_params* params, int (*poll)(void* ctx), void* poll_ctx,
                         double* x_out, double* y_out, nir_pdhg_info* infos, nir_pdhg_info* total);

void nir_pdhg_batch_free(nir_pdhg_batch* b);

/* --- the solution check on the device ---
 *
 * verify_solution (src/io/sol_io.hpp:25-106) run on the GPU against the LP
 * the handle holds.  *out receives what nir_verify_solution
 * (include/nir_sol.h) reports on the host for the same LP, point, integer
 * marks, claimed objective and tolerance, bit for bit, with no quadratic part
 * (the PDHG path takes LPs only):
 *   - row activities are double-double sums in the reference's order,
 *     one row per thread;
 *   - the objective is the double-double sum of Model::eval_objective
 *     (src/model/model.hpp:73-98).
 * The host check in libnir_mps.so remains the reference for this one.
 *
 * x: ncol host doubles, or NULL for the point the last nir_pdhg_solve on this
 * handle returned, which is still on the device (NULL before any solve is an
 * input error).  vartype: ncol bytes (1 integer, 2 binary) or NULL
 * (all continuous).  claimed_obj: NaN when there is none (obj_rel_err is then
 * 0).  Returns 0, or NIR_STATUS_INPUT_ERROR / NIR_STATUS_INTERNAL_ERROR with
 * nir_pdhg_last_error(). */
int nir_pdhg_verify(nir_pdhg* h, const double* x, const int8_t* vartype, double claimed_obj, double tol,
                    nir_verify_report* out);

/* The same check for every instance of a batch, in one pass over the
 * batch's device matrix, replacing `count` host verify_solution calls.
 *   - x: the instances' points concatenated in instance order (sum of ncol
 *     doubles), or NULL for the points the last nir_pdhg_batch_solve
 *     returned, which are still on the device.  x == NULL before any batch
 *     solve is an input error.
 *   - vartype: concatenated likewise, or NULL.
 *   - claimed_obj: count doubles, or NULL (none).
 *   - out: count reports, in instance order. */
int nir_pdhg_batch_verify(nir_pdhg_batch* b, const double* x, const int8_t* vartype, const double* claimed_obj,
                          double tol, nir_verify_report* out);

/* --- no-allocation entry point --- */

/* A CSR matrix that already lives in device memory (all DEVICE pointers). */
typedef struct nir_csr_dev {
    int32_t rows, cols;
    const int32_t* row_ptr;   /* rows+1, row_ptr[0] = 0                        */
    const int32_t* col_idx;   /* row_ptr[rows] entries                          */
    const double* value;      /* row_ptr[rows] entries                          */
} nir_csr_dev;

/* The reference PDHG loop (the NIR_ALGO_REFERENCE kernels, bit for bit) on
 * an LP the caller already holds in device memory, without allocating any
 * device memory.  No counterpart in the reference: it exists for callers
 * that cannot call cudaMalloc -- processes whose device memory is owned by
 * their own pool allocator, and latency-critical callers that may not take
 * cudaMalloc's implicit device synchronisation.
 *   A, At          CSR of A (nrow x ncol) and of A' (ncol x nrow), each row's
 *                  entries in ascending column order (A' = the CSC of A)
 *   cost..rowup    device vectors (bounds as in nir_lp.h)
 *   stream         cudaStream_t to run on (NULL = the default stream)
 *   x_out, y_out   device outputs (ncol, nrow), also the loop's iterates
 *   iterations, status  host outputs (as nir_pdhg_solve with REFERENCE)
 * Scratch lives in one file-scope device array of 2^20 doubles (8 MiB) per
 * GPU, held until the process exits; the LP must satisfy
 * 32 + 2*ncol + nrow + ceil(nrow/256) <= 2^20, else NIR_STATUS_INPUT_ERROR.
 * The first call on a device resolves the array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture.  The address is kept for the life of the
 * process: after a cudaDeviceReset of that device it is stale, so do not
 * call this entry point on a device that was reset.  Every call waits for
 * its stream (it reads the stop test back every 32 iterations).  All calls
 * share the array and each call clears the state it needs: calls that
 * overlap on the GPU (other streams, other threads) race.  Returns *status. */
int nir_pdhg_reference_solve_noalloc(const nir_csr_dev* A, const nir_csr_dev* At, const double* cost,
                                     const double* collo, const double* colup, const double* rowlo,
                                     const double* rowup, int64_t max_iters, void* stream, double* x_out,
                                     double* y_out, int64_t* iterations, int32_t* status);

#ifdef __cplusplus
}
#endif
#endif
