/*
 * nir_mlp.h -- C ABI of the warm-start network (libnir_mlp.so, sm_100a).
 *
 * A multilayer perceptron that maps the perturbation features of an LP of a
 * fixed-structure family (demand and cost factors) to an initial primal
 * iterate, dual iterate and primal weight for the PDLP engine
 * (nir_pdhg_params.x_init / y_init / omega_init in nir_pdhg.h).  The
 * reference has no learned component: this is new, and the PDLP engine
 * stays both the fallback and the arbiter (a warm start counts only when the
 * solve it seeds reaches the same relative-KKT tolerance).
 *
 * Layers: d_in -> width (ReLU) -> ... (depth hidden layers) -> d_out.
 * FP32 master weights; activations, weight copies and gradients with
 * respect to activations in BF16; every contraction accumulates in FP32 on
 * the tensor cores (hand-written kernels, mma.sync m16n8k16 BF16).
 * Training: mean-squared error over the outputs with weight 1 (outputs
 * with weight 0 are padding), Adam.
 *
 * Shapes: d_in, d_out and batch sizes must be multiples of 8 (callers pad
 * with zero features and zero-weight outputs).  Host arrays are row-major
 * float32, one sample per row.  Every call is synchronous on the handle's
 * own stream; a handle must not be used from two threads at once.
 * Errors return a nonzero code and set nir_mlp_last_error().
 */
#ifndef NIR_MLP_H
#define NIR_MLP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct nir_mlp_config {
    int32_t d_in;     /* input features (multiple of 8)                    */
    int32_t width;    /* hidden width (multiple of 8), e.g. 512            */
    int32_t depth;    /* hidden layers, >= 1, e.g. 3                       */
    int32_t d_out;    /* outputs (multiple of 8)                           */
    uint64_t seed;    /* weight initialisation and shuffling               */
    float lr;         /* Adam step size                                    */
    float beta1;      /* Adam moment decays                                */
    float beta2;
    float eps;
} nir_mlp_config;

typedef struct nir_mlp nir_mlp;

/* Allocates the network on `device` (weights initialised from cfg->seed,
 * zero biases).  Returns 0 or an error code. */
int nir_mlp_create(const nir_mlp_config* cfg, int device, nir_mlp** out);
void nir_mlp_free(nir_mlp* h);
const char* nir_mlp_last_error(void);

/* Number of parameters (weights and biases, all layers) and the flat
 * layout used by get/set/gradients: per layer l = 0..depth, W_l
 * (out_l x in_l, row-major) then b_l (out_l). */
int64_t nir_mlp_param_count(const nir_mlp* h);
int nir_mlp_get_params(nir_mlp* h, float* out);
int nir_mlp_set_params(nir_mlp* h, const float* in);

/* Per-output loss weights (d_out floats, 1 = real output, 0 = padding).
 * Default: all 1. */
int nir_mlp_set_output_weights(nir_mlp* h, const float* w);

/* Training set, copied to the device (x as BF16, targets as FP32). */
int nir_mlp_set_data(nir_mlp* h, const float* x, const float* targets, int32_t n);

/* `epochs` passes over the training set in minibatches of `batch`
 * (a multiple of 8; a last partial batch is dropped), sample order
 * shuffled per epoch from the seed.  epoch_loss (optional, `epochs`
 * floats) receives each epoch's mean minibatch loss. */
int nir_mlp_train(nir_mlp* h, int32_t epochs, int32_t batch, float* epoch_loss);

/* Forward pass of n samples (n a multiple of 8): y (n x d_out). */
int nir_mlp_predict(nir_mlp* h, const float* x, int32_t n, float* y);

/* The same forward pass from FP32 samples already on this handle's device
 * (x_dev: n x d_in, row-major, written before the call by work that has
 * finished, e.g. nir_blend_features_build); y on the host. */
int nir_mlp_predict_device(nir_mlp* h, const float* x_dev, int32_t n, float* y);

/* The output map of nir_mlp_predict_device_affine, for n samples:
 *   out[i] = shift[i] + scale[i] * min(max(pred[i][col], lo), hi)   (FP64)
 * scale and shift are host arrays of n doubles, copied to the device here
 * (NULL scale = 1, NULL shift = 0).  It turns a network's standardised
 * output into a starting point (a box-scaled x, or a de-standardised y)
 * without a trip through the host. */
int nir_mlp_set_affine(nir_mlp* h, int32_t n, int32_t col, double lo, double hi, const double* scale,
                       const double* shift);

/* The forward pass of nir_mlp_predict_device followed by the output map
 * set by nir_mlp_set_affine (for the same n): *out_dev receives the device
 * address of the n FP64 results, owned by the handle, valid until its next
 * call and complete when this returns (nir_pdhg_params.x_init / y_init
 * take it as is). */
int nir_mlp_predict_device_affine(nir_mlp* h, const float* x_dev, int32_t n, const double** out_dev);

/* Loss and gradients of one minibatch (n a multiple of 8, at most 4096)
 * without updating the weights: grads in the flat parameter layout. */
int nir_mlp_gradients(nir_mlp* h, const float* x, const float* targets, int32_t n, float* loss, float* grads);

/* The GEMM the layers use, for checking: C (M x N, row-major FP32) =
 * sum_k A(m, k) B(n, k) with A and B given as FP32 and rounded to BF16.
 * a_kmaj: A(m, k) = A[m * lda + k], else A[k * lda + m]; b_kmaj likewise
 * for B(n, k).  Contiguous extents and leading dimensions must be
 * multiples of 8. */
int nir_mlp_gemm_check(nir_mlp* h, int a_kmaj, int b_kmaj, int32_t M, int32_t N, int32_t K, const float* A,
                       int32_t lda, const float* B, int32_t ldb, float* C);

/* Mean device time (microseconds, CUDA events, after one warm-up) of the
 * forward-layer GEMM (bias + ReLU epilogue) on M x K and N x K BF16
 * operands, for throughput measurements: 2*M*N*K FLOP per call. */
int nir_mlp_gemm_time(nir_mlp* h, int32_t M, int32_t N, int32_t K, int32_t reps, double* us);

/* Event timing of the last nir_mlp_train: mean microseconds per minibatch
 * step (forward, loss, backward, Adam) and the tensor-core FLOPs of one
 * step (2 * batch * sum of in_l * out_l, forward plus both backward
 * products). */
int nir_mlp_step_stats(nir_mlp* h, double* us_per_step, double* flops_per_step);

/* --- the blending family's per-variable features on the device ---
 *
 * The inputs of the warm-start networks (nirnaya_b200/learned.py,
 * WarmStart.col_features / row_features) built on the GPU, so that a
 * prediction uploads only the instance's factors (nd + n doubles) instead
 * of 16 features per variable.  Instance (f, g): demand factors f (the first
 * nd rows' lower bounds are rowlo0 * f) and cost factors g (cost = cost0 * g).
 * Columns j (nf features each, the template's values elsewhere):
 *   F[j][0] = (g_j - 1) / 0.1
 *   F[j][1] = cost0_j g_j / cscale
 *   F[j][2] = (cost0_j g_j - atybar_j) / cscale
 *   F[j][6] = (sum_k D[j][k] (f_k - 1)) / max(dem_w_j, 1e-12) / 0.2,
 *             D the n x nd CSR of the columns' demand-row coefficients
 * Rows i:
 *   F[i][1] = (f_i - 1) / 0.2                                   (i < nd)
 *   F[i][4] = (axbar_i - lo_i) / bscale_i if lo_i is finite, else 0,
 *             lo_i = rowlo0_i f_i (i < nd) or rowlo0_i
 *   F[i][5] = (rowup_i - axbar_i) / bscale_i if rowup_i is finite, else 0
 *   F[i][6] = (sum_j |A|[i][j] (g_j - 1)) / max(row_abs_i, 1e-12) / 0.1,
 *             |A| the m x n CSR of the absolute values of A
 * Computed in FP64 and rounded to FP32, each sum in its CSR order.  No
 * counterpart in the reference (it has no learned component). */
typedef struct nir_blend_feature_data {
    int32_t n, m, nd, nf;          /* columns, rows, demand rows (the first nd), features (>= 7) */
    const float* col_template;     /* n x nf, row-major                                         */
    const float* row_template;     /* m x nf                                                    */
    const double* cost0;           /* per column                                                */
    const double* atybar;
    const double* dem_w;
    double cscale;
    const int64_t* dem_rp;         /* n + 1 */
    const int32_t* dem_ci;         /* demand-row index of each entry (< nd)                     */
    const double* dem_val;
    const double* rowlo0;          /* per row (+-inf where unbounded)                           */
    const double* rowup;
    const double* axbar;
    const double* bscale;
    const double* row_abs;
    const int64_t* abs_rp;         /* m + 1 */
    const int32_t* abs_ci;         /* column index of each entry (< n)                          */
    const double* abs_val;
} nir_blend_feature_data;

typedef struct nir_blend_features nir_blend_features;

/* Copies the family's data to `device`.  Returns 0 or an error code. */
int nir_blend_features_create(const nir_blend_feature_data* d, int32_t device, nir_blend_features** out);
/* Features of instance (f: nd, g: n) into device arrays the handle owns
 * (valid until its next call); synchronous. */
int nir_blend_features_build(nir_blend_features* h, const double* f, const double* g, const float** col_dev,
                             const float** row_dev);
void nir_blend_features_free(nir_blend_features* h);

#ifdef __cplusplus
}
#endif

#endif /* NIR_MLP_H */
