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

#ifdef __cplusplus
}
#endif

#endif /* NIR_MLP_H */
