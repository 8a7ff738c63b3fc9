// Warm-start network: hand-written BF16 tensor-core GEMMs (mma.sync
// m16n8k16, FP32 accumulation), fused epilogues, Adam, all on one stream.
// C ABI: include/nir_mlp.h.
//
// GEMM.  C[M x N] = sum_k A(m, k) * B(n, k).  Each operand is stored either
// K-major (element (r, k) at P[r * ld + k]) or MN-major (at P[k * ld + r]);
// the three products of a dense layer use all three combinations:
//   forward   Y  = X * W^T      A = X  K-major,  B = W  K-major
//   input grad dX = dY * W      A = dY K-major,  B = W  MN-major
//   weight grad dW = dY^T * X   A = dY MN-major, B = X  MN-major
// A CTA (8 warps) computes a 128 x 128 tile in steps of 32 along K; tiles
// stream global -> shared with 16-byte cp.async (zero-filled outside the
// matrix) through a 3-stage pipeline; warps read fragments with ldmatrix
// (.trans for MN-major tiles) from XOR-swizzled rows (no bank conflicts)
// and issue 16 mma.sync per 16-wide K step on a 64 x 32 warp tile.
// Products with few output tiles and a long K split K over blockIdx.z into
// FP32 partials that a second kernel sums in a fixed order (deterministic)
// before the epilogue.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "nir_mlp.h"

namespace {

thread_local std::string g_err;

#define MLP_CUDA(call)                                                                              \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            throw std::runtime_error(std::string(#call) + ": " + cudaGetErrorString(e_));           \
    } while (0)
#define MLP_LAUNCHED() MLP_CUDA(cudaGetLastError())

using bf16 = __nv_bfloat16;

constexpr int BM = 128, BN = 128, BK = 32, STAGES = 3, THREADS = 256;
constexpr int TILE_BYTES = BM * BK * 2;                 // one operand tile, 8 KB
constexpr int SMEM_BYTES = STAGES * 2 * TILE_BYTES;     // 48 KB

enum Epi : int { EPI_BIAS_RELU_BF16 = 0, EPI_BIAS_F32 = 1, EPI_MASK_BF16 = 2, EPI_F32 = 3 };

struct GemmArgs {
    const bf16* A;
    int lda;
    const bf16* B;
    int ldb;
    int M, N, K;
    int kps;           // K range per split (multiple of BK)
    int splits;        // gridDim.z; > 1: partials to ws
    int epi;
    const float* bias;
    bf16* out_bf;
    float* out_f;
    int ldc;
    const bf16* mask;  // EPI_MASK_BF16: multiply by (mask > 0)
    int ldm;
    float* ws;         // splits x M x N partials
};

// Byte offset of 16-byte chunk c of row r in a swizzled tile.
__device__ __forceinline__ int kmaj_off(int r, int c) { return r * 64 + ((c ^ ((r >> 1) & 3)) << 4); }   // 128 x 32
__device__ __forceinline__ int mnmaj_off(int r, int c) { return r * 256 + ((c ^ (r & 7)) << 4); }       // 32 x 128

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, bool valid) {
    const int n = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(n));
}

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t (&r)[4]) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(addr));
}

__device__ __forceinline__ void ldsm_x4_t(uint32_t addr, uint32_t (&r)[4]) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(addr));
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// One operand tile (rows r0.., K range k0..k0+BK) into shared memory.
// K-major: 128 rows x 4 chunks; MN-major: 32 K-rows x 16 chunks.
template <bool KMAJ>
__device__ __forceinline__ void load_tile(uint32_t sbase, const bf16* __restrict__ P, int ld, int rows, int r0,
                                          int k0, int kend) {
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const int idx = threadIdx.x + i * THREADS;
        if (KMAJ) {
            const int r = idx >> 2, c = idx & 3;
            const int gr = r0 + r, gk = k0 + c * 8;
            const bool ok = gr < rows && gk < kend;
            cp_async16(sbase + kmaj_off(r, c), ok ? (const void*)(P + (size_t)gr * ld + gk) : (const void*)P, ok);
        } else {
            const int r = idx >> 4, c = idx & 15;
            const int gk = k0 + r, gr = r0 + c * 8;
            const bool ok = gk < kend && gr < rows;
            cp_async16(sbase + mnmaj_off(r, c), ok ? (const void*)(P + (size_t)gk * ld + gr) : (const void*)P, ok);
        }
    }
}

template <bool AK, bool BKM>
__global__ void __launch_bounds__(THREADS) k_gemm(GemmArgs g) {
    extern __shared__ __align__(128) unsigned char smem[];
    const uint32_t sb = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp >> 2, wn = warp & 3;  // 2 x 4 warps, 64 x 32 each
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int kbeg = blockIdx.z * g.kps;
    const int kend = min(g.K, kbeg + g.kps);
    const int KT = (kend > kbeg) ? (kend - kbeg + BK - 1) / BK : 0;

    float acc[4][4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;

    auto stageA = [&](int s) { return sb + s * 2 * TILE_BYTES; };
    auto stageB = [&](int s) { return sb + s * 2 * TILE_BYTES + TILE_BYTES; };

#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
        if (s < KT) {
            load_tile<AK>(stageA(s), g.A, g.lda, g.M, m0, kbeg + s * BK, kend);
            load_tile<BKM>(stageB(s), g.B, g.ldb, g.N, n0, kbeg + s * BK, kend);
        }
        asm volatile("cp.async.commit_group;\n" ::);
    }

    for (int kt = 0; kt < KT; ++kt) {
        asm volatile("cp.async.wait_group %0;\n" ::"n"(STAGES - 2));
        __syncthreads();
        const int nk = kt + STAGES - 1;
        if (nk < KT) {
            load_tile<AK>(stageA(nk % STAGES), g.A, g.lda, g.M, m0, kbeg + nk * BK, kend);
            load_tile<BKM>(stageB(nk % STAGES), g.B, g.ldb, g.N, n0, kbeg + nk * BK, kend);
        }
        asm volatile("cp.async.commit_group;\n" ::);
        const uint32_t sa = stageA(kt % STAGES), sbb = stageB(kt % STAGES);
#pragma unroll
        for (int kk = 0; kk < BK; kk += 16) {
            uint32_t af[4][4];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi) {
                const int mb = wm * 64 + mi * 16;
                if (AK) {
                    const int r = mb + (lane & 15), c = (kk >> 3) + (lane >> 4);
                    ldsm_x4(sa + kmaj_off(r, c), af[mi]);
                } else {
                    const int j = lane >> 3;
                    const int r = kk + (j >> 1) * 8 + (lane & 7), c = (mb + (j & 1) * 8) >> 3;
                    ldsm_x4_t(sa + mnmaj_off(r, c), af[mi]);
                }
            }
            uint32_t bfr[2][4];
#pragma unroll
            for (int np = 0; np < 2; ++np) {
                const int nb = wn * 32 + np * 16;
                const int j = lane >> 3;
                if (BKM) {
                    const int r = nb + (j >> 1) * 8 + (lane & 7), c = (kk >> 3) + (j & 1);
                    ldsm_x4(sbb + kmaj_off(r, c), bfr[np]);
                } else {
                    const int r = kk + (j & 1) * 8 + (lane & 7), c = (nb + (j >> 1) * 8) >> 3;
                    ldsm_x4_t(sbb + mnmaj_off(r, c), bfr[np]);
                }
            }
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni)
                    mma_bf16(acc[mi][ni], af[mi], bfr[ni >> 1][(ni & 1) * 2], bfr[ni >> 1][(ni & 1) * 2 + 1]);
        }
    }
    asm volatile("cp.async.wait_group 0;\n" ::);

    const int gq = lane >> 2, tq = lane & 3;
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int row = m0 + wm * 64 + mi * 16 + gq + (e >> 1) * 8;
                const int col = n0 + wn * 32 + ni * 8 + tq * 2 + (e & 1);
                if (row >= g.M || col >= g.N) continue;
                const float v = acc[mi][ni][e];
                if (g.splits > 1) {
                    g.ws[((size_t)blockIdx.z * g.M + row) * g.N + col] = v;
                    continue;
                }
                const size_t o = (size_t)row * g.ldc + col;
                switch (g.epi) {
                    case EPI_BIAS_RELU_BF16: g.out_bf[o] = __float2bfloat16_rn(fmaxf(v + g.bias[col], 0.f)); break;
                    case EPI_BIAS_F32: g.out_f[o] = v + g.bias[col]; break;
                    case EPI_MASK_BF16:
                        g.out_bf[o] = __float2bfloat16_rn(__bfloat162float(g.mask[(size_t)row * g.ldm + col]) > 0.f ? v : 0.f);
                        break;
                    default: g.out_f[o] = v; break;
                }
            }
}

// Sums the split-K partials in split order and applies the epilogue.
__global__ void k_splitk_reduce(GemmArgs g) {
    const size_t total = (size_t)g.M * g.N;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        float v = 0.f;
        for (int z = 0; z < g.splits; ++z) v += g.ws[(size_t)z * total + i];
        const int row = int(i / g.N), col = int(i % g.N);
        const size_t o = (size_t)row * g.ldc + col;
        switch (g.epi) {
            case EPI_BIAS_RELU_BF16: g.out_bf[o] = __float2bfloat16_rn(fmaxf(v + g.bias[col], 0.f)); break;
            case EPI_BIAS_F32: g.out_f[o] = v + g.bias[col]; break;
            case EPI_MASK_BF16:
                g.out_bf[o] = __float2bfloat16_rn(__bfloat162float(g.mask[(size_t)row * g.ldm + col]) > 0.f ? v : 0.f);
                break;
            default: g.out_f[o] = v; break;
        }
    }
}

// ------------------------------------------------------------ elementwise

__global__ void k_to_bf16(size_t n, const float* __restrict__ a, bf16* __restrict__ b) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        b[i] = __float2bfloat16_rn(a[i]);
}

// out[i] = shift[i] + scale[i] * clamp(pred[i * ld + col], lo, hi), FP64
// (r0 = the first sample of this chunk; pred holds the chunk's rows).  The
// product and the sum are rounded separately (no fused multiply-add), the
// clamp passes a NaN through, and a missing scale or shift is no operation,
// so the result is the host's numpy expression bit for bit.
__global__ void k_affine_out(int rows, int r0, const float* __restrict__ pred, int ld, int col, double lo, double hi,
                             const double* __restrict__ scale, const double* __restrict__ shift,
                             double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows) return;
    const int g = r0 + i;
    double p = double(pred[(size_t)i * ld + col]);
    p = (p < lo) ? lo : ((p > hi) ? hi : p);
    const double v = scale ? __dmul_rn(scale[g], p) : p;
    out[g] = shift ? __dadd_rn(shift[g], v) : v;
}

template <typename T>
__global__ void k_gather_rows(const int* __restrict__ idx, int rows, int cols, const T* __restrict__ src,
                              T* __restrict__ dst) {
    const size_t total = (size_t)rows * cols;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int r = int(i / cols), c = int(i % cols);
        dst[i] = src[(size_t)idx[r] * cols + c];
    }
}

__device__ __forceinline__ float block_sum_f(float v, float* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = v;
    __syncthreads();
    float t = 0.f;
    if (threadIdx.x == 0)
        for (int i = 0; i < int(blockDim.x >> 5); ++i) t += sh[i];
    __syncthreads();
    return t;
}

// dY = scale * w * (pred - target) (BF16) and per-block sums of w*(pred-target)^2.
__global__ void k_loss(int rows, int cols, const float* __restrict__ pred, const float* __restrict__ tgt,
                       const float* __restrict__ w, float scale, bf16* __restrict__ dy, float* __restrict__ part) {
    __shared__ float sh[32];
    const size_t total = (size_t)rows * cols;
    float s = 0.f;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const float wc = w[i % cols];
        const float d = pred[i] - tgt[i];
        s += wc * d * d;
        dy[i] = __float2bfloat16_rn(scale * (wc * d));
    }
    s = block_sum_f(s, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void k_sum_partials(int n, const float* __restrict__ part, float mul, float* __restrict__ out, int slot) {
    __shared__ float sh[32];
    float s = 0.f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += part[i];
    s = block_sum_f(s, sh);
    if (threadIdx.x == 0) out[slot] = s * mul;
}

// db[c] = sum over rows of dY[r][c] in two deterministic passes: chunk z
// of kColChunkRows rows -> part[z][c] (rows in order), then the chunks in
// order.
constexpr int kColChunkRows = 128;

__global__ void k_colsum_part(int rows, int cols, const bf16* __restrict__ dy, float* __restrict__ part) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    const int r0 = blockIdx.y * kColChunkRows, r1 = min(rows, r0 + kColChunkRows);
    float s = 0.f;
    for (int r = r0; r < r1; ++r) s += __bfloat162float(dy[(size_t)r * cols + c]);
    part[(size_t)blockIdx.y * cols + c] = s;
}

__global__ void k_colsum_final(int chunks, int cols, const float* __restrict__ part, float* __restrict__ db) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float s = 0.f;
    for (int z = 0; z < chunks; ++z) s += part[(size_t)z * cols + c];
    db[c] = s;
}

__global__ void k_adam(size_t n, float* __restrict__ w, bf16* __restrict__ wb, const float* __restrict__ g,
                       float* __restrict__ m, float* __restrict__ v, float lr, float b1, float b2, float eps, float bc1,
                       float bc2) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
        w[i] = wi;
        if (wb) wb[i] = __float2bfloat16_rn(wi);
    }
}

// Uniform(-a, a) from a counter hash (splitmix64) of (seed, index).
__global__ void k_init_uniform(size_t n, uint64_t seed, float a, float* __restrict__ w, bf16* __restrict__ wb) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        uint64_t z = seed + 0x9e3779b97f4a7c15ULL * (i + 1);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        z ^= z >> 31;
        const float u = float(z >> 40) * (1.0f / 16777216.0f);  // [0, 1)
        const float x = (2.f * u - 1.f) * a;
        w[i] = x;
        if (wb) wb[i] = __float2bfloat16_rn(x);
    }
}

unsigned grid1d(size_t n, int cap = 148 * 16) {
    size_t b = (n + 255) / 256;
    return unsigned(std::max<size_t>(1, std::min<size_t>(b, cap)));
}

}  // namespace

// ------------------------------------------------------------ the handle

struct nir_mlp {
    nir_mlp_config cfg{};
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;
    std::vector<int> dims;  // d_in, width x depth, d_out
    struct Layer {
        int in = 0, out = 0;
        float *W = nullptr, *b = nullptr, *gW = nullptr, *gb = nullptr;
        float *mW = nullptr, *vW = nullptr, *mb = nullptr, *vb = nullptr;
        bf16* Wb = nullptr;
    };
    std::vector<Layer> layers;
    float* outw = nullptr;  // per-output loss weights
    float outw_sum = 0.f;
    // activations for up to cap_rows samples
    int cap_rows = 0;
    bf16* x = nullptr;
    std::vector<bf16*> act;  // hidden outputs
    float* pred = nullptr;
    float* tgt = nullptr;
    bf16* dy = nullptr;
    bf16 *g0 = nullptr, *g1 = nullptr;  // hidden-size gradient ping-pong
    float* ws = nullptr;
    size_t ws_len = 0;
    float* colsum_ws = nullptr;
    size_t colsum_len = 0;
    float* part = nullptr;
    float* losses = nullptr;  // device loss per step
    int losses_len = 0;
    // training set
    int n_data = 0;
    bf16* data_x = nullptr;
    float* data_y = nullptr;
    int* perm = nullptr;
    int64_t adam_t = 0;
    double us_per_step = 0.0, flops_per_step = 0.0;
    float* stage = nullptr;  // FP32 staging of uploaded rows, grown on demand
    size_t stage_len = 0;
    // output map of nir_mlp_predict_device_affine
    int aff_n = 0, aff_col = 0;
    double aff_lo = 0.0, aff_hi = 0.0;
    double *aff_scale = nullptr, *aff_shift = nullptr, *aff_out = nullptr;
    std::vector<void*> allocs;

    template <typename T>
    T* alloc(size_t n) {
        void* p = nullptr;
        MLP_CUDA(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
        MLP_CUDA(cudaMemsetAsync(p, 0, std::max<size_t>(n, 1) * sizeof(T), stream));
        allocs.push_back(p);
        return static_cast<T*>(p);
    }
    void release(void* p) {
        for (auto& q : allocs)
            if (q == p) {
                cudaFree(q);
                q = nullptr;
            }
    }
    ~nir_mlp() {
        cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        for (void* p : allocs)
            if (p) cudaFree(p);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

void check_mult8(int v, const char* what) {
    if (v <= 0 || v % 8 != 0) throw std::invalid_argument(std::string(what) + " must be a positive multiple of 8");
}

// C = op(A) op(B)^T with the given storage (see the file header).
void gemm(nir_mlp* h, bool a_kmaj, bool b_kmaj, const bf16* A, int lda, const bf16* B, int ldb, int M, int N, int K,
          int epi, const float* bias, bf16* out_bf, float* out_f, int ldc, const bf16* mask, int ldm) {
    if (M <= 0 || N <= 0) return;
    if (K % 8 != 0 || (!a_kmaj && M % 8 != 0) || (!b_kmaj && N % 8 != 0) || lda % 8 != 0 || ldb % 8 != 0)
        throw std::invalid_argument("gemm: contiguous extents must be multiples of 8");
    GemmArgs g{};
    g.A = A;
    g.lda = lda;
    g.B = B;
    g.ldb = ldb;
    g.M = M;
    g.N = N;
    g.K = K;
    g.epi = epi;
    g.bias = bias;
    g.out_bf = out_bf;
    g.out_f = out_f;
    g.ldc = ldc;
    g.mask = mask;
    g.ldm = ldm;
    const int tm = (M + BM - 1) / BM, tn = (N + BN - 1) / BN;
    const int KT = (K + BK - 1) / BK;
    int splits = 1;
    const int want = 2 * h->sms;
    if (tm * tn < want && KT >= 16) splits = std::min(KT / 8, (want + tm * tn - 1) / (tm * tn));
    splits = std::max(splits, 1);
    g.kps = ((KT + splits - 1) / splits) * BK;
    splits = (K + g.kps - 1) / g.kps;
    g.splits = splits;
    if (splits > 1) {
        const size_t need = (size_t)splits * M * N;
        if (need > h->ws_len) {
            h->release(h->ws);
            h->ws = h->alloc<float>(need);
            h->ws_len = need;
        }
        g.ws = h->ws;
    }
    dim3 grid(tn, tm, splits);
    auto launch = [&](auto kern) {
        MLP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
        kern<<<grid, THREADS, SMEM_BYTES, h->stream>>>(g);
    };
    if (a_kmaj && b_kmaj) launch(k_gemm<true, true>);
    else if (a_kmaj && !b_kmaj) launch(k_gemm<true, false>);
    else if (!a_kmaj && !b_kmaj) launch(k_gemm<false, false>);
    else launch(k_gemm<false, true>);
    MLP_LAUNCHED();
    if (splits > 1) {
        k_splitk_reduce<<<grid1d((size_t)M * N), 256, 0, h->stream>>>(g);
        MLP_LAUNCHED();
    }
}

void ensure_rows(nir_mlp* h, int rows) {
    if (rows <= h->cap_rows) return;
    for (bf16* p : h->act) h->release(p);
    for (void* p : {(void*)h->x, (void*)h->pred, (void*)h->tgt, (void*)h->dy, (void*)h->g0, (void*)h->g1})
        if (p) h->release(p);
    const int din = h->cfg.d_in, dout = h->cfg.d_out, wmax = h->cfg.width;
    h->x = h->alloc<bf16>((size_t)rows * din);
    h->act.assign(h->cfg.depth, nullptr);
    for (auto& a : h->act) a = h->alloc<bf16>((size_t)rows * h->cfg.width);
    h->pred = h->alloc<float>((size_t)rows * dout);
    h->tgt = h->alloc<float>((size_t)rows * dout);
    h->dy = h->alloc<bf16>((size_t)rows * dout);
    h->g0 = h->alloc<bf16>((size_t)rows * wmax);
    h->g1 = h->alloc<bf16>((size_t)rows * wmax);
    h->cap_rows = rows;
}

void forward(nir_mlp* h, int rows) {
    const bf16* in = h->x;
    const int L = int(h->layers.size());
    for (int l = 0; l < L; ++l) {
        auto& ly = h->layers[l];
        if (l + 1 < L) {
            gemm(h, true, true, in, ly.in, ly.Wb, ly.in, rows, ly.out, ly.in, EPI_BIAS_RELU_BF16, ly.b, h->act[l],
                 nullptr, ly.out, nullptr, 0);
            in = h->act[l];
        } else {
            gemm(h, true, true, in, ly.in, ly.Wb, ly.in, rows, ly.out, ly.in, EPI_BIAS_F32, ly.b, nullptr, h->pred,
                 ly.out, nullptr, 0);
        }
    }
}

// Loss (device slot) and dY, then every layer's gradients.
void backward(nir_mlp* h, int rows, int loss_slot) {
    const int dout = h->cfg.d_out;
    const float denom = float(rows) * std::max(h->outw_sum, 1.f);
    const unsigned gb = grid1d((size_t)rows * dout, 1024);
    k_loss<<<gb, 256, 0, h->stream>>>(rows, dout, h->pred, h->tgt, h->outw, 2.f / denom, h->dy, h->part);
    k_sum_partials<<<1, 256, 0, h->stream>>>(int(gb), h->part, 1.f / denom, h->losses, loss_slot);
    MLP_LAUNCHED();
    const int L = int(h->layers.size());
    const bf16* g = h->dy;
    for (int l = L - 1; l >= 0; --l) {
        auto& ly = h->layers[l];
        const bf16* in = (l == 0) ? h->x : h->act[l - 1];
        // dW = g^T in   (out x in), contraction over the rows
        gemm(h, false, false, g, ly.out, in, ly.in, ly.out, ly.in, rows, EPI_F32, nullptr, nullptr, ly.gW, ly.in,
             nullptr, 0);
        {
            const int chunks = (rows + kColChunkRows - 1) / kColChunkRows;
            const size_t need = (size_t)chunks * ly.out;
            if (need > h->colsum_len) {
                h->release(h->colsum_ws);
                h->colsum_ws = h->alloc<float>(need);
                h->colsum_len = need;
            }
            k_colsum_part<<<dim3((ly.out + 255) / 256, chunks), 256, 0, h->stream>>>(rows, ly.out, g, h->colsum_ws);
            k_colsum_final<<<(ly.out + 255) / 256, 256, 0, h->stream>>>(chunks, ly.out, h->colsum_ws, ly.gb);
            MLP_LAUNCHED();
        }
        if (l > 0) {
            bf16* gn = (g == h->g0) ? h->g1 : h->g0;
            // d(in) = g W, masked by the ReLU of the layer below
            gemm(h, true, false, g, ly.out, ly.Wb, ly.in, rows, ly.in, ly.out, EPI_MASK_BF16, nullptr, gn, nullptr,
                 ly.in, h->act[l - 1], ly.in);
            g = gn;
        }
    }
}

void adam(nir_mlp* h) {
    h->adam_t += 1;
    const float b1 = h->cfg.beta1, b2 = h->cfg.beta2;
    const float bc1 = 1.f - std::pow(b1, float(h->adam_t)), bc2 = 1.f - std::pow(b2, float(h->adam_t));
    for (auto& ly : h->layers) {
        const size_t nw = (size_t)ly.in * ly.out;
        k_adam<<<grid1d(nw), 256, 0, h->stream>>>(nw, ly.W, ly.Wb, ly.gW, ly.mW, ly.vW, h->cfg.lr, b1, b2, h->cfg.eps,
                                                   bc1, bc2);
        k_adam<<<grid1d(ly.out), 256, 0, h->stream>>>(ly.out, ly.b, nullptr, ly.gb, ly.mb, ly.vb, h->cfg.lr, b1, b2,
                                                       h->cfg.eps, bc1, bc2);
    }
    MLP_LAUNCHED();
}

void ensure_losses(nir_mlp* h, int n) {
    if (n <= h->losses_len) return;
    h->release(h->losses);
    h->losses = h->alloc<float>(n);
    h->losses_len = n;
}

// Host FP32 rows -> device BF16, through a staging buffer that grows on
// demand and is kept (no allocation per call once it is large enough).
void upload_rows(nir_mlp* h, const float* x, int rows, bf16* dst, int cols) {
    const size_t len = (size_t)rows * cols;
    if (len > h->stage_len) {
        if (h->stage) h->release(h->stage);
        h->stage = h->alloc<float>(len);
        h->stage_len = len;
    }
    MLP_CUDA(cudaMemcpyAsync(h->stage, x, len * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    k_to_bf16<<<grid1d(len), 256, 0, h->stream>>>(len, h->stage, dst);
    MLP_LAUNCHED();
    MLP_CUDA(cudaStreamSynchronize(h->stream));
}

int fail(const std::exception& e, bool input) {
    g_err = e.what();
    return input ? 2 : 3;
}

}  // namespace

extern "C" {

const char* nir_mlp_last_error(void) { return g_err.c_str(); }

int nir_mlp_create(const nir_mlp_config* cfg, int device, nir_mlp** out) {
    if (!cfg || !out) {
        g_err = "null argument";
        return 2;
    }
    *out = nullptr;
    auto h = std::make_unique<nir_mlp>();
    try {
        check_mult8(cfg->d_in, "d_in");
        check_mult8(cfg->width, "width");
        check_mult8(cfg->d_out, "d_out");
        if (cfg->depth < 1 || cfg->depth > 16) throw std::invalid_argument("depth must be in [1, 16]");
        h->cfg = *cfg;
        h->device = device;
        MLP_CUDA(cudaSetDevice(device));
        MLP_CUDA(cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, device));
        MLP_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        h->dims.push_back(cfg->d_in);
        for (int i = 0; i < cfg->depth; ++i) h->dims.push_back(cfg->width);
        h->dims.push_back(cfg->d_out);
        for (size_t l = 0; l + 1 < h->dims.size(); ++l) {
            nir_mlp::Layer ly;
            ly.in = h->dims[l];
            ly.out = h->dims[l + 1];
            const size_t nw = (size_t)ly.in * ly.out;
            ly.W = h->alloc<float>(nw);
            ly.Wb = h->alloc<bf16>(nw);
            ly.gW = h->alloc<float>(nw);
            ly.mW = h->alloc<float>(nw);
            ly.vW = h->alloc<float>(nw);
            ly.b = h->alloc<float>(ly.out);
            ly.gb = h->alloc<float>(ly.out);
            ly.mb = h->alloc<float>(ly.out);
            ly.vb = h->alloc<float>(ly.out);
            // He-uniform for ReLU layers, smaller for the linear output
            const bool last = (l + 2 == h->dims.size());
            const float a = (last ? 0.5f : 1.f) * std::sqrt(6.f / float(ly.in));
            k_init_uniform<<<grid1d(nw), 256, 0, h->stream>>>(nw, cfg->seed * 1315423911ULL + l, a, ly.W, ly.Wb);
            MLP_LAUNCHED();
            h->layers.push_back(ly);
        }
        h->outw = h->alloc<float>(cfg->d_out);
        std::vector<float> ones(cfg->d_out, 1.f);
        MLP_CUDA(cudaMemcpyAsync(h->outw, ones.data(), ones.size() * sizeof(float), cudaMemcpyHostToDevice, h->stream));
        h->outw_sum = float(cfg->d_out);
        h->part = h->alloc<float>(1024);
        ensure_losses(h.get(), 1024);
        MLP_CUDA(cudaStreamSynchronize(h->stream));
    } catch (const std::invalid_argument& e) {
        return fail(e, true);
    } catch (const std::exception& e) {
        return fail(e, false);
    }
    *out = h.release();
    return 0;
}

void nir_mlp_free(nir_mlp* h) { delete h; }

int64_t nir_mlp_param_count(const nir_mlp* h) {
    if (!h) return -1;
    int64_t n = 0;
    for (auto& ly : h->layers) n += (int64_t)ly.in * ly.out + ly.out;
    return n;
}

int nir_mlp_get_params(nir_mlp* h, float* out) {
    if (!h || !out) return 2;
    try {
        MLP_CUDA(cudaSetDevice(h->device));
        size_t o = 0;
        for (auto& ly : h->layers) {
            const size_t nw = (size_t)ly.in * ly.out;
            MLP_CUDA(cudaMemcpyAsync(out + o, ly.W, nw * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
            o += nw;
            MLP_CUDA(cudaMemcpyAsync(out + o, ly.b, ly.out * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
            o += ly.out;
        }
        MLP_CUDA(cudaStreamSynchronize(h->stream));
    } catch (const std::exception& e) {
        return fail(e, false);
    }
    return 0;
}

int nir_mlp_set_params(nir_mlp* h, const float* in) {
    if (!h || !in) return 2;
    try {
        MLP_CUDA(cudaSetDevice(h->device));
        size_t o = 0;
        for (auto& ly : h->layers) {
            const size_t nw = (size_t)ly.in * ly.out;
            MLP_CUDA(cudaMemcpyAsync(ly.W, in + o, nw * sizeof(float), cudaMemcpyHostToDevice, h->stream));
            k_to_bf16<<<grid1d(nw), 256, 0, h->stream>>>(nw, ly.W, ly.Wb);
            MLP_LAUNCHED();
            o += nw;
            MLP_CUDA(cudaMemcpyAsync(ly.b, in + o, ly.out * sizeof(float), cudaMemcpyHostToDevice, h->stream));
            o += ly.out;
            MLP_CUDA(cudaMemsetAsync(ly.mW, 0, nw * sizeof(float), h->stream));
            MLP_CUDA(cudaMemsetAsync(ly.vW, 0, nw * sizeof(float), h->stream));
            MLP_CUDA(cudaMemsetAsync(ly.mb, 0, ly.out * sizeof(float), h->stream));
            MLP_CUDA(cudaMemsetAsync(ly.vb, 0, ly.out * sizeof(float), h->stream));
        }
        h->adam_t = 0;
        MLP_CUDA(cudaStreamSynchronize(h->stream));
    } catch (const std::exception& e) {
        return fail(e, false);
    }
    return 0;
}

int nir_mlp_set_output_weights(nir_mlp* h, const float* w) {
    if (!h || !w) return 2;
    try {
        MLP_CUDA(cudaSetDevice(h->device));
        double s = 0.0;
        for (int i = 0; i < h->cfg.d_out; ++i) {
            if (!(w[i] >= 0.f)) throw std::invalid_argument("output weights must be >= 0");
            s += w[i];
        }
        MLP_CUDA(cudaMemcpyAsync(h->outw, w, h->cfg.d_out * sizeof(float), cudaMemcpyHostToDevice, h->stream));
        MLP_CUDA(cudaStreamSynchronize(h->stream));
        h->outw_sum = float(s);
    } catch (const std::invalid_argument& e) {
        return fail(e, true);
    } catch (const std::exception& e) {
        return fail(e, false);
    }
    return 0;
}

int nir_mlp_set_data(nir_mlp* h, const float* x, const float* targets, int32_t n) {
    if (!h || !x || !targets || n < 1) {
        g_err = "invalid arguments";
        return 2;
    }
    try {
        MLP_CUDA(cudaSetDevice(h->device));
        h->release(h->data_x);
        h->release(h->data_y);
        h->release(h->perm);
        const int din = h->cfg.d_in, dout = h->cfg.d_out;
        h->data_x = h->alloc<bf16>((size_t)n * din);
        h->data_y = h->alloc<float>((size_t)n * dout);
        h->perm = h->alloc<int>(n);
        // in slices so that the FP32 staging buffer stays small
        const int slice = std::max(1, int((size_t(256) << 20) / (sizeof(float) * din)));
        for (int r = 0; r < n; r += slice) {
            const int k = std::min(slice, n - r);
            upload_rows(h, x + (size_t)r * din, k, h->data_x + (size_t)r * din, din);
        }
        MLP_CUDA(cudaMemcpyAsync(h->data_y, targets, (size_t)n * dout * sizeof(float), cudaMemcpyHostToDevice,
                                 h->stream));
        MLP_CUDA(cudaStreamSynchronize(h->stream));
        h->n_data = n;
    } catch (const std::exception& e) {
        return fail(e, false);
    }
    return 0;
}

int nir_mlp_train(nir_mlp* h, int32_t epochs, int32_t batch, float* epoch_loss) {
    if (!h || epochs < 0 || batch < 8 || batch % 8 != 0) {
        g_err = "invalid arguments (batch must be a positive multiple of 8)";
        return 2;
    }
    if (h->n_data < batch) {
        g_err = "training set smaller than one batch";
        return 2;
    }
    try {
        MLP_CUDA(cudaSetDevice(h->device));
        ensure_rows(h, batch);
        const int steps = h->n_data / batch;
        ensure_losses(h, steps);
        std::mt19937_64 rng(h->cfg.seed ^ 0x5bd1e995ULL ^ (uint64_t)h->adam_t);
        std::vector<int> perm(h->n_data);
        std::vector<float> lossv(steps);
        cudaEvent_t e0, e1;
        MLP_CUDA(cudaEventCreate(&e0));
        MLP_CUDA(cudaEventCreate(&e1));
        double total_ms = 0.0;
        long long total_steps = 0;
        for (int ep = 0; ep < epochs; ++ep) {
            for (int i = 0; i < h->n_data; ++i) perm[i] = i;
            std::shuffle(perm.begin(), perm.end(), rng);
            MLP_CUDA(cudaMemcpyAsync(h->perm, perm.data(), perm.size() * sizeof(int), cudaMemcpyHostToDevice,
                                     h->stream));
            MLP_CUDA(cudaEventRecord(e0, h->stream));
            for (int s = 0; s < steps; ++s) {
                const int* idx = h->perm + (size_t)s * batch;
                k_gather_rows<bf16><<<grid1d((size_t)batch * h->cfg.d_in), 256, 0, h->stream>>>(
                    idx, batch, h->cfg.d_in, h->data_x, h->x);
                k_gather_rows<float><<<grid1d((size_t)batch * h->cfg.d_out), 256, 0, h->stream>>>(
                    idx, batch, h->cfg.d_out, h->data_y, h->tgt);
                MLP_LAUNCHED();
                forward(h, batch);
                backward(h, batch, s);
                adam(h);
            }
            MLP_CUDA(cudaEventRecord(e1, h->stream));
            MLP_CUDA(cudaMemcpyAsync(lossv.data(), h->losses, steps * sizeof(float), cudaMemcpyDeviceToHost,
                                     h->stream));
            MLP_CUDA(cudaStreamSynchronize(h->stream));
            float ms = 0.f;
            MLP_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            total_ms += ms;
            total_steps += steps;
            if (epoch_loss) {
                double m = 0.0;
                for (float v : lossv) m += v;
                epoch_loss[ep] = float(m / steps);
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (total_steps > 0) h->us_per_step = 1000.0 * total_ms / double(total_steps);
        double f = 0.0;
        for (auto& ly : h->layers) f += 2.0 * double(batch) * ly.in * ly.out;
        // forward, weight gradient, input gradient (none for the first layer)
        h->flops_per_step = 3.0 * f - 2.0 * double(batch) * h->layers[0].in * h->layers[0].out;
    } catch (const std::exception& e) {
        return fail(e, false);
    }
    return 0;
}

int nir_mlp_predict(nir_mlp* h, const float* x, int32_t n, float* y) {
    if (!h || !x || !y || n < 8 || n % 8 != 0) {
        g_err = "invalid arguments (n must be a positive multiple of 8)";
        return 2;
    }
    try {
        MLP_CUDA(cudaSetDevice(h->device));
        // one chunk for a whole family member's variables (70,000 at the
        // 20,000 x 50,000 blending size): fewer uploads and synchronisations
        const int chunk = std::min(n, 65536);
        ensure_rows(h, chunk);
        for (int r = 0; r < n; r += chunk) {
            const int k = std::min(chunk, n - r);  // a multiple of 8
            upload_rows(h, x + (size_t)r * h->cfg.d_in, k, h->x, h->cfg.d_in);
            forward(h, k);
            MLP_CUDA(cudaMemcpyAsync(y + (size_t)r * h->cfg.d_out, h->pred, (size_t)k * h->cfg.d_out * sizeof(float),
                                     cudaMemcpyDeviceToHost, h->stream));
            MLP_CUDA(cudaStreamSynchronize(h->stream));
        }
    } catch (const std::exception& e) {
        return fail(e, false);
    }
    return 0;
}

int nir_mlp_predict_device(nir_mlp* h, const float* x_dev, int32_t n, float* y) {
    if (!h || !x_dev || !y || n < 8 || n % 8 != 0) {
        g_err = "invalid arguments (n must be a positive multiple of 8)";
        return 2;
    }
    try {
        MLP_CUDA(cudaSetDevice(h->device));
        const int chunk = std::min(n, 65536);
        ensure_rows(h, chunk);
        for (int r = 0; r < n; r += chunk) {
            const int k = std::min(chunk, n - r);
            const size_t len = (size_t)k * h->cfg.d_in;
            k_to_bf16<<<grid1d(len), 256, 0, h->stream>>>(len, x_dev + (size_t)r * h->cfg.d_in, h->x);
            MLP_LAUNCHED();
            forward(h, k);
            MLP_CUDA(cudaMemcpyAsync(y + (size_t)r * h->cfg.d_out, h->pred, (size_t)k * h->cfg.d_out * sizeof(float),
                                     cudaMemcpyDeviceToHost, h->stream));
            MLP_CUDA(cudaStreamSynchronize(h->stream));
        }
    } catch (const std::exception& e) {
        return fail(e, false);
    }
    return 0;
}

int nir_mlp_set_affine(nir_mlp* h, int32_t n, int32_t col, double lo, double hi, const double* scale,
                       const double* shift) {
    if (!h || n < 8 || n % 8 != 0 || col < 0 || col >= h->cfg.d_out || !(lo <= hi)) {
        g_err = "invalid arguments (n a positive multiple of 8, 0 <= col < d_out, lo <= hi)";
        return 2;
    }
    try {
        MLP_CUDA(cudaSetDevice(h->device));
        for (double** q : {&h->aff_scale, &h->aff_shift, &h->aff_out}) {
            if (*q) h->release(*q);
            *q = nullptr;
        }
        h->aff_out = h->alloc<double>(size_t(n));
        if (scale) {
            h->aff_scale = h->alloc<double>(size_t(n));
            MLP_CUDA(cudaMemcpyAsync(h->aff_scale, scale, size_t(n) * sizeof(double), cudaMemcpyHostToDevice,
                                     h->stream));
        }
        if (shift) {
            h->aff_shift = h->alloc<double>(size_t(n));
            MLP_CUDA(cudaMemcpyAsync(h->aff_shift, shift, size_t(n) * sizeof(double), cudaMemcpyHostToDevice,
                                     h->stream));
        }
        MLP_CUDA(cudaStreamSynchronize(h->stream));
        h->aff_n = n;
        h->aff_col = col;
        h->aff_lo = lo;
        h->aff_hi = hi;
    } catch (const std::exception& e) {
        h->aff_n = 0;
        return fail(e, false);
    }
    return 0;
}

int nir_mlp_predict_device_affine(nir_mlp* h, const float* x_dev, int32_t n, const double** out_dev) {
    if (!h || !x_dev || !out_dev || n < 8 || n % 8 != 0 || n != h->aff_n) {
        g_err = "invalid arguments (n must be the n of nir_mlp_set_affine)";
        return 2;
    }
    try {
        MLP_CUDA(cudaSetDevice(h->device));
        const int chunk = std::min(n, 65536);
        ensure_rows(h, chunk);
        for (int r = 0; r < n; r += chunk) {
            const int k = std::min(chunk, n - r);
            const size_t len = (size_t)k * h->cfg.d_in;
            k_to_bf16<<<grid1d(len), 256, 0, h->stream>>>(len, x_dev + (size_t)r * h->cfg.d_in, h->x);
            MLP_LAUNCHED();
            forward(h, k);
            k_affine_out<<<unsigned((k + 255) / 256), 256, 0, h->stream>>>(k, r, h->pred, h->cfg.d_out, h->aff_col,
                                                                          h->aff_lo, h->aff_hi, h->aff_scale,
                                                                          h->aff_shift, h->aff_out);
            MLP_LAUNCHED();
        }
        MLP_CUDA(cudaStreamSynchronize(h->stream));
        *out_dev = h->aff_out;
    } catch (const std::exception& e) {
        return fail(e, false);
    }
    return 0;
}

int nir_mlp_gradients(nir_mlp* h, const float* x, const float* targets, int32_t n, float* loss, float* grads) {
    if (!h || !x || !targets || n < 8 || n % 8 != 0 || n > 4096) {
        g_err = "invalid arguments (n must be a multiple of 8 in [8, 4096])";
        return 2;
    }
    try {
        MLP_CUDA(cudaSetDevice(h->device));
        ensure_rows(h, n);
        upload_rows(h, x, n, h->x, h->cfg.d_in);
        MLP_CUDA(cudaMemcpyAsync(h->tgt, targets, (size_t)n * h->cfg.d_out * sizeof(float), cudaMemcpyHostToDevice,
                                 h->stream));
        forward(h, n);
        backward(h, n, 0);
        float lv = 0.f;
        MLP_CUDA(cudaMemcpyAsync(&lv, h->losses, sizeof(float), cudaMemcpyDeviceToHost, h->stream));
        if (grads) {
            size_t o = 0;
            for (auto& ly : h->layers) {
                const size_t nw = (size_t)ly.in * ly.out;
                MLP_CUDA(cudaMemcpyAsync(grads + o, ly.gW, nw * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
                o += nw;
                MLP_CUDA(cudaMemcpyAsync(grads + o, ly.gb, ly.out * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
                o += ly.out;
            }
        }
        MLP_CUDA(cudaStreamSynchronize(h->stream));
        if (loss) *loss = lv;
    } catch (const std::exception& e) {
        return fail(e, false);
    }
    return 0;
}

int nir_mlp_gemm_check(nir_mlp* h, int a_kmaj, int b_kmaj, int32_t M, int32_t N, int32_t K, const float* A,
                       int32_t lda, const float* B, int32_t ldb, float* C) {
    if (!h || !A || !B || !C || M < 1 || N < 1 || K < 1) {
        g_err = "invalid arguments";
        return 2;
    }
    try {
        MLP_CUDA(cudaSetDevice(h->device));
        const size_t na = a_kmaj ? (size_t)M * lda : (size_t)K * lda;
        const size_t nb = b_kmaj ? (size_t)N * ldb : (size_t)K * ldb;
        if ((a_kmaj && lda < K) || (!a_kmaj && lda < M) || (b_kmaj && ldb < K) || (!b_kmaj && ldb < N))
            throw std::invalid_argument("leading dimension too small");
        bf16* da = h->alloc<bf16>(na);
        bf16* db = h->alloc<bf16>(nb);
        float* dc = h->alloc<float>((size_t)M * N);
        upload_rows(h, A, 1, da, int(na));
        upload_rows(h, B, 1, db, int(nb));
        gemm(h, a_kmaj != 0, b_kmaj != 0, da, lda, db, ldb, M, N, K, EPI_F32, nullptr, nullptr, dc, N, nullptr, 0);
        MLP_CUDA(cudaMemcpyAsync(C, dc, (size_t)M * N * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
        MLP_CUDA(cudaStreamSynchronize(h->stream));
        h->release(da);
        h->release(db);
        h->release(dc);
    } catch (const std::invalid_argument& e) {
        return fail(e, true);
    } catch (const std::exception& e) {
        return fail(e, false);
    }
    return 0;
}

int nir_mlp_gemm_time(nir_mlp* h, int32_t M, int32_t N, int32_t K, int32_t reps, double* us) {
    if (!h || !us || M < 8 || N < 8 || K < 8 || M % 8 || N % 8 || K % 8 || reps < 1) {
        g_err = "invalid arguments";
        return 2;
    }
    try {
        MLP_CUDA(cudaSetDevice(h->device));
        bf16* a = h->alloc<bf16>((size_t)M * K);
        bf16* b = h->alloc<bf16>((size_t)N * K);
        bf16* c = h->alloc<bf16>((size_t)M * N);
        float* bias = h->alloc<float>(N);
        cudaEvent_t e0, e1;
        MLP_CUDA(cudaEventCreate(&e0));
        MLP_CUDA(cudaEventCreate(&e1));
        gemm(h, true, true, a, K, b, K, M, N, K, EPI_BIAS_RELU_BF16, bias, c, nullptr, N, nullptr, 0);  // warm-up
        MLP_CUDA(cudaEventRecord(e0, h->stream));
        for (int r = 0; r < reps; ++r)
            gemm(h, true, true, a, K, b, K, M, N, K, EPI_BIAS_RELU_BF16, bias, c, nullptr, N, nullptr, 0);
        MLP_CUDA(cudaEventRecord(e1, h->stream));
        MLP_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        MLP_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        *us = 1000.0 * ms / reps;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        h->release(a);
        h->release(b);
        h->release(c);
        h->release(bias);
    } catch (const std::exception& e) {
        return fail(e, false);
    }
    return 0;
}

int nir_mlp_step_stats(nir_mlp* h, double* us_per_step, double* flops_per_step) {
    if (!h) return 2;
    if (us_per_step) *us_per_step = h->us_per_step;
    if (flops_per_step) *flops_per_step = h->flops_per_step;
    return 0;
}

}  // extern "C"

// ---------------------------------------------------------------- blending-family features

namespace {

__global__ void k_blend_cols(int n, int nf, const float* __restrict__ tmpl, const double* __restrict__ g,
                             const double* __restrict__ f, const double* __restrict__ cost0,
                             const double* __restrict__ atybar, const double* __restrict__ dem_w, double cscale,
                             const long long* __restrict__ rp, const int* __restrict__ ci,
                             const double* __restrict__ val, float* __restrict__ out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const float* t = tmpl + (size_t)j * nf;
    float* o = out + (size_t)j * nf;
    for (int k = 0; k < nf; ++k) o[k] = t[k];
    const double gj = g[j];
    const double c = cost0[j] * gj;
    double dp = 0.0;
    for (long long q = rp[j]; q < rp[j + 1]; ++q) dp += val[q] * (f[ci[q]] - 1.0);
    o[0] = float((gj - 1.0) / 0.1);
    o[1] = float(c / cscale);
    o[2] = float((c - atybar[j]) / cscale);
    o[6] = float(dp / fmax(dem_w[j], 1e-12) / 0.2);
}

__global__ void k_blend_rows(int m, int nd, int nf, const float* __restrict__ tmpl, const double* __restrict__ f,
                             const double* __restrict__ g, const double* __restrict__ rowlo0,
                             const double* __restrict__ rowup, const double* __restrict__ axbar,
                             const double* __restrict__ bscale, const double* __restrict__ row_abs,
                             const long long* __restrict__ rp, const int* __restrict__ ci,
                             const double* __restrict__ val, float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const float* t = tmpl + (size_t)i * nf;
    float* o = out + (size_t)i * nf;
    for (int k = 0; k < nf; ++k) o[k] = t[k];
    const double lo = (i < nd) ? rowlo0[i] * f[i] : rowlo0[i];
    const double up = rowup[i];
    double gp = 0.0;
    for (long long q = rp[i]; q < rp[i + 1]; ++q) gp += val[q] * (g[ci[q]] - 1.0);
    if (i < nd) o[1] = float((f[i] - 1.0) / 0.2);
    o[4] = float((isfinite(lo) ? axbar[i] - lo : 0.0) / bscale[i]);
    o[5] = float((isfinite(up) ? up - axbar[i] : 0.0) / bscale[i]);
    o[6] = float(gp / fmax(row_abs[i], 1e-12) / 0.1);
}

}  // namespace

struct nir_blend_features {
    int device = 0;
    cudaStream_t stream = nullptr;
    int n = 0, m = 0, nd = 0, nf = 0;
    double cscale = 1.0;
    std::vector<void*> allocs;
    float *col_t = nullptr, *row_t = nullptr, *col_out = nullptr, *row_out = nullptr;
    double *cost0 = nullptr, *atybar = nullptr, *dem_w = nullptr, *dem_val = nullptr;
    double *rowlo0 = nullptr, *rowup = nullptr, *axbar = nullptr, *bscale = nullptr, *row_abs = nullptr,
           *abs_val = nullptr;
    long long *dem_rp = nullptr, *abs_rp = nullptr;
    int *dem_ci = nullptr, *abs_ci = nullptr;
    double *f = nullptr, *g = nullptr;

    template <typename T>
    T* upload(const T* src, size_t count) {
        void* p = nullptr;
        MLP_CUDA(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)));
        allocs.push_back(p);
        if (src && count) MLP_CUDA(cudaMemcpy(p, src, count * sizeof(T), cudaMemcpyHostToDevice));
        return static_cast<T*>(p);
    }
    ~nir_blend_features() {
        cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        for (void* p : allocs) cudaFree(p);
        if (stream) cudaStreamDestroy(stream);
    }
};

extern "C" {

int nir_blend_features_create(const nir_blend_feature_data* d, int32_t device, nir_blend_features** out) {
    if (!d || !out || d->n < 0 || d->m < 0 || d->nd < 0 || d->nd > d->m || d->nf < 7 || !d->col_template ||
        !d->row_template || !d->cost0 || !d->atybar || !d->dem_w || !d->dem_rp || !d->rowlo0 || !d->rowup ||
        !d->axbar || !d->bscale || !d->row_abs || !d->abs_rp) {
        g_err = "invalid blending-feature data";
        return 2;
    }
    *out = nullptr;
    auto h = std::make_unique<nir_blend_features>();
    try {
        const long long dn = d->dem_rp[d->n], an = d->abs_rp[d->m];
        if (dn < 0 || an < 0 || (dn > 0 && (!d->dem_ci || !d->dem_val)) || (an > 0 && (!d->abs_ci || !d->abs_val)))
            throw std::invalid_argument("invalid feature operators");
        for (long long q = 0; q < dn; ++q)
            if (d->dem_ci[q] < 0 || d->dem_ci[q] >= d->nd) throw std::invalid_argument("demand index out of range");
        for (long long q = 0; q < an; ++q)
            if (d->abs_ci[q] < 0 || d->abs_ci[q] >= d->n) throw std::invalid_argument("column index out of range");
        h->device = device;
        MLP_CUDA(cudaSetDevice(device));
        MLP_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        h->n = d->n;
        h->m = d->m;
        h->nd = d->nd;
        h->nf = d->nf;
        h->cscale = d->cscale;
        const size_t n = size_t(d->n), m = size_t(d->m), nf = size_t(d->nf);
        h->col_t = h->upload(d->col_template, n * nf);
        h->row_t = h->upload(d->row_template, m * nf);
        h->col_out = h->upload<float>(nullptr, n * nf);
        h->row_out = h->upload<float>(nullptr, m * nf);
        h->cost0 = h->upload(d->cost0, n);
        h->atybar = h->upload(d->atybar, n);
        h->dem_w = h->upload(d->dem_w, n);
        h->rowlo0 = h->upload(d->rowlo0, m);
        h->rowup = h->upload(d->rowup, m);
        h->axbar = h->upload(d->axbar, m);
        h->bscale = h->upload(d->bscale, m);
        h->row_abs = h->upload(d->row_abs, m);
        static_assert(sizeof(long long) == sizeof(int64_t), "64-bit offsets");
        h->dem_rp = h->upload(reinterpret_cast<const long long*>(d->dem_rp), n + 1);
        h->dem_ci = h->upload(d->dem_ci, size_t(dn));
        h->dem_val = h->upload(d->dem_val, size_t(dn));
        h->abs_rp = h->upload(reinterpret_cast<const long long*>(d->abs_rp), m + 1);
        h->abs_ci = h->upload(d->abs_ci, size_t(an));
        h->abs_val = h->upload(d->abs_val, size_t(an));
        h->f = h->upload<double>(nullptr, std::max<size_t>(size_t(d->nd), 1));
        h->g = h->upload<double>(nullptr, n);
    } catch (const std::invalid_argument& e) {
        return fail(e, true);
    } catch (const std::exception& e) {
        return fail(e, false);
    }
    *out = h.release();
    return 0;
}

int nir_blend_features_build(nir_blend_features* h, const double* f, const double* g, const float** col_dev,
                             const float** row_dev) {
    if (!h || (!f && h->nd > 0) || (!g && h->n > 0) || !col_dev || !row_dev) {
        g_err = "invalid arguments";
        return 2;
    }
    try {
        MLP_CUDA(cudaSetDevice(h->device));
        cudaStream_t s = h->stream;
        if (h->nd) MLP_CUDA(cudaMemcpyAsync(h->f, f, size_t(h->nd) * sizeof(double), cudaMemcpyHostToDevice, s));
        if (h->n) MLP_CUDA(cudaMemcpyAsync(h->g, g, size_t(h->n) * sizeof(double), cudaMemcpyHostToDevice, s));
        if (h->n)
            k_blend_cols<<<unsigned((h->n + 255) / 256), 256, 0, s>>>(h->n, h->nf, h->col_t, h->g, h->f, h->cost0,
                                                                     h->atybar, h->dem_w, h->cscale, h->dem_rp,
                                                                     h->dem_ci, h->dem_val, h->col_out);
        if (h->m)
            k_blend_rows<<<unsigned((h->m + 255) / 256), 256, 0, s>>>(h->m, h->nd, h->nf, h->row_t, h->f, h->g,
                                                                     h->rowlo0, h->rowup, h->axbar, h->bscale,
                                                                     h->row_abs, h->abs_rp, h->abs_ci, h->abs_val,
                                                                     h->row_out);
        MLP_LAUNCHED();
        MLP_CUDA(cudaStreamSynchronize(s));
        *col_dev = h->col_out;
        *row_dev = h->row_out;
    } catch (const std::exception& e) {
        return fail(e, false);
    }
    return 0;
}

void nir_blend_features_free(nir_blend_features* h) { delete h; }

}  // extern "C"
