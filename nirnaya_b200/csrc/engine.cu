// Host side of the B200 PDHG engine and its C ABI (include/nir_pdhg.h).
//
// One handle = one LP resident on one GPU: CSR(A) and CSR(A') (the CSC of
// A read as rows), original and scaled FP64 values, FP32 values, and every
// vector the iteration touches.  A solve runs launch chunks of K
// iterations (each chunk ends with the FP64 KKT evaluation, the restart /
// primal-weight controller and a status snapshot to host-mapped memory),
// captured once into CUDA graphs and replayed with a few chunks in flight.
// The host only reads the snapshots, polls the caller's deadline and
// decides when to switch from FP32 to the FP64 polish.

#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <limits>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "dev_common.cuh"
#include "k_adaptive.cuh"
#include "k_persistent.cuh"
#include "k_reference.cuh"
#include "k_setup.cuh"
#include "k_verify.cuh"
#include "k_cta.cuh"
#include "k_iter.cuh"
#include "k_batch.cuh"
#include "nir_pdhg.h"

namespace {

thread_local std::string g_err;

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

#define NIR_CUDA(call)                                                                                  \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess)                                                                          \
            throw CudaError(std::string(#call) + ": " + cudaGetErrorString(e_) + " (" __FILE__ ":" +    \
                            std::to_string(__LINE__) + ")");                                            \
    } while (0)

#define NIR_LAUNCHED() NIR_CUDA(cudaGetLastError())

inline unsigned grid_for(long long n, int b = nir::kBlock) {
    long long g = (n + b - 1) / b;
    return unsigned(g < 1 ? 1 : g);
}

double now_sec() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// ---- double-double accumulation for the objective (Dekker / Knuth
// error-free transformations; the reference's Model::eval_objective,
// src/model/model.hpp:73-98, evaluates c'x + offset the same way).
struct DD {
    double hi = 0.0, lo = 0.0;
};
inline void two_sum(double a, double b, double& s, double& e) {
    s = a + b;
    double bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}
inline void quick_two_sum(double a, double b, double& s, double& e) {
    s = a + b;
    e = b - (s - a);
}
inline DD dd_add(DD a, DD b) {
    double s1, s2, t1, t2;
    two_sum(a.hi, b.hi, s1, s2);
    two_sum(a.lo, b.lo, t1, t2);
    s2 += t1;
    quick_two_sum(s1, s2, s1, s2);
    s2 += t2;
    DD r;
    quick_two_sum(s1, s2, r.hi, r.lo);
    return r;
}
inline DD dd_add_prod(DD a, double x, double y) {
    DD p;
    p.hi = x * y;
    p.lo = std::fma(x, y, -p.hi);
    return dd_add(a, p);
}

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

// The per-orientation layout choice of a solve.
struct LayChoice {
    int lay_a = nir::kLayWarp, cap_a = 256;    // A (dual half-iteration, KKT rows)
    int lay_at = nir::kLayWarp, cap_at = 256;  // A' (primal half-iteration, KKT columns)
};

// Groups of parallel columns of an LP (engine_parallel.cuh).
struct ParallelGroups {
    std::vector<int> rep_of;  // per column: its representative, or -1
    std::vector<double> lam;  // per partner column: lambda (A_j' ~ lambda A_rep)
    std::vector<int> row_of;  // per representative: its new row (>= m), or -1
    int groups = 0;
};

}  // namespace

// ---------------------------------------------------------------- handle

struct Orient {
    int rows = 0, cols = 0;
    long long nnz = 0;
    int* rp = nullptr;
    int* ci = nullptr;
    double* v_orig = nullptr;
    double* v64 = nullptr;
    float* v32 = nullptr;
    float* v32_orig = nullptr;  // for the FP32 SpMV test entry point
    std::vector<int> h_rp;
    int cap = 0;
    int nblk = 0;
    int2* blk = nullptr;  // (first row, first nonzero) of each row block, plus an end entry
    struct Layout {
        int cap, nblk;
        int2* blk;
    };
    std::vector<Layout> layouts;  // every layout built so far, one per capacity used
    // CTA-block layouts (k_cta.cuh), one per capacity used: descriptors and
    // the padded stream of indices and values.  `it` is the one the
    // iteration and KKT kernels use (a deque keeps references stable).
    struct Cta {
        int cap = 0, nblk = 0;
        long long qlen = 0;
        int4* blk = nullptr;
        int* ci = nullptr;
        double* v64 = nullptr;     // scaled FP64 values (refreshed after each preconditioning)
        float* v32 = nullptr;      // scaled FP32 values
        double* vorig = nullptr;   // original values (kernel measurement entry points, on demand)
        float* v32orig = nullptr;  // original values rounded to FP32
    };
    std::deque<Cta> ctas;
    int it = -1;
    int lay = -1;  // layout the iteration and KKT kernels use: nir::kLayWarp (blk, cap) or nir::kLayCta (ctas[it])
    const Cta& cur() const {
        if (it < 0) throw std::logic_error("internal: no CTA layout in use");
        return ctas[size_t(it)];
    }
};

struct Snapshot {
    nir::HostSnap* ring = nullptr;  // host-mapped
    long long* d_seq = nullptr;
};

struct ChunkGraph {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    unsigned long long key = 0;
    bool valid = false;
};

struct nir_pdhg {
    int device = 0;
    cudaStream_t stream = nullptr;
    int m = 0, n = 0;
    long long nnz = 0;
    double offset = 0.0;
    Orient A, At;
    // original vectors on the device (bounds sanitised to +-inf)
    double *c = nullptr, *l = nullptr, *u = nullptr, *rl = nullptr, *ru = nullptr;
    std::vector<double> h_c, h_l, h_u, h_rl, h_ru;
    // scaling and scaled vectors
    double *dr = nullptr, *dc = nullptr;
    // what dr, dc and the scaled matrix copies hold: they depend on the
    // matrix and the scaling parameters only, so solves that change only
    // the vectors (nir_pdhg_update_vectors) reuse them and ||A||_2
    struct ScaleState {
        bool valid = false;
        bool enabled = false;
        int ruiz = -1, pc = -1;
        bool norm_valid = false;
        int power_iters = -1;
        double norm = 0.0;
    } scaled;
    double *c64 = nullptr, *l64 = nullptr, *u64 = nullptr, *rl64 = nullptr, *ru64 = nullptr;
    float *c32 = nullptr, *l32 = nullptr, *u32 = nullptr, *rl32 = nullptr, *ru32 = nullptr;
    // iterates
    double *x64 = nullptr, *xb64 = nullptr, *x064 = nullptr, *xp64 = nullptr;
    double *y64 = nullptr, *y064 = nullptr, *yp64 = nullptr;
    float *x32 = nullptr, *xb32 = nullptr, *x032 = nullptr, *xp32 = nullptr;
    float *y32 = nullptr, *y032 = nullptr, *yp32 = nullptr;
    double *tmp_n = nullptr, *tmp_m = nullptr, *out_x = nullptr, *out_y = nullptr;
    float *tmp_n32 = nullptr, *tmp_m32 = nullptr;
    double* part = nullptr;
    size_t part_len = 0;
    double* hist = nullptr;
    nir::DevState* st = nullptr;
    Snapshot snap;
    unsigned char* flush = nullptr;
    size_t flush_bytes = 0;
    double* ceil_out = nullptr;        // one running sum per thread of the ceiling kernels
    nir::DevState* st_time = nullptr;  // running copy of the state for nir_pdhg_time_iteration
    std::vector<DevBuf> bufs;
    long long device_bytes = 0;
    ChunkGraph graphs[3];
    long long last_iters = 0;
    LayChoice tuned[3];                    // autotuned layouts per NIR_PREC_*
    bool tuned_ok[3] = {false, false, false};
    int sms = 148;
    struct Occ {
        const void* fn;
        size_t smem;
        int per_sm;
    };
    std::vector<Occ> occ;
    bool profiling = false;
    nir_pdhg_kernel_time ktime{};
    unsigned* gs_count = nullptr;  // grid barrier of the persistent chunk kernel
    unsigned* gs_gen = nullptr;
    int* gs_err = nullptr;
    int launches = 0;
    const double* last_x = nullptr;  // the point the last solve returned, still on the device (null before one)
    // the engine's row order: internal row k is the caller's row
    // row_orig[k] (empty: the caller's order; see row_order below)
    std::vector<int> row_orig;
    int* d_row_orig = nullptr;
    // the equivalent LP the PDHG / PDLP solves run on when the LP has
    // parallel columns (engine_parallel.cuh), and its column groups
    std::unique_ptr<nir_pdhg> inner;
    std::unique_ptr<ParallelGroups> par;
    // the device solution check's buffers, allocated by its first call
    struct Verify {
        bool ready = false;
        int count = 0;  // instances the per-instance arrays hold
        double *x = nullptr, *rv = nullptr, *obj = nullptr, *claimed = nullptr, *offset = nullptr;
        int8_t *vt = nullptr, *rs = nullptr;
        long long* fb = nullptr;
        void *b = nullptr, *g = nullptr;  // nir::vfy::Rec[count] each
        nir_verify_report* rep = nullptr;
        int *row_off = nullptr, *col_off = nullptr;  // one instance: {0, m}, {0, n}
    } vfy;

    // zero-filled allocation with `pad` spare elements past the end (the
    // row-block copies read 16-byte windows that may reach past the end)
    template <typename T>
    T* allocz(size_t count, size_t pad = 8) {
        T* p = alloc<T>(count + pad);
        NIR_CUDA(cudaMemsetAsync(p, 0, (count + pad) * sizeof(T), stream));
        return p;
    }

    template <typename T>
    T* alloc(size_t count) {
        void* p = nullptr;
        size_t bytes = std::max<size_t>(1, count) * sizeof(T);
        NIR_CUDA(cudaMalloc(&p, bytes));
        bufs.push_back({p, bytes});
        device_bytes += (long long)bytes;
        return static_cast<T*>(p);
    }

    ~nir_pdhg() {
        if (device >= 0) cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        for (auto& g : graphs) {
            if (g.ge) cudaGraphExecDestroy(g.ge);
            if (g.g) cudaGraphDestroy(g.g);
        }
        for (auto& b : bufs) cudaFree(b.p);
        if (snap.ring) cudaFreeHost(snap.ring);
        if (stream) cudaStreamDestroy(stream);
        inner.reset();
    }
};

namespace {

// Copies ordered on the handle's (non-blocking) stream, then waited for.
void h2d(nir_pdhg* h, void* dst, const void* src, size_t bytes) {
    NIR_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, h->stream));
    NIR_CUDA(cudaStreamSynchronize(h->stream));
}
void d2h(nir_pdhg* h, void* dst, const void* src, size_t bytes) {
    NIR_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, h->stream));
    NIR_CUDA(cudaStreamSynchronize(h->stream));
}

// Warp row blocks: consecutive rows packed while their nonzeros fit in
// `cap` (<= 256) and there are at most 32 of them; a longer row gets a
// block of its own.  Returns the (first row, first nonzero) descriptors,
// one per block plus the end (rows, nnz).
using nir::build_row_blocks;
using nir::check_row_blocks;

void set_blocks(nir_pdhg* h, Orient& o, int cap) {
    if (o.cap == cap && o.blk) return;
    // a capacity used before keeps its device copy: switching back and forth
    // (the autotuner, or solves with different spmv_block_nnz) allocates once
    for (const auto& l : o.layouts)
        if (l.cap == cap) {
            o.blk = l.blk;
            o.nblk = l.nblk;
            o.cap = cap;
            return;
        }
    std::vector<int2> b = build_row_blocks(o.h_rp, cap);
    check_row_blocks(b, o.h_rp, cap);
    o.nblk = int(b.size()) - 1;
    o.blk = h->alloc<int2>(b.size());
    h2d(h, o.blk, b.data(), b.size() * sizeof(int2));
    o.cap = cap;
    o.layouts.push_back({cap, o.nblk, o.blk});
}

// The CTA-block layout of an orientation for capacity `cap` (256 E), built
// on first use: descriptors checked on the host, then the padded stream of
// column indices filled on the device; the value streams are filled by
// pad_scaled (scaled values) or cta_orig_values (original values).
Orient::Cta& cta_layout(nir_pdhg* h, Orient& o, int cap) {
    for (auto& c : o.ctas)
        if (c.cap == cap) return c;
    std::vector<int4> b = nir::build_cta_blocks(o.h_rp, cap);
    nir::check_cta_blocks(b, o.h_rp, cap);
    Orient::Cta c;
    c.cap = cap;
    c.nblk = int(b.size()) - 1;
    c.qlen = b.back().z;
    c.blk = h->alloc<int4>(b.size());
    h2d(h, c.blk, b.data(), b.size() * sizeof(int4));
    // 8 spare entries keep every allocation non-empty
    c.ci = h->allocz<int>(size_t(c.qlen), 8);
    c.v64 = h->allocz<double>(size_t(c.qlen), 8);
    c.v32 = h->allocz<float>(size_t(c.qlen), 8);
    cudaStream_t s = h->stream;
    if (c.nblk > 0 && o.nnz > 0) {
        const unsigned g = unsigned(std::max(1, std::min(c.nblk, 4 * h->sms)));
        nir::k_pad_stream<double><<<g, nir::kBlock, 0, s>>>(c.blk, c.nblk, o.ci, o.v_orig, c.ci, c.v64);
        NIR_LAUNCHED();
    }
    NIR_CUDA(cudaStreamSynchronize(s));
    o.ctas.push_back(c);
    return o.ctas.back();
}

// The original values in a CTA layout's padded stream (FP64 and rounded to
// FP32), for the kernel measurement entry points.
void cta_orig_values(nir_pdhg* h, Orient& o, Orient::Cta& c) {
    if (c.vorig) return;
    cudaStream_t s = h->stream;
    c.vorig = h->allocz<double>(size_t(c.qlen), 8);
    c.v32orig = h->allocz<float>(size_t(c.qlen), 8);
    if (c.nblk > 0 && o.nnz > 0) {
        if (!o.v32_orig) {
            o.v32_orig = h->allocz<float>(o.nnz);
            nir::k_to_float<<<grid_for(o.nnz), nir::kBlock, 0, s>>>(o.nnz, o.v_orig, o.v32_orig);
            NIR_LAUNCHED();
        }
        const unsigned g = unsigned(std::max(1, std::min(c.nblk, 4 * h->sms)));
        nir::k_pad_stream<double><<<g, nir::kBlock, 0, s>>>(c.blk, c.nblk, o.ci, o.v_orig, nullptr, c.vorig);
        nir::k_pad_stream<float><<<g, nir::kBlock, 0, s>>>(c.blk, c.nblk, o.ci, o.v32_orig, nullptr, c.v32orig);
        NIR_LAUNCHED();
    }
    NIR_CUDA(cudaStreamSynchronize(s));
}

// Warp row-block capacity: 256 nonzeros (8 per lane) when the matrix gives
// every SM many warps, smaller for small matrices so that the grid still
// covers the GPU.
int auto_cap(long long nnz, int rows) {
    (void)rows;
    int sms = 148;
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    long long per = nnz / (long long)(32 * std::max(sms, 1));
    int cap = 32;
    while (cap < nir::kWarpCapMax && cap * 2 <= per) cap *= 2;
    return cap;
}

void validate_lp(const nir_lp_view* lp) {
    if (!lp) throw std::invalid_argument("null LP");
    if (lp->nrow < 0 || lp->ncol < 0) throw std::invalid_argument("negative dimension");
    if (!lp->col_start || (lp->nnz > 0 && (!lp->row_index || !lp->value)))
        throw std::invalid_argument("missing matrix arrays");
    if ((lp->ncol > 0 && (!lp->cost || !lp->collo || !lp->colup)) || (lp->nrow > 0 && (!lp->rowlo || !lp->rowup)))
        throw std::invalid_argument("missing vector arrays");
    if (lp->col_start[0] != 0 || lp->col_start[lp->ncol] != lp->nnz) throw std::invalid_argument("column starts");
    if (lp->nnz >= (1LL << 31) - 1) throw std::invalid_argument("more than 2^31-2 nonzeros");
    for (int j = 0; j < lp->ncol; ++j)
        if (lp->col_start[j + 1] < lp->col_start[j]) throw std::invalid_argument("column starts not nondecreasing");
    for (long long k = 0; k < lp->nnz; ++k) {
        if (lp->row_index[k] < 0 || lp->row_index[k] >= lp->nrow) throw std::invalid_argument("row index out of range");
        if (!std::isfinite(lp->value[k])) throw std::invalid_argument("non-finite matrix entry");
    }
    for (int j = 0; j < lp->ncol; ++j)
        if (!std::isfinite(lp->cost[j])) throw std::invalid_argument("non-finite cost");
}

// The engine's row order.  On an LP whose row lengths are skewed (the
// longest row at least 8 times the mean, m >= 1024) the rows are held
// longest first (stable).  The SpMV of A then starts its long rows first,
// so that they do not finish last, and the entries of y that A' y gathers
// most often sit together, so that they stay in L1.  On the 200,000 x
// 500,000 power-law LP this took the FP64 iteration from 74 to 59 us and
// the solve from 11.1 to 9.4 s, with the same iterations.  Every row keeps
// its entries and their order and every column its entries' order, so the
// reference loop's sequential sums are the same bits (the row-block SpMVs
// sum a row by a tree that depends on the rows sharing its block, so they
// agree to rounding), and the caller sees its own order: row-indexed
// inputs and outputs are mapped at the C ABI.  NIR_PDHG_ROW_ORDER=0 keeps the caller's order,
// =1 reorders whatever the lengths.
std::vector<int> row_order(const nir_lp_view* lp) {
    const int m = lp->nrow;
    const char* env = std::getenv("NIR_PDHG_ROW_ORDER");
    const std::string mode = env ? env : "";
    if (mode == "0" || m <= 1) return {};
    std::vector<long long> len(static_cast<size_t>(m), 0);
    for (long long k = 0; k < lp->nnz; ++k) ++len[size_t(lp->row_index[k])];
    const long long mx = *std::max_element(len.begin(), len.end());
    const bool skewed = m >= 1024 && double(mx) >= 8.0 * double(lp->nnz) / double(m);
    if (mode != "1" && !skewed) return {};
    std::vector<int> order(static_cast<size_t>(m));
    for (int i = 0; i < m; ++i) order[size_t(i)] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return len[size_t(a)] > len[size_t(b)]; });
    bool identity = true;
    for (int i = 0; i < m && identity; ++i) identity = order[size_t(i)] == i;
    if (identity) return {};
    return order;
}

// An LP view in the engine's row order: the row indices relabelled (each
// column keeps its entries in their order) and the row bounds permuted,
// in the buffers given.
nir_lp_view reorder_rows(const nir_lp_view* lp, const std::vector<int>& row_orig, std::vector<int>& ri,
                         std::vector<double>& rl, std::vector<double>& ru) {
    const int m = lp->nrow;
    std::vector<int> inv(static_cast<size_t>(m));
    for (int k = 0; k < m; ++k) inv[size_t(row_orig[size_t(k)])] = k;
    ri.resize(size_t(lp->nnz));
    for (long long k = 0; k < lp->nnz; ++k) ri[size_t(k)] = inv[size_t(lp->row_index[k])];
    rl.resize(size_t(m));
    ru.resize(size_t(m));
    for (int k = 0; k < m; ++k) {
        rl[size_t(k)] = lp->rowlo[row_orig[size_t(k)]];
        ru[size_t(k)] = lp->rowup[row_orig[size_t(k)]];
    }
    nir_lp_view v = *lp;
    v.row_index = ri.data();
    v.rowlo = rl.data();
    v.rowup = ru.data();
    return v;
}

// True when p is device (or managed) memory, as a starting point given by
// its device address is; false for host memory, pinned or pageable.
bool device_resident(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// A starting vector that the host must read (to remap it): a device-resident
// one is copied into buf first.
const double* host_readable(const double* p, size_t len, std::vector<double>& buf) {
    if (!p || !device_resident(p)) return p;
    buf.resize(len);
    NIR_CUDA(cudaMemcpy(buf.data(), p, len * sizeof(double), cudaMemcpyDefault));
    return buf.data();
}

// A row-indexed vector of the caller's into the engine's order, and back.
void rows_in(const nir_pdhg* h, const double* src, std::vector<double>& dst) {
    dst.resize(size_t(h->m));
    for (int k = 0; k < h->m; ++k) dst[size_t(k)] = src[h->row_orig[size_t(k)]];
}
void rows_out(const nir_pdhg* h, const double* src, double* dst) {
    for (int k = 0; k < h->m; ++k) dst[h->row_orig[size_t(k)]] = src[k];
}

void upload_vectors(nir_pdhg* h, const double* cost, const double* collo, const double* colup, const double* rowlo,
                    const double* rowup) {
    const int n = h->n, m = h->m;
    auto sanitize = [](double b, bool lower) {
        bool f = std::isfinite(b) && std::fabs(b) < 1e20;
        return f ? b : (lower ? -INFINITY : INFINITY);
    };
    if (cost) h->h_c.assign(cost, cost + n);
    if (collo) {
        h->h_l.resize(n);
        for (int j = 0; j < n; ++j) h->h_l[j] = sanitize(collo[j], true);
    }
    if (colup) {
        h->h_u.resize(n);
        for (int j = 0; j < n; ++j) h->h_u[j] = sanitize(colup[j], false);
    }
    if (rowlo) {
        h->h_rl.resize(m);
        for (int i = 0; i < m; ++i) h->h_rl[i] = sanitize(rowlo[i], true);
    }
    if (rowup) {
        h->h_ru.resize(m);
        for (int i = 0; i < m; ++i) h->h_ru[i] = sanitize(rowup[i], false);
    }
    auto up = [&](double* d, const std::vector<double>& v) {
        if (!v.empty()) NIR_CUDA(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    };
    if (cost) up(h->c, h->h_c);
    if (collo) up(h->l, h->h_l);
    if (colup) up(h->u, h->h_u);
    if (rowlo) up(h->rl, h->h_rl);
    if (rowup) up(h->ru, h->h_ru);
    NIR_CUDA(cudaStreamSynchronize(h->stream));
}

void create_impl(nir_pdhg* h, const nir_lp_view* lp, int device) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0)
        throw CudaError("no CUDA device available (the PDHG engine has no CPU fallback)");
    if (device < 0 || device >= ndev) throw std::invalid_argument("device ordinal out of range");
    h->device = device;
    NIR_CUDA(cudaSetDevice(device));
    NIR_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    NIR_CUDA(cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, device));
    const int m = lp->nrow, n = lp->ncol;
    const long long nnz = lp->nnz;
    h->m = m;
    h->n = n;
    h->nnz = nnz;
    h->offset = lp->obj_offset;
    cudaStream_t s = h->stream;

    // A' = CSC of A read as rows.
    Orient& T = h->At;
    T.rows = n;
    T.cols = m;
    T.nnz = nnz;
    T.rp = h->allocz<int>(n + 1);
    T.ci = h->allocz<int>(nnz);
    T.v_orig = h->allocz<double>(nnz);
    T.v64 = h->allocz<double>(nnz);
    T.v32 = h->allocz<float>(nnz);
    long long* d_start = h->alloc<long long>(n + 1);
    NIR_CUDA(cudaMemcpyAsync(d_start, lp->col_start, (n + 1) * sizeof(long long), cudaMemcpyHostToDevice, s));
    NIR_CUDA(cudaMemcpyAsync(T.ci, lp->row_index, nnz * sizeof(int), cudaMemcpyHostToDevice, s));
    NIR_CUDA(cudaMemcpyAsync(T.v_orig, lp->value, nnz * sizeof(double), cudaMemcpyHostToDevice, s));
    nir::k_offsets_to_int<<<grid_for(n + 1), nir::kBlock, 0, s>>>(n + 1, d_start, T.rp);
    NIR_LAUNCHED();
    T.h_rp.resize(n + 1);
    for (int j = 0; j <= n; ++j) T.h_rp[j] = int(lp->col_start[j]);

    // A: stable radix sort of the CSC entries by row keeps each row's
    // entries in ascending column order (the reference's scatter order).
    Orient& R = h->A;
    R.rows = m;
    R.cols = n;
    R.nnz = nnz;
    R.rp = h->allocz<int>(m + 1);
    R.ci = h->allocz<int>(nnz);
    R.v_orig = h->allocz<double>(nnz);
    R.v64 = h->allocz<double>(nnz);
    R.v32 = h->allocz<float>(nnz);
    {
        int* col_of = h->alloc<int>(nnz);
        int* ids = h->alloc<int>(nnz);
        int* perm = h->alloc<int>(nnz);
        int* keys_out = h->alloc<int>(nnz);
        nir::k_expand_cols<<<grid_for(n), nir::kBlock, 0, s>>>(n, d_start, col_of);
        NIR_LAUNCHED();
        nir::k_iota<<<grid_for(nnz), nir::kBlock, 0, s>>>(nnz, ids);
        NIR_LAUNCHED();
        int end_bit = 1;
        while ((1LL << end_bit) <= (long long)m) ++end_bit;
        size_t tmp_bytes = 0;
        NIR_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, T.ci, keys_out, ids, perm, (int)nnz, 0, end_bit, s));
        void* tmp = h->alloc<unsigned char>(tmp_bytes);
        NIR_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, T.ci, keys_out, ids, perm, (int)nnz, 0, end_bit, s));
        nir::k_row_ptr_from_sorted<<<grid_for(m + 1), nir::kBlock, 0, s>>>(m, nnz, keys_out, R.rp);
        NIR_LAUNCHED();
        nir::k_gather_csr<<<grid_for(nnz), nir::kBlock, 0, s>>>(nnz, perm, col_of, T.v_orig, R.ci, R.v_orig);
        NIR_LAUNCHED();
        R.h_rp.resize(m + 1);
        NIR_CUDA(cudaMemcpyAsync(R.h_rp.data(), R.rp, (m + 1) * sizeof(int), cudaMemcpyDeviceToHost, s));
        NIR_CUDA(cudaStreamSynchronize(s));
        // scratch of the transpose is released right away
        for (void* p : {(void*)col_of, (void*)ids, (void*)perm, (void*)keys_out, tmp, (void*)d_start}) {
            for (auto it = h->bufs.begin(); it != h->bufs.end(); ++it)
                if (it->p == p) {
                    h->device_bytes -= (long long)it->bytes;
                    cudaFree(it->p);
                    h->bufs.erase(it);
                    break;
                }
        }
    }

    // vectors
    h->c = h->alloc<double>(n);
    h->l = h->alloc<double>(n);
    h->u = h->alloc<double>(n);
    h->rl = h->alloc<double>(m);
    h->ru = h->alloc<double>(m);
    upload_vectors(h, lp->cost, lp->collo, lp->colup, lp->rowlo, lp->rowup);
    h->dr = h->alloc<double>(m);
    h->dc = h->alloc<double>(n);
    h->c64 = h->alloc<double>(n);
    h->l64 = h->alloc<double>(n);
    h->u64 = h->alloc<double>(n);
    h->rl64 = h->alloc<double>(m);
    h->ru64 = h->alloc<double>(m);
    h->c32 = h->alloc<float>(n);
    h->l32 = h->alloc<float>(n);
    h->u32 = h->alloc<float>(n);
    h->rl32 = h->alloc<float>(m);
    h->ru32 = h->alloc<float>(m);
    h->x64 = h->alloc<double>(n);
    h->xb64 = h->alloc<double>(n);
    h->x064 = h->alloc<double>(n);
    h->xp64 = h->alloc<double>(n);
    h->y64 = h->alloc<double>(m);
    h->y064 = h->alloc<double>(m);
    h->yp64 = h->alloc<double>(m);
    h->x32 = h->alloc<float>(n);
    h->xb32 = h->alloc<float>(n);
    h->x032 = h->alloc<float>(n);
    h->xp32 = h->alloc<float>(n);
    h->y32 = h->alloc<float>(m);
    h->y032 = h->alloc<float>(m);
    h->yp32 = h->alloc<float>(m);
    h->tmp_n = h->alloc<double>(n);
    h->tmp_m = h->alloc<double>(m);
    h->tmp_n32 = h->alloc<float>(n);
    h->tmp_m32 = h->alloc<float>(m);
    h->out_x = h->alloc<double>(n);
    h->out_y = h->alloc<double>(m);
    h->st = h->alloc<nir::DevState>(1);
    h->hist = h->alloc<double>(8 * nir::kHist);
    h->snap.d_seq = h->alloc<long long>(1);
    h->gs_count = h->allocz<unsigned>(1);
    h->gs_gen = h->allocz<unsigned>(1);
    h->gs_err = h->allocz<int>(1);
    NIR_CUDA(cudaMemsetAsync(h->snap.d_seq, 0, sizeof(long long), s));
    NIR_CUDA(cudaHostAlloc((void**)&h->snap.ring, sizeof(nir::HostSnap) * nir::kSnapRing, cudaHostAllocMapped));
    std::memset(h->snap.ring, 0, sizeof(nir::HostSnap) * nir::kSnapRing);
    NIR_CUDA(cudaStreamSynchronize(s));
}

// Launch shape of a row-block kernel: one warp per warp row block.
struct LaunchCfg {
    int grid;
    size_t smem;
};

// Shared-memory carveout preference of the SpMV kernels, in percent of the
// maximum, set before their occupancy query: 28 % (64 KB) holds the 2-4
// resident CTAs' shared memory and leaves the rest of the 256 KB to L1 for
// the gathers (C2's A' y 2-3 % faster than the CUDA driver's 100 KB choice; 0 %,
// "prefer L1", cut the resident CTAs and made the iteration 35 % slower).
#ifndef NIR_SMEM_CARVEOUT
#define NIR_SMEM_CARVEOUT 28
#endif
template <typename K>
void prefer_carveout(K* kernel) {
    if (NIR_SMEM_CARVEOUT >= 0)
        NIR_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, NIR_SMEM_CARVEOUT));
}

// Persistent grid: as many CTAs as are resident at once (occupancy), at most
// one warp per warp row block.  The occupancy query runs once per kernel
// (outside any stream capture: warm_cfgs is called before capturing).
template <typename TA, typename K>
LaunchCfg warp_cfg(nir_pdhg* h, K* kernel, int nblk) {
    const size_t smem = size_t(nir::warp_smem_bytes<TA>());
    int per = 0;
    for (auto& e : h->occ)
        if (e.fn == (const void*)kernel && e.smem == smem) per = e.per_sm;
    if (per == 0) {
        prefer_carveout(kernel);
        NIR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, nir::kBlock, smem));
        per = std::max(per, 1);
        h->occ.push_back({(const void*)kernel, smem, per});
    }
    const int need = std::max(1, (nblk + nir::kWarps - 1) / nir::kWarps);
    return {std::min(need, per * h->sms), smem};
}

int max_grid(const nir_pdhg* h) { return 8 * h->sms; }  // 2048 threads per SM / kBlock

// Partial-sum area large enough for any kernel of this handle.
void ensure_partials(nir_pdhg* h) {
    size_t need = 12 * size_t(max_grid(h)) + size_t(grid_for(std::max(h->m, h->n))) + 16;
    if (h->part && h->part_len >= need) return;
    h->part = h->alloc<double>(need);
    h->part_len = need;
}

struct PartLayout {
    double *P, *D, *KR, *KC, *misc;
};

PartLayout part_layout(nir_pdhg* h) {
    const int G = max_grid(h);
    PartLayout L;
    L.P = h->part;
    L.D = L.P + 2 * G;
    L.KR = L.D + 2 * G;
    L.KC = L.KR + 4 * G;
    L.misc = L.KC + 4 * G;
    return L;
}

// ---------------------------------------------------------------- precision views

// Iterate vectors by type: FP32 (x32 ...) or FP64 (x64 ...).
template <typename TX>
struct Vec;

template <>
struct Vec<float> {
    static float* x(nir_pdhg* h) { return h->x32; }
    static float* xb(nir_pdhg* h) { return h->xb32; }
    static float* x0(nir_pdhg* h) { return h->x032; }
    static float* xp(nir_pdhg* h) { return h->xp32; }
    static float* y(nir_pdhg* h) { return h->y32; }
    static float* y0(nir_pdhg* h) { return h->y032; }
    static float* yp(nir_pdhg* h) { return h->yp32; }
    static const float* c(nir_pdhg* h) { return h->c32; }
    static const float* l(nir_pdhg* h) { return h->l32; }
    static const float* u(nir_pdhg* h) { return h->u32; }
    static const float* rl(nir_pdhg* h) { return h->rl32; }
    static const float* ru(nir_pdhg* h) { return h->ru32; }
};

template <>
struct Vec<double> {
    static double* x(nir_pdhg* h) { return h->x64; }
    static double* xb(nir_pdhg* h) { return h->xb64; }
    static double* x0(nir_pdhg* h) { return h->x064; }
    static double* xp(nir_pdhg* h) { return h->xp64; }
    static double* y(nir_pdhg* h) { return h->y64; }
    static double* y0(nir_pdhg* h) { return h->y064; }
    static double* yp(nir_pdhg* h) { return h->yp64; }
    static const double* c(nir_pdhg* h) { return h->c64; }
    static const double* l(nir_pdhg* h) { return h->l64; }
    static const double* u(nir_pdhg* h) { return h->u64; }
    static const double* rl(nir_pdhg* h) { return h->rl64; }
    static const double* ru(nir_pdhg* h) { return h->ru64; }
};

// The layout an orientation's iteration and KKT kernels use (o.lay) as the
// kernels see it, and its scaled values: the CSR's own arrays for the warp
// layout, the padded stream for the CTA layout.
nir::Lay lay_of(const Orient& o) {
    if (o.lay == nir::kLayWarp) return nir::Lay{o.blk, o.nblk, o.cap, o.rp, o.ci};
    const Orient::Cta& L = o.cur();
    return nir::Lay{L.blk, L.nblk, 0, o.rp, L.ci};
}

template <typename TV>
const TV* vals_of(const Orient& o);
template <>
const float* vals_of<float>(const Orient& o) {
    return o.lay == nir::kLayWarp ? o.v32 : o.cur().v32;
}
template <>
const double* vals_of<double>(const Orient& o) {
    return o.lay == nir::kLayWarp ? o.v64 : o.cur().v64;
}

int lay_nblk(const Orient& o) { return o.lay == nir::kLayWarp ? o.nblk : o.cur().nblk; }

// Dynamic shared memory of a kernel over a layout (the warp layout's
// product slices; the CTA layout's shared memory is static).
template <int LAY, typename TA>
constexpr size_t lay_smem() {
    return LAY == nir::kLayWarp ? size_t(nir::warp_smem_bytes<TA>()) : size_t(0);
}

// Persistent grid of a layout kernel: as many CTAs as are resident at once,
// at most one warp per warp row block (warp layout) or one CTA per block
// (CTA layout).  The occupancy query runs once per kernel (outside any
// stream capture).
template <int LAY, typename TA, typename K>
int lay_grid(nir_pdhg* h, K* kernel, int nblk) {
    const size_t smem = lay_smem<LAY, TA>();
    int per = 0;
    for (auto& e : h->occ)
        if (e.fn == (const void*)kernel && e.smem == smem) per = e.per_sm;
    if (per == 0) {
        prefer_carveout(kernel);
        NIR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, nir::kBlock, smem));
        per = std::max(per, 1);
        h->occ.push_back({(const void*)kernel, smem, per});
    }
    const int need = LAY == nir::kLayWarp ? std::max(1, (nblk + nir::kWarps - 1) / nir::kWarps) : std::max(1, nblk);
    return std::min(need, per * h->sms);
}

// Calls f(LP, LD) with the layouts of A' (primal) and A (dual) as
// std::integral_constant values.
template <class F>
void with_lays(const nir_pdhg* h, F&& f) {
    using W = std::integral_constant<int, nir::kLayWarp>;
    using Cc = std::integral_constant<int, nir::kLayCta>;
    const bool pc = h->At.lay == nir::kLayCta, dc = h->A.lay == nir::kLayCta;
    if (pc && dc) f(Cc{}, Cc{});
    else if (pc) f(Cc{}, W{});
    else if (dc) f(W{}, Cc{});
    else f(W{}, W{});
}

constexpr int kCtaCap = 256 * nir::kLayCta;  // nonzeros per block of the CTA layout

// Sets up the chosen layouts (built on first use).
void use_layouts(nir_pdhg* h, const LayChoice& c) {
    for (int t = 0; t < 2; ++t) {
        Orient& o = t ? h->At : h->A;
        const int lay = t ? c.lay_at : c.lay_a, cap = t ? c.cap_at : c.cap_a;
        if (lay == nir::kLayWarp) {
            set_blocks(h, o, cap);
        } else {
            cta_layout(h, o, kCtaCap);
            for (size_t k = 0; k < o.ctas.size(); ++k)
                if (o.ctas[k].cap == kCtaCap) o.it = int(k);
        }
        o.lay = lay;
    }
}

// Copies the scaled values (written by precondition) into the padded
// streams of the orientations that use the CTA layout.
void pad_scaled(nir_pdhg* h) {
    cudaStream_t s = h->stream;
    for (Orient* o : {&h->A, &h->At}) {
        if (o->lay != nir::kLayCta) continue;
        const Orient::Cta& L = o->cur();
        if (L.nblk <= 0 || o->nnz <= 0) continue;
        const unsigned g = unsigned(std::max(1, std::min(L.nblk, 4 * h->sms)));
        nir::k_pad_stream<double><<<g, nir::kBlock, 0, s>>>(L.blk, L.nblk, o->ci, o->v64, nullptr, L.v64);
        nir::k_pad_stream<float><<<g, nir::kBlock, 0, s>>>(L.blk, L.nblk, o->ci, o->v32, nullptr, L.v32);
        NIR_LAUNCHED();
        h->launches += 2;
    }
}

// The two FP64 KKT passes of a check over the layouts in use, at (xp, yp)
// of type TX; returns their grids (the number of partials each wrote).
template <typename TX>
void launch_kkt(nir_pdhg* h, int phase, double* partKR, double* partKC, const TX* xp, const TX* yp, int* gkr,
                int* gkc) {
    cudaStream_t s = h->stream;
    with_lays(h, [&](auto lp, auto ld) {
        constexpr int LP = decltype(lp)::value, LD = decltype(ld)::value;
        *gkr = lay_grid<LD, double>(h, nir::k_kkt_rows<LD, TX>, lay_nblk(h->A));
        *gkc = lay_grid<LP, double>(h, nir::k_kkt_cols<LP, TX>, lay_nblk(h->At));
        nir::KktArgs kr{lay_of(h->A), vals_of<double>(h->A), partKR, h->st, phase};
        nir::k_kkt_rows<LD, TX><<<*gkr, nir::kBlock, lay_smem<LD, double>(), s>>>(kr, xp, yp, h->dr, h->rl, h->ru);
        nir::KktArgs kc{lay_of(h->At), vals_of<double>(h->At), partKC, h->st, phase};
        nir::k_kkt_cols<LP, TX><<<*gkc, nir::kBlock, lay_smem<LP, double>(), s>>>(kc, xp, yp, h->dc, h->c, h->l, h->u);
        NIR_LAUNCHED();
    });
    h->launches += 2;
}

// Occupancy queries of the KKT kernels before any capture.
template <typename TX>
void warm_kkt(nir_pdhg* h) {
    with_lays(h, [&](auto lp, auto ld) {
        constexpr int LP = decltype(lp)::value, LD = decltype(ld)::value;
        lay_grid<LD, double>(h, nir::k_kkt_rows<LD, TX>, lay_nblk(h->A));
        lay_grid<LP, double>(h, nir::k_kkt_cols<LP, TX>, lay_nblk(h->At));
    });
}

struct SolveCfg {
    nir_pdhg_params p;
    int K = 64;
    int halpern = 1;
    int restarts = 1;
    int mixed = 0;
    double bnorm = 0.0, cnorm = 0.0;
    int persistent = 0;    // non-check iterations in one cooperative launch per chunk
    int barrier_test = 0;  // persistent launch whose barrier cannot complete (bounded-wait test)
};

// Optional event timing of the first iteration of a chunk.
struct ChunkTimer {
    cudaEvent_t e[4] = {nullptr, nullptr, nullptr, nullptr};
    bool armed = false;
    int K = 1;
    int prec = 0;  // 0: the timed chunk streams FP32 values, 1: FP64
};

// One launch chunk: K iterations (the last one a check), the KKT passes,
// the controller, the restart copy and the status snapshot.  TV = type of
// the matrix values, TX = type of the iterates, LP / LD = layouts of A' / A.
template <typename TV, typename TX, int LP, int LD>
void launch_fast_chunk_l(nir_pdhg* h, const SolveCfg& cfg, int phase, ChunkTimer* tm) {
    if (tm) tm->prec = (sizeof(TV) == 8) ? 1 : 0;
    cudaStream_t s = h->stream;
    const PartLayout L = part_layout(h);
    const int K = cfg.K;
    const int nbt = lay_nblk(h->At), nba = lay_nblk(h->A);
    const nir::Lay lt = lay_of(h->At), la = lay_of(h->A);
    const TV* valAt = vals_of<TV>(h->At);
    const TV* valA = vals_of<TV>(h->A);
    const size_t sp = lay_smem<LP, TX>(), sd = lay_smem<LD, TX>();
    const int gp1 = lay_grid<LP, TX>(h, nir::k_primal<LP, TV, TX, true>, nbt);
    const int gp0 = lay_grid<LP, TX>(h, nir::k_primal<LP, TV, TX, false>, nbt);
    const int gd1 = lay_grid<LD, TX>(h, nir::k_dual<LD, TV, TX, true>, nba);
    const int gd0 = lay_grid<LD, TX>(h, nir::k_dual<LD, TV, TX, false>, nba);
    int i_first = 0;
    if (cfg.persistent && K > 1) {
        // iterations 0..K-2 in one cooperative launch; the check pair below
        const size_t sc = std::max(sp, sd);
        const int gc = std::min(lay_grid<LP, TX>(h, nir::k_chunk<LP, LD, TV, TX>, nbt),
                                lay_grid<LD, TX>(h, nir::k_chunk<LP, LD, TV, TX>, nba));
        nir::IterArgs ap{lt, L.P, h->st, 0, cfg.halpern, phase, cfg.p.reflection};
        nir::IterArgs ad{la, L.D, h->st, 0, cfg.halpern, phase, cfg.p.reflection};
        nir::ChunkPtrs<TV, TX> v{valAt,          valA,           Vec<TX>::x(h),  Vec<TX>::xb(h), Vec<TX>::xp(h),
                                 Vec<TX>::y(h),  Vec<TX>::yp(h), Vec<TX>::c(h),  Vec<TX>::l(h),  Vec<TX>::u(h),
                                 Vec<TX>::x0(h), Vec<TX>::rl(h), Vec<TX>::ru(h), Vec<TX>::y0(h)};
        // ~1 s of SM clock per wait; 0.1 s and one CTA too many in the test
        nir::GridSync gs{h->gs_count, h->gs_gen, h->gs_err, unsigned(gc) + (cfg.barrier_test ? 1u : 0u),
                         cfg.barrier_test ? 200000000LL : 2000000000LL};
        nir::DevState* st = h->st;
        int i0 = 0, iters = K - 1;
        void* args[] = {&ap, &ad, &v, &i0, &iters, &gs, &st};
        NIR_CUDA(cudaLaunchCooperativeKernel((const void*)nir::k_chunk<LP, LD, TV, TX>, dim3(gc), dim3(nir::kBlock),
                                             args, sc, s));
        h->launches += 1;
        i_first = K - 1;
    }
    for (int i = i_first; i < K; ++i) {
        const bool check = (i == K - 1);
        nir::IterArgs ap{lt, L.P, h->st, i, cfg.halpern, phase, cfg.p.reflection};
        nir::IterArgs ad{la, L.D, h->st, i, cfg.halpern, phase, cfg.p.reflection};
        const bool timed = tm && tm->armed && i == 0 && !cfg.persistent;
        if (timed) NIR_CUDA(cudaEventRecord(tm->e[0], s));
        if (check)
            nir::k_primal<LP, TV, TX, true><<<gp1, nir::kBlock, sp, s>>>(
                ap, valAt, Vec<TX>::y(h), Vec<TX>::x(h), Vec<TX>::xb(h), Vec<TX>::xp(h), Vec<TX>::c(h), Vec<TX>::l(h),
                Vec<TX>::u(h), Vec<TX>::x0(h));
        else
            nir::k_primal<LP, TV, TX, false><<<gp0, nir::kBlock, sp, s>>>(
                ap, valAt, Vec<TX>::y(h), Vec<TX>::x(h), Vec<TX>::xb(h), Vec<TX>::xp(h), Vec<TX>::c(h), Vec<TX>::l(h),
                Vec<TX>::u(h), Vec<TX>::x0(h));
        NIR_LAUNCHED();
        if (timed) NIR_CUDA(cudaEventRecord(tm->e[1], s));
        if (check)
            nir::k_dual<LD, TV, TX, true><<<gd1, nir::kBlock, sd, s>>>(ad, valA, Vec<TX>::xb(h), Vec<TX>::y(h),
                                                                       Vec<TX>::yp(h), Vec<TX>::rl(h), Vec<TX>::ru(h),
                                                                       Vec<TX>::y0(h));
        else
            nir::k_dual<LD, TV, TX, false><<<gd0, nir::kBlock, sd, s>>>(ad, valA, Vec<TX>::xb(h), Vec<TX>::y(h),
                                                                        Vec<TX>::yp(h), Vec<TX>::rl(h), Vec<TX>::ru(h),
                                                                        Vec<TX>::y0(h));
        NIR_LAUNCHED();
        if (timed) NIR_CUDA(cudaEventRecord(tm->e[2], s));
        h->launches += 2;
    }
    int gkr = 0, gkc = 0;
    launch_kkt<TX>(h, phase, L.KR, L.KC, Vec<TX>::xp(h), Vec<TX>::yp(h), &gkr, &gkc);
    h->launches -= 2;  // counted with the chunk below
    nir::CtlArgs ca;
    ca.partP = L.P;
    ca.partD = L.D;
    ca.partKR = L.KR;
    ca.partKC = L.KC;
    ca.nP = gp1;
    ca.nD = gd1;
    ca.nKR = gkr;
    ca.nKC = gkc;
    ca.offset = h->offset;
    ca.tol = cfg.p.tol;
    ca.feas_tol = cfg.p.feas_tol;
    ca.K = K;
    ca.restarts_on = cfg.restarts;
    ca.mixed = (cfg.mixed && phase == 0) ? 1 : 0;
    ca.phase = phase;
    ca.suff = cfg.p.restart_sufficient;
    ca.nec = cfg.p.restart_necessary;
    ca.art = cfg.p.restart_artificial;
    ca.theta = cfg.p.primal_weight_smoothing;
    ca.polish_stall = cfg.p.polish_stall_checks;
    ca.polish_switch = cfg.p.polish_switch_kkt;
    ca.anchor_at_restart = cfg.p.restart_anchor ? 1 : 0;
    ca.weight_decades = cfg.p.primal_weight_decades;
    ca.hist = h->hist;
    nir::k_control<<<1, nir::kBlock, 0, s>>>(ca, h->st);
    NIR_LAUNCHED();
    const int nm = std::max(h->n, h->m);
    nir::k_apply_restart<TX><<<grid_for(nm), nir::kBlock, 0, s>>>(h->n, h->m, h->st, phase, Vec<TX>::x(h),
                                                                   Vec<TX>::x0(h), Vec<TX>::xp(h), Vec<TX>::y(h),
                                                                   Vec<TX>::y0(h), Vec<TX>::yp(h));
    NIR_LAUNCHED();
    nir::k_snap<<<1, 32, 0, s>>>(h->st, h->snap.ring, h->snap.d_seq);
    NIR_LAUNCHED();
    if (tm && tm->armed) NIR_CUDA(cudaEventRecord(tm->e[3], s));
    h->launches += 5;
}

template <typename TV, typename TX>
void launch_fast_chunk(nir_pdhg* h, const SolveCfg& cfg, int phase, ChunkTimer* tm) {
    with_lays(h, [&](auto lp, auto ld) {
        launch_fast_chunk_l<TV, TX, decltype(lp)::value, decltype(ld)::value>(h, cfg, phase, tm);
    });
}

// Runs the occupancy queries of a chunk's kernels before any capture.
template <typename TV, typename TX>
void warm_cfgs(nir_pdhg* h) {
    with_lays(h, [&](auto lp, auto ld) {
        constexpr int LP = decltype(lp)::value, LD = decltype(ld)::value;
        const int nbt = lay_nblk(h->At), nba = lay_nblk(h->A);
        lay_grid<LP, TX>(h, nir::k_primal<LP, TV, TX, true>, nbt);
        lay_grid<LP, TX>(h, nir::k_primal<LP, TV, TX, false>, nbt);
        lay_grid<LD, TX>(h, nir::k_dual<LD, TV, TX, true>, nba);
        lay_grid<LD, TX>(h, nir::k_dual<LD, TV, TX, false>, nba);
        lay_grid<LP, TX>(h, nir::k_chunk<LP, LD, TV, TX>, nbt);
        lay_grid<LD, TX>(h, nir::k_chunk<LP, LD, TV, TX>, nba);
    });
    warm_kkt<TX>(h);
}

// Identity of everything a captured chunk bakes into its kernel arguments
// (FNV-1a over the values), so a graph is only replayed for the same ones.
struct KeyHash {
    unsigned long long h = 1469598103934665603ULL;
    template <typename V>
    KeyHash& add(const V& v) {
        const unsigned char* p = reinterpret_cast<const unsigned char*>(&v);
        for (size_t i = 0; i < sizeof(V); ++i) {
            h ^= p[i];
            h *= 1099511628211ULL;
        }
        return *this;
    }
};

// prec: 0 = FP32 values and iterates, 1 = FP32 values with FP64 iterates,
// 2 = FP64 values and iterates.
unsigned long long chunk_key(const nir_pdhg* h, const SolveCfg& c, int phase, int prec) {
    KeyHash k;
    k.add(phase).add(prec).add(c.K).add(c.halpern).add(c.restarts).add(c.mixed);
    k.add(c.p.reflection).add(c.p.restart_sufficient).add(c.p.restart_necessary).add(c.p.restart_artificial);
    k.add(c.p.primal_weight_smoothing).add(c.p.polish_stall_checks).add(c.p.polish_switch_kkt).add(c.p.tol);
    k.add(c.p.feas_tol).add(c.p.restart_anchor).add(c.p.primal_weight_decades).add(c.p.polish_fresh).add(h->offset).add(h->part).add(h->hist);
    // the layouts of a single LP (the batch keys its own)
    if (h->A.lay >= 0) k.add(h->A.lay).add(lay_of(h->A).blk).add(lay_of(h->A).cap);
    if (h->At.lay >= 0) k.add(h->At.lay).add(lay_of(h->At).blk).add(lay_of(h->At).cap);
    k.add(c.persistent).add(c.barrier_test);
    return k.h;
}

void precondition(nir_pdhg* h, const nir_pdhg_params& p, bool enable);
double rhs_norm(const nir_pdhg* h);
double norm2(const std::vector<double>& v);

// Relative-KKT probe of the reference loop: norms of the original b and c.
struct RefProbe {
    double bnorm, cnorm, tol;
};

void launch_ref_chunk(nir_pdhg* h, int K, const RefProbe* probe) {
    cudaStream_t s = h->stream;
    const PartLayout L = part_layout(h);
    const unsigned gm = grid_for(h->m), gn = grid_for(h->n);
    for (int i = 0; i < K; ++i) {
        nir::k_ref_primal<<<std::max(gn, 1u), nir::kBlock, 0, s>>>(h->n, h->At.rp, h->At.ci, h->At.v_orig, h->y64, h->c,
                                                                    h->l, h->u, h->x64, h->xb64, h->st, i);
        NIR_LAUNCHED();
        nir::k_ref_dual<<<std::max(gm, 1u), nir::kBlock, 0, s>>>(h->m, h->A.rp, h->A.ci, h->A.v_orig, h->xb64, h->rl,
                                                                  h->ru, h->y64, L.misc, h->st, i);
        NIR_LAUNCHED();
        nir::k_ref_stop<<<1, nir::kBlock, 0, s>>>(L.misc, std::max<int>(gm, 1), h->st, i, K);
        NIR_LAUNCHED();
        h->launches += 3;
    }
    if (probe) {
        // KKT of (x, y) on the unscaled matrix (dr = dc = 1): reads only
        int gkr = 0, gkc = 0;
        launch_kkt<double>(h, 0, L.KR, L.KC, h->x64, h->y64, &gkr, &gkc);
        nir::k_ref_probe<<<1, nir::kBlock, 0, s>>>(L.KR, gkr, L.KC, gkc, probe->bnorm, probe->cnorm, h->offset,
                                                   probe->tol, h->st);
        NIR_LAUNCHED();
        h->launches += 1;
    }
    nir::k_snap<<<1, 32, 0, s>>>(h->st, h->snap.ring, h->snap.d_seq);
    NIR_LAUNCHED();
    h->launches += 1;
}

// Captures (once) and returns the graph for a chunk kind.
template <class F>
cudaGraphExec_t chunk_graph(nir_pdhg* h, int slot, unsigned long long key, F&& launch) {
    ChunkGraph& g = h->graphs[slot];
    if (g.ge && g.valid && g.key == key) return g.ge;
    if (g.ge) {
        cudaGraphExecDestroy(g.ge);
        g.ge = nullptr;
    }
    if (g.g) {
        cudaGraphDestroy(g.g);
        g.g = nullptr;
    }
    NIR_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    int before = h->launches;
    try {
        launch();
    } catch (...) {
        cudaGraph_t tmp;
        cudaStreamEndCapture(h->stream, &tmp);
        if (tmp) cudaGraphDestroy(tmp);
        throw;
    }
    h->launches = before;  // counted when replayed
    NIR_CUDA(cudaStreamEndCapture(h->stream, &g.g));
    NIR_CUDA(cudaGraphInstantiate(&g.ge, g.g, 0));
    g.key = key;
    g.valid = true;
    return g.ge;
}

struct LoopResult {
    nir::HostSnap last{};
    bool stopped_by_host = false;
    double t_switch = 0.0;
};

int launches_per_chunk(int K, bool ref) { return ref ? 3 * K + 1 : 2 * K + 5; }

// Runs chunks until the device reports done, the phase changes, or the
// caller's poll / time limit stops it.  Keeps `depth` chunks in flight.
template <class F>
LoopResult run_chunks(nir_pdhg* h, const nir_pdhg_params& p, int (*poll)(void*), void* ctx, double t_start, int phase,
                      int per_chunk, F&& launch_one, ChunkTimer* tm) {
    const int depth = tm ? 1 : 3;  // timed chunks run one at a time
    cudaEvent_t ev[3];
    for (auto& e : ev) NIR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    LoopResult R;
    long long launched = 0, completed = 0;
    bool stop_launch = false;
    long long seq0 = 0;
    {
        // sequence number of the snapshot before this loop
        long long s = 0;
        d2h(h, &s, h->snap.d_seq, sizeof(long long));
        seq0 = s;
    }
    try {
        for (;;) {
            while (!stop_launch && launched - completed < depth) {
                launch_one();
                h->launches += per_chunk;
                NIR_CUDA(cudaEventRecord(ev[launched % depth], h->stream));
                ++launched;
            }
            if (completed == launched) break;
            NIR_CUDA(cudaEventSynchronize(ev[completed % depth]));
            ++completed;
            if (tm && tm->armed) {
                float a = 0, b = 0, c = 0;
                if (cudaEventElapsedTime(&a, tm->e[0], tm->e[1]) == cudaSuccess &&
                    cudaEventElapsedTime(&b, tm->e[1], tm->e[2]) == cudaSuccess &&
                    cudaEventElapsedTime(&c, tm->e[0], tm->e[3]) == cudaSuccess) {
                    const int q = tm->prec;
                    h->ktime.primal_us[q] += 1000.0 * a;
                    h->ktime.dual_us[q] += 1000.0 * b;
                    h->ktime.iter_us[q] += 1000.0 * c / std::max(1, tm->K);
                    h->ktime.samples[q] += 1;
                }
            }
            const nir::HostSnap snap = h->snap.ring[(seq0 + completed) % nir::kSnapRing];
            R.last = snap;
            if (stop_launch) continue;
            if (snap.done || snap.phase != phase) {
                stop_launch = true;
                continue;
            }
            bool expire = (poll && poll(ctx) != 0);
            if (p.time_limit > 0.0 && now_sec() - t_start >= p.time_limit) expire = true;
            if (expire) {
                R.stopped_by_host = true;
                stop_launch = true;
            }
        }
        NIR_CUDA(cudaStreamSynchronize(h->stream));
    } catch (...) {
        for (auto& e : ev) cudaEventDestroy(e);
        throw;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    return R;
}

LayChoice default_layouts(const nir_pdhg* h);

double host_objective(const nir_pdhg* h, const std::vector<double>& x) {
    DD s;
    s.hi = h->offset;
    for (int j = 0; j < h->n; ++j)
        if (h->h_c[j] != 0.0 && x[j] != 0.0) s = dd_add_prod(s, h->h_c[j], x[j]);
    return s.hi + s.lo;
}

void fill_info_common(nir_pdhg* h, const nir::DevState& st, nir_pdhg_info* info) {
    info->restarts = st.restarts;
    info->rel_kkt = st.kkt;
    info->rel_primal = st.kp;
    info->rel_dual = st.kd;
    info->rel_gap = st.kg;
    info->max_rel_row_viol = st.max_rel_row;
    info->primal_weight = st.omega;
    info->step_size = st.eta;
    (void)h;
}

// ---------------------------------------------------------------- reference algorithm

int solve_reference(nir_pdhg* h, const nir_pdhg_params& p, int (*poll)(void*), void* ctx, double* x_out, double* y_out,
                    nir_pdhg_info* info) {
    cudaStream_t s = h->stream;
    const double t0 = now_sec();
    ensure_partials(h);
    const int n = h->n, m = h->m;
    nir::DevState st0{};
    st0.max_iters = p.max_iters;
    st0.best_kkt = INFINITY;
    st0.kkt = st0.kp = st0.kd = st0.kg = st0.max_rel_row = NAN;
    st0.probe_hit = -1;
    NIR_CUDA(cudaMemcpyAsync(h->st, &st0, sizeof(st0), cudaMemcpyHostToDevice, s));
    // optional relative-KKT probe every chunk (tol > 0): unscaled FP64 copy
    // of the values and warp row blocks for the KKT kernels
    const bool probing = p.tol > 0.0;
    RefProbe probe{0.0, 0.0, p.tol};
    if (probing) {
        use_layouts(h, default_layouts(h));
        precondition(h, p, false);
        pad_scaled(h);
        warm_kkt<double>(h);
        probe.bnorm = rhs_norm(h);
        probe.cnorm = norm2(h->h_c);
    }
    // power iteration, src/gpu/pdhg_solver.hpp:33-45
    nir::k_fill<<<grid_for(n), nir::kBlock, 0, s>>>(n, 1.0, h->tmp_n);
    NIR_LAUNCHED();
    for (int r = 0; r < 12; ++r) {
        nir::k_ref_spmv<<<std::max(grid_for(m), 1u), nir::kBlock, 0, s>>>(m, h->A.rp, h->A.ci, h->A.v_orig, h->tmp_n, h->tmp_m);
        nir::k_ref_spmv<<<std::max(grid_for(n), 1u), nir::kBlock, 0, s>>>(n, h->At.rp, h->At.ci, h->At.v_orig, h->tmp_m, h->tmp_n);
        nir::k_ref_norm<<<1, 32, 0, s>>>(n, h->tmp_n, h->st);
        nir::k_ref_div<<<std::max(grid_for(n), 1u), nir::kBlock, 0, s>>>(n, h->tmp_n, h->st);
        NIR_LAUNCHED();
        h->launches += 4;
    }
    nir::k_ref_steps<<<1, 32, 0, s>>>(h->st);
    nir::k_ref_init<<<std::max(grid_for(std::max(n, m)), 1u), nir::kBlock, 0, s>>>(n, m, h->l, h->u, h->x64, h->y64);
    NIR_LAUNCHED();
    h->launches += 3;
    const int K = 32;
    const double t_setup = now_sec();
    [[maybe_unused]] LoopResult R;
    if (p.max_iters > 0) {
        const RefProbe* pr = probing ? &probe : nullptr;
        auto launch = [&]() { launch_ref_chunk(h, K, pr); };
        if (p.use_graphs) {
            KeyHash key;
            key.add(1000).add(probing).add(probe.bnorm).add(probe.cnorm).add(probe.tol).add(h->offset);
            if (probing) key.add(lay_of(h->A).blk).add(lay_of(h->At).blk).add(h->A.lay).add(h->At.lay);
            key.add(h->part);
            cudaGraphExec_t ge = chunk_graph(h, 0, key.h, launch);
            const int per = launches_per_chunk(K, true) + (probing ? 3 : 0);
            R = run_chunks(h, p, poll, ctx, t0, 0, per, [&]() { NIR_CUDA(cudaGraphLaunch(ge, s)); }, nullptr);
        } else {
            R = run_chunks(h, p, poll, ctx, t0, 0, 0, launch, nullptr);
        }
    }
    nir::DevState st;
    d2h(h, &st, h->st, sizeof(st));
    std::vector<double> x(n), y(m);
    d2h(h, x.data(), h->x64, n * sizeof(double));
    d2h(h, y.data(), h->y64, m * sizeof(double));
    if (x_out) std::memcpy(x_out, x.data(), n * sizeof(double));
    if (y_out) std::memcpy(y_out, y.data(), m * sizeof(double));
    h->last_x = h->x64;
    int status;
    if (st.ref_stopped) status = NIR_STATUS_OPTIMAL;
    else if (st.done) status = NIR_STATUS_ITERATION_LIMIT;
    else status = NIR_STATUS_TIME_LIMIT;
    if (p.max_iters <= 0) status = NIR_STATUS_ITERATION_LIMIT;
    info->status = status;
    info->iterations = st.done ? st.ref_iterations : st.iter;
    info->iterations_fp64 = info->iterations;
    info->objective = host_objective(h, x);
    info->step_size = st.tau;
    info->primal_weight = 1.0;
    info->setup_seconds = t_setup - t0;
    info->solve_seconds = now_sec() - t_setup;
    // probed KKT of the last full chunk (NaN without the probe)
    info->rel_kkt = st.kkt;
    info->rel_primal = st.kp;
    info->rel_dual = st.kd;
    info->rel_gap = st.kg;
    info->max_rel_row_viol = st.max_rel_row;
    info->iterations_to_tol = st.probe_hit;
    (void)R;
    return status;
}

// ---------------------------------------------------------------- PDHG / PDLP

void precondition(nir_pdhg* h, const nir_pdhg_params& p, bool enable) {
    cudaStream_t s = h->stream;
    const int n = h->n, m = h->m;
    auto& sc = h->scaled;
    if (sc.valid && sc.enabled == enable && (!enable || (sc.ruiz == p.ruiz_iters && sc.pc == p.pock_chambolle))) {
        // the matrix scaling of the last solve holds: scale the vectors only
        nir::k_scale_vectors<<<std::max(grid_for(std::max(n, m)), 1u), nir::kBlock, 0, s>>>(
            n, m, h->c, h->l, h->u, h->rl, h->ru, h->dc, h->dr, h->c64, h->l64, h->u64, h->rl64, h->ru64, h->c32,
            h->l32, h->u32, h->rl32, h->ru32);
        NIR_LAUNCHED();
        h->launches += 1;
        return;
    }
    sc = nir_pdhg::ScaleState{};
    nir::k_fill<<<grid_for(m), nir::kBlock, 0, s>>>(m, 1.0, h->dr);
    nir::k_fill<<<grid_for(n), nir::kBlock, 0, s>>>(n, 1.0, h->dc);
    NIR_LAUNCHED();
    if (enable) {
        const unsigned gwm = grid_for((long long)m * 32), gwn = grid_for((long long)n * 32);
        for (int it = 0; it < p.ruiz_iters + (p.pock_chambolle ? 1 : 0); ++it) {
            const int mode = it < p.ruiz_iters ? 0 : 1;  // 0 = l-inf (Ruiz), 1 = l1 (Pock-Chambolle)
            nir::k_row_stat<<<std::max(gwm, 1u), nir::kBlock, 0, s>>>(m, h->A.rp, h->A.ci, h->A.v_orig, h->dr, h->dc, mode,
                                                                     h->tmp_m);
            nir::k_row_stat<<<std::max(gwn, 1u), nir::kBlock, 0, s>>>(n, h->At.rp, h->At.ci, h->At.v_orig, h->dc, h->dr,
                                                                     mode, h->tmp_n);
            nir::k_apply_stat<<<grid_for(m), nir::kBlock, 0, s>>>(m, h->tmp_m, h->dr);
            nir::k_apply_stat<<<grid_for(n), nir::kBlock, 0, s>>>(n, h->tmp_n, h->dc);
            NIR_LAUNCHED();
            h->launches += 4;
        }
        nir::k_round_pow2<<<grid_for(m), nir::kBlock, 0, s>>>(m, h->dr);
        nir::k_round_pow2<<<grid_for(n), nir::kBlock, 0, s>>>(n, h->dc);
        NIR_LAUNCHED();
    }
    const unsigned gwm = grid_for((long long)m * 32), gwn = grid_for((long long)n * 32);
    nir::k_scale_values<<<std::max(gwm, 1u), nir::kBlock, 0, s>>>(m, h->A.rp, h->A.ci, h->A.v_orig, h->dr, h->dc, 1,
                                                                 h->A.v64, h->A.v32);
    nir::k_scale_values<<<std::max(gwn, 1u), nir::kBlock, 0, s>>>(n, h->At.rp, h->At.ci, h->At.v_orig, h->dc, h->dr, 0,
                                                                 h->At.v64, h->At.v32);
    nir::k_scale_vectors<<<std::max(grid_for(std::max(n, m)), 1u), nir::kBlock, 0, s>>>(
        n, m, h->c, h->l, h->u, h->rl, h->ru, h->dc, h->dr, h->c64, h->l64, h->u64, h->rl64, h->ru64, h->c32, h->l32,
        h->u32, h->rl32, h->ru32);
    NIR_LAUNCHED();
    h->launches += 7;
    sc.valid = true;
    sc.enabled = enable;
    sc.ruiz = p.ruiz_iters;
    sc.pc = p.pock_chambolle;
}

// ||A_scaled||_2 by power iteration on A'A (FP64, deterministic), kept
// with the scaling it was computed for.
double power_norm(nir_pdhg* h, int rounds) {
    auto& sc = h->scaled;
    if (sc.valid && sc.norm_valid && sc.power_iters == rounds) return sc.norm;
    cudaStream_t s = h->stream;
    const int n = h->n, m = h->m;
    const PartLayout L = part_layout(h);
    const unsigned gwm = grid_for((long long)m * 32), gwn = grid_for((long long)n * 32);
    nir::k_power_start<<<std::max(grid_for(n), 1u), nir::kBlock, 0, s>>>(n, h->tmp_n);
    nir::k_sumsq_partials<<<std::max(grid_for(n), 1u), nir::kBlock, 0, s>>>(n, h->tmp_n, L.misc);
    nir::k_norm_finalize<<<1, nir::kBlock, 0, s>>>(L.misc, std::max<int>(grid_for(n), 1), h->st);
    nir::k_scale_by_inv_norm<<<std::max(grid_for(n), 1u), nir::kBlock, 0, s>>>(n, h->tmp_n, h->st);
    NIR_LAUNCHED();
    for (int r = 0; r < rounds; ++r) {
        nir::k_spmv_warp64<<<std::max(gwm, 1u), nir::kBlock, 0, s>>>(m, h->A.rp, h->A.ci, h->A.v64, h->tmp_n, h->tmp_m);
        nir::k_spmv_warp64<<<std::max(gwn, 1u), nir::kBlock, 0, s>>>(n, h->At.rp, h->At.ci, h->At.v64, h->tmp_m, h->tmp_n);
        nir::k_sumsq_partials<<<std::max(grid_for(n), 1u), nir::kBlock, 0, s>>>(n, h->tmp_n, L.misc);
        nir::k_norm_finalize<<<1, nir::kBlock, 0, s>>>(L.misc, std::max<int>(grid_for(n), 1), h->st);
        nir::k_scale_by_inv_norm<<<std::max(grid_for(n), 1u), nir::kBlock, 0, s>>>(n, h->tmp_n, h->st);
        NIR_LAUNCHED();
        h->launches += 5;
    }
    nir::DevState st;
    NIR_CUDA(cudaMemcpyAsync(&st, h->st, sizeof(st), cudaMemcpyDeviceToHost, s));
    NIR_CUDA(cudaStreamSynchronize(s));
    const double norm = std::sqrt(st.ref_norm_est);  // ||A'A u|| ~ sigma_max^2 for unit u
    if (sc.valid) {
        sc.norm_valid = true;
        sc.power_iters = rounds;
        sc.norm = norm;
    }
    return norm;
}

double norm2(const std::vector<double>& v) {
    DD s;
    for (double a : v) s = dd_add_prod(s, a, a);
    return std::sqrt(s.hi + s.lo);
}

double rhs_norm(const nir_pdhg* h) {
    DD s;
    for (int i = 0; i < h->m; ++i) {
        double b = 0.0;
        if (std::isfinite(h->h_rl[i])) b = std::fabs(h->h_rl[i]);
        if (std::isfinite(h->h_ru[i])) b = std::max(b, std::fabs(h->h_ru[i]));
        s = dd_add_prod(s, b, b);
    }
    return std::sqrt(s.hi + s.lo);
}

// Layouts without timing: warp row blocks, the capacity by size.
LayChoice default_layouts(const nir_pdhg* h) {
    LayChoice c;
    c.cap_a = c.cap_at = auto_cap(h->nnz, std::max(h->m, h->n));
    return c;
}

// The autotuner: picks, for each orientation separately, the layout of its
// SpMV (warp row blocks of 32, 64, 128 or 256 nonzeros, or CTA blocks of
// 1024) by timing the plain SpMV of each candidate in the value and iterate
// precision the solve starts in, on scratch vectors.  The choice is cached
// per handle and precision.
template <typename TV, typename TX>
float time_candidate(nir_pdhg* h, Orient& o, int lay, int cap) {
    cudaStream_t s = h->stream;
    const bool tr = &o == &h->At;
    const TX* in = reinterpret_cast<const TX*>(std::is_same<TX, float>::value ? (tr ? (void*)h->tmp_m32 : (void*)h->tmp_n32)
                                                                              : (tr ? (void*)h->tmp_m : (void*)h->tmp_n));
    TX* out = reinterpret_cast<TX*>(tr ? h->out_x : h->out_y);
    cudaEvent_t a, b;
    NIR_CUDA(cudaEventCreate(&a));
    NIR_CUDA(cudaEventCreate(&b));
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        NIR_CUDA(cudaEventRecord(a, s));
        if (lay == nir::kLayWarp) {
            set_blocks(h, o, cap);
            auto* kern = nir::k_spmv_adaptive<TX, TV, TX>;
            const int g = lay_grid<nir::kLayWarp, TX>(h, kern, o.nblk);
            const TV* v = std::is_same<TV, float>::value ? (const TV*)o.v32 : (const TV*)o.v64;
            kern<<<g, nir::kBlock, lay_smem<nir::kLayWarp, TX>(), s>>>(o.blk, o.nblk, cap, o.rp, o.ci, v, in, out);
        } else {
            Orient::Cta& L = cta_layout(h, o, kCtaCap);
            auto* kern = nir::k_spmv_cta<TX, TV, TX, nir::kLayCta>;
            const int g = lay_grid<nir::kLayCta, TX>(h, kern, L.nblk);
            const TV* v = std::is_same<TV, float>::value ? (const TV*)L.v32 : (const TV*)L.v64;
            kern<<<g, nir::kBlock, 0, s>>>(L.blk, L.nblk, o.rp, L.ci, v, in, out);
        }
        NIR_LAUNCHED();
        NIR_CUDA(cudaEventRecord(b, s));
        NIR_CUDA(cudaEventSynchronize(b));
        float ms = 0.0f;
        NIR_CUDA(cudaEventElapsedTime(&ms, a, b));
        if (rep > 0) best = std::min(best, ms);  // the first launch warms up
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return best;
}

// The tuned layouts depend only on the sparsity structure, the precision
// and the device, and they fix the per-row summation order: one
// process-wide table keyed by those makes every handle on the same matrix
// use the same layouts (bit-identical results across handles).
std::mutex g_tune_mu;
std::vector<std::pair<unsigned long long, LayChoice>> g_tuned;

unsigned long long structure_key(const nir_pdhg* h, int prec) {
    KeyHash k;
    k.add(h->device).add(h->m).add(h->n).add(h->nnz).add(prec).add(3);  // 3: warp or CTA per orientation
    for (int v : h->A.h_rp) k.add(v);
    for (int v : h->At.h_rp) k.add(v);
    return k.h;
}

LayChoice pick_layouts(nir_pdhg* h, const nir_pdhg_params& p) {
    if (p.spmv_block_nnz > 0) {
        LayChoice c;
        if (p.spmv_block_nnz == kCtaCap) {
            c.lay_a = c.lay_at = nir::kLayCta;
            c.cap_a = c.cap_at = kCtaCap;
        } else if (p.spmv_block_nnz == 32 || p.spmv_block_nnz == 64 || p.spmv_block_nnz == 128 ||
                   p.spmv_block_nnz == 256) {
            c.cap_a = c.cap_at = p.spmv_block_nnz;
        } else {
            throw std::invalid_argument("spmv_block_nnz must be 0, 32, 64, 128, 256 (warp row blocks) or 1024 "
                                        "(CTA blocks)");
        }
        return c;
    }
    const int prec = p.precision;  // FP64 starts with FP64 values, MIXED and FP32 with FP32 values
    if (h->tuned_ok[prec]) return h->tuned[prec];
    const unsigned long long key = structure_key(h, prec);
    {
        std::lock_guard<std::mutex> g(g_tune_mu);
        for (auto& e : g_tuned)
            if (e.first == key) {
                h->tuned[prec] = e.second;
                h->tuned_ok[prec] = true;
                return e.second;
            }
    }
    // the scratch inputs only need to hold finite values
    nir::k_fill<<<grid_for(h->n), nir::kBlock, 0, h->stream>>>(h->n, 0.5, h->tmp_n);
    nir::k_fill<<<grid_for(h->m), nir::kBlock, 0, h->stream>>>(h->m, 0.5, h->tmp_m);
    nir::k_to_float<<<grid_for(h->n), nir::kBlock, 0, h->stream>>>(h->n, h->tmp_n, h->tmp_n32);
    nir::k_to_float<<<grid_for(h->m), nir::kBlock, 0, h->stream>>>(h->m, h->tmp_m, h->tmp_m32);
    NIR_LAUNCHED();
    LayChoice c;
    for (int t = 0; t < 2; ++t) {
        Orient& o = t ? h->At : h->A;
        float best = 1e30f;
        int lay = nir::kLayWarp, cap = auto_cap(h->nnz, o.rows);
        auto consider = [&](int l, int k) {
            float ms;
            if (prec == NIR_PREC_FP64) ms = time_candidate<double, double>(h, o, l, k);
            else if (prec == NIR_PREC_MIXED) ms = time_candidate<float, double>(h, o, l, k);
            else ms = time_candidate<float, float>(h, o, l, k);
            if (ms <= best * 1.02f) {  // near-ties go to the later candidate (larger blocks)
                best = std::min(best, ms);
                lay = l;
                cap = k;
            }
        };
        for (int k : {32, 64, 128, 256}) consider(nir::kLayWarp, k);
        consider(nir::kLayCta, kCtaCap);
        if (t) {
            c.lay_at = lay;
            c.cap_at = cap;
        } else {
            c.lay_a = lay;
            c.cap_a = cap;
        }
    }
    h->tuned[prec] = c;
    h->tuned_ok[prec] = true;
    std::lock_guard<std::mutex> g(g_tune_mu);
    g_tuned.emplace_back(key, c);
    return c;
}

int solve_fast(nir_pdhg* h, const nir_pdhg_params& p, int (*poll)(void*), void* ctx, double* x_out, double* y_out,
               nir_pdhg_info* info) {
    cudaStream_t s = h->stream;
    const double t0 = now_sec();
    const int n = h->n, m = h->m;
    const bool pdlp = p.algorithm == NIR_ALGO_PDLP;
    use_layouts(h, pick_layouts(h, p));
    ensure_partials(h);
    // value / iterate precision of each phase: FP64 (double, double); MIXED
    // (float, double) then the FP64 polish; FP32 (float, float)
    if (p.precision == NIR_PREC_FP32) warm_cfgs<float, float>(h);
    if (p.precision == NIR_PREC_MIXED) warm_cfgs<float, double>(h);
    if (p.precision != NIR_PREC_FP32) warm_cfgs<double, double>(h);
    SolveCfg cfg;
    cfg.p = p;
    cfg.K = std::max(1, p.check_every);
    cfg.halpern = pdlp ? 1 : 0;
    cfg.restarts = pdlp ? 1 : 0;
    cfg.mixed = (p.precision == NIR_PREC_MIXED) ? 1 : 0;
    {
        // persistent chunks on request (not while profiling, whose per-kernel
        // events need the two-kernel path)
        int coop = 0;
        NIR_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, h->device));
        const bool want = p.persistent == 1 || p.persistent == 2;
        if (want && !coop) throw std::invalid_argument("persistent chunks need cooperative launch support");
        cfg.persistent = (want && coop && !h->profiling) ? 1 : 0;
        cfg.barrier_test = (cfg.persistent && p.persistent == 2) ? 1 : 0;
        if (cfg.persistent) {
            NIR_CUDA(cudaMemsetAsync(h->gs_count, 0, sizeof(unsigned), s));
            NIR_CUDA(cudaMemsetAsync(h->gs_gen, 0, sizeof(unsigned), s));
            NIR_CUDA(cudaMemsetAsync(h->gs_err, 0, sizeof(int), s));
        }
    }
    cfg.bnorm = rhs_norm(h);
    cfg.cnorm = norm2(h->h_c);
    h->ktime = nir_pdhg_kernel_time{};

    NIR_CUDA(cudaMemsetAsync(h->hist, 0, sizeof(double) * 8 * nir::kHist, s));
    precondition(h, p, pdlp && (p.ruiz_iters > 0 || p.pock_chambolle));
    pad_scaled(h);
    nir::DevState st0{};
    st0.max_iters = p.max_iters;
    st0.best_kkt = INFINITY;
    st0.bnorm = cfg.bnorm;
    st0.cnorm = cfg.cnorm;
    double eta, omega;
    if (pdlp) {
        const double sig = power_norm(h, std::max(1, p.power_iters));
        eta = p.step_factor / std::max(sig, 1e-30);
        // primal weight: ||c^|| / ||b^|| in the scaled space
        std::vector<double> dc(n), dr(m);
        d2h(h, dc.data(), h->dc, n * sizeof(double));
        d2h(h, dr.data(), h->dr, m * sizeof(double));
        DD cs, bs;
        for (int j = 0; j < n; ++j) cs = dd_add_prod(cs, h->h_c[j] * dc[j], h->h_c[j] * dc[j]);
        for (int i = 0; i < m; ++i) {
            double b = 0.0;
            if (std::isfinite(h->h_rl[i])) b = std::fabs(h->h_rl[i]);
            if (std::isfinite(h->h_ru[i])) b = std::max(b, std::fabs(h->h_ru[i]));
            b *= dr[i];
            bs = dd_add_prod(bs, b, b);
        }
        const double cn = std::sqrt(cs.hi + cs.lo), bn = std::sqrt(bs.hi + bs.lo);
        omega = (cn > 1e-10 && bn > 1e-10) ? cn / bn : 1.0;
        if (p.omega_init > 0.0) omega = p.omega_init;
        st0.eta = eta;
        st0.omega = omega;
        st0.log_omega0 = std::log(omega);
        st0.tau = eta / omega;
        st0.sigma = eta * omega;
    } else {
        // plain PDHG: the reference's fixed steps from its own power iteration
        NIR_CUDA(cudaMemcpyAsync(h->st, &st0, sizeof(st0), cudaMemcpyHostToDevice, s));
        nir::k_fill<<<std::max(grid_for(n), 1u), nir::kBlock, 0, s>>>(n, 1.0, h->tmp_n);
        for (int r = 0; r < 12; ++r) {
            nir::k_ref_spmv<<<std::max(grid_for(m), 1u), nir::kBlock, 0, s>>>(m, h->A.rp, h->A.ci, h->A.v_orig, h->tmp_n, h->tmp_m);
            nir::k_ref_spmv<<<std::max(grid_for(n), 1u), nir::kBlock, 0, s>>>(n, h->At.rp, h->At.ci, h->At.v_orig, h->tmp_m, h->tmp_n);
            nir::k_ref_norm<<<1, 32, 0, s>>>(n, h->tmp_n, h->st);
            nir::k_ref_div<<<std::max(grid_for(n), 1u), nir::kBlock, 0, s>>>(n, h->tmp_n, h->st);
        }
        nir::k_ref_steps<<<1, 32, 0, s>>>(h->st);
        NIR_LAUNCHED();
        nir::DevState tmp;
        NIR_CUDA(cudaMemcpyAsync(&tmp, h->st, sizeof(tmp), cudaMemcpyDeviceToHost, s));
        NIR_CUDA(cudaStreamSynchronize(s));
        eta = tmp.tau;
        omega = 1.0;
        st0.eta = eta;
        st0.omega = 1.0;
        st0.tau = eta;
        st0.sigma = eta;
    }
    NIR_CUDA(cudaMemcpyAsync(h->st, &st0, sizeof(st0), cudaMemcpyHostToDevice, s));
    // starting point
    double* d_xin = nullptr;
    double* d_yin = nullptr;
    // host or device memory (a device-resident start is copied on the device)
    if (p.x_init) {
        NIR_CUDA(cudaMemcpyAsync(h->out_x, p.x_init, n * sizeof(double), cudaMemcpyDefault, s));
        d_xin = h->out_x;
    }
    if (p.y_init) {
        NIR_CUDA(cudaMemcpyAsync(h->out_y, p.y_init, m * sizeof(double), cudaMemcpyDefault, s));
        d_yin = h->out_y;
    }
    if (!pdlp && !p.x_init) {
        // the reference's box-midpoint start (dr = dc = 1 here)
        nir::k_ref_init<<<std::max(grid_for(std::max(n, m)), 1u), nir::kBlock, 0, s>>>(n, m, h->l, h->u, h->out_x, h->out_y);
        d_xin = h->out_x;
        d_yin = h->out_y;
    }
    nir::k_init_iterates<<<std::max(grid_for(std::max(n, m)), 1u), nir::kBlock, 0, s>>>(
        n, m, d_xin, d_yin, h->dc, h->dr, h->l64, h->u64, h->x64, h->x064, h->y64, h->y064, h->x32, h->x032, h->y32,
        h->y032, h->l32, h->u32);
    NIR_LAUNCHED();
    // plain PDHG never reads the anchors in the update, but CHECK reads x0
    NIR_CUDA(cudaStreamSynchronize(s));
    const double t_setup = now_sec();

    ChunkTimer tm;
    if (h->profiling) {
        for (auto& e : tm.e) NIR_CUDA(cudaEventCreate(&e));
        tm.armed = true;
        tm.K = cfg.K;
    }
    const bool fp64_first = (p.precision == NIR_PREC_FP64);
    LoopResult R;
    double t_switch = 0.0;
    try {
        // prec: 0 = (float values, float iterates), 1 = (float, double), 2 = (double, double)
        auto run_phase = [&](int phase, int prec) {
            auto launch = [&, phase, prec]() {
                ChunkTimer* t = h->profiling ? &tm : nullptr;
                if (prec == 2) launch_fast_chunk<double, double>(h, cfg, phase, t);
                else if (prec == 1) launch_fast_chunk<float, double>(h, cfg, phase, t);
                else launch_fast_chunk<float, float>(h, cfg, phase, t);
            };
            const int per = launches_per_chunk(cfg.K, false);
            if (p.use_graphs && !h->profiling && !cfg.persistent) {
                cudaGraphExec_t ge = chunk_graph(h, 1 + phase, chunk_key(h, cfg, phase, prec), launch);
                return run_chunks(h, p, poll, ctx, t0, phase, per, [&]() { NIR_CUDA(cudaGraphLaunch(ge, s)); }, nullptr);
            }
            return run_chunks(h, p, poll, ctx, t0, phase, 0, launch, h->profiling ? &tm : nullptr);
        };
        if (p.max_iters > 0) {
            R = run_phase(0, fp64_first ? 2 : (p.precision == NIR_PREC_MIXED ? 1 : 0));
            if (!R.stopped_by_host && cfg.mixed && !R.last.done && R.last.phase == 1) {
                // the FP32 values stopped improving the KKT error: polish with
                // the FP64 values from the last evaluated point.  The iterates
                // are FP64 in both phases.
                t_switch = now_sec() - t_setup;
                nir::DevState cur;
                d2h(h, &cur, h->st, sizeof(cur));
                if (p.polish_fresh != 2) {
                    // a fresh start at (x+, y+): iterate and anchor both there
                    nir::k_restart_at<<<std::max(grid_for(std::max(n, m)), 1u), nir::kBlock, 0, s>>>(
                        n, m, h->xp64, h->yp64, h->x64, h->x064, h->y64, h->y064);
                    cur.k_base = 0;
                    cur.have_anchor = 0;
                }
                // polish_fresh == 2: a pure change of the matrix precision; the
                // Halpern iterate, its anchor and every counter carry on
                NIR_LAUNCHED();
                cur.apply_restart = 0;
                cur.switch_request = 0;
                cur.stall = 0;
                if (p.polish_fresh == 1) {
                    // the FP64 phase as a fresh solve warm-started at (x+, y+):
                    // initial primal weight, restart schedule from the switch
                    cur.omega = std::exp(cur.log_omega0);
                    cur.tau = cur.eta / cur.omega;
                    cur.sigma = cur.eta * cur.omega;
                    cur.it_phase = cur.iter;
                }
                h2d(h, h->st, &cur, sizeof(cur));
                long long it_switch = cur.iter;
                R = run_phase(1, 2);
                info->iterations_fp64 = 0;
                nir::DevState fin;
                d2h(h, &fin, h->st, sizeof(fin));
                info->iterations_fp64 = fin.iter - it_switch;
            }
        }
    } catch (...) {
        if (tm.armed)
            for (auto& e : tm.e) cudaEventDestroy(e);
        throw;
    }
    if (tm.armed)
        for (auto& e : tm.e) cudaEventDestroy(e);
    nir::DevState st;
    d2h(h, &st, h->st, sizeof(st));
    const bool out64 = p.precision != NIR_PREC_FP32;
    const unsigned g = std::max(grid_for(std::max(n, m)), 1u);
    if (out64) nir::k_unscale_out<double><<<g, nir::kBlock, 0, s>>>(n, m, h->xp64, h->yp64, h->dc, h->dr, h->out_x, h->out_y);
    else nir::k_unscale_out<float><<<g, nir::kBlock, 0, s>>>(n, m, h->xp32, h->yp32, h->dc, h->dr, h->out_x, h->out_y);
    NIR_LAUNCHED();
    std::vector<double> x(n), y(m);
    NIR_CUDA(cudaMemcpyAsync(x.data(), h->out_x, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    NIR_CUDA(cudaMemcpyAsync(y.data(), h->out_y, m * sizeof(double), cudaMemcpyDeviceToHost, s));
    NIR_CUDA(cudaStreamSynchronize(s));
    if (x_out) std::memcpy(x_out, x.data(), n * sizeof(double));
    if (y_out) std::memcpy(y_out, y.data(), m * sizeof(double));
    h->last_x = h->out_x;
    int status;
    if (st.done) status = st.status;
    else if (R.stopped_by_host) status = NIR_STATUS_TIME_LIMIT;
    else status = NIR_STATUS_ITERATION_LIMIT;
    if (p.max_iters <= 0) status = NIR_STATUS_ITERATION_LIMIT;
    fill_info_common(h, st, info);
    info->status = status;
    info->iterations = st.iter;
    h->last_iters = st.iter;
    if (fp64_first) info->iterations_fp64 = st.iter;
    info->objective = host_objective(h, x);
    info->setup_seconds = t_setup - t0;
    info->solve_seconds = now_sec() - t_setup;
    info->time_to_fp64_seconds = t_switch;
    info->iterations_to_tol = (status == NIR_STATUS_OPTIMAL) ? st.iter : -1;
    if (status == NIR_STATUS_INTERNAL_ERROR) g_err = "a grid barrier of the persistent chunk kernel exceeded its wait bound";
    return status;
}

}  // namespace

#include "engine_parallel.cuh"

// ---------------------------------------------------------------- C ABI

extern "C" {

int nir_pdhg_default_params(nir_pdhg_params* p) {
    if (!p) return NIR_STATUS_INPUT_ERROR;
    std::memset(p, 0, sizeof(*p));
    p->algorithm = NIR_ALGO_PDLP;
    p->precision = NIR_PREC_MIXED;
    p->tol = 1e-6;
    p->feas_tol = 0.0;
    p->max_iters = 1000000;
    p->time_limit = 0.0;
    p->check_every = 64;
    p->ruiz_iters = 10;
    p->pock_chambolle = 1;
    p->reflection = 1.0;
    p->restart_sufficient = 0.2;
    p->restart_necessary = 0.8;
    p->restart_artificial = 0.36;
    p->primal_weight_smoothing = 0.5;
    p->step_factor = 0.998;
    p->power_iters = 64;
    p->polish_stall_checks = 40;
    p->polish_switch_kkt = 0.0;
    p->spmv_block_nnz = 0;
    p->use_graphs = 1;
    p->verbose = 0;
    p->restart_anchor = 1;
    p->polish_fresh = 2;
    p->x_init = nullptr;
    p->y_init = nullptr;
    p->omega_init = 0.0;
    p->primal_weight_decades = 1.0;
    p->persistent = 0;
    return 0;
}

const char* nir_pdhg_last_error(void) { return g_err.c_str(); }

int nir_pdhg_create(const nir_lp_view* lp, int device, nir_pdhg** out) {
    if (!out) {
        g_err = "null output handle";
        return NIR_STATUS_INPUT_ERROR;
    }
    *out = nullptr;
    try {
        validate_lp(lp);
    } catch (const std::exception& e) {
        g_err = e.what();
        return NIR_STATUS_INPUT_ERROR;
    }
    auto h = std::make_unique<nir_pdhg>();
    h->device = -1;
    try {
        // the engine's row order (row_order): the LP as the handle holds it
        std::vector<int> ri;
        std::vector<double> rl, ru;
        h->row_orig = row_order(lp);
        const nir_lp_view v = h->row_orig.empty() ? *lp : reorder_rows(lp, h->row_orig, ri, rl, ru);
        create_impl(h.get(), &v, device);
        build_parallel(h.get(), &v, device);
        if (!h->row_orig.empty()) {
            h->d_row_orig = h->alloc<int>(h->row_orig.size());
            h2d(h.get(), h->d_row_orig, h->row_orig.data(), h->row_orig.size() * sizeof(int));
        }
    } catch (const std::invalid_argument& e) {
        g_err = e.what();
        return NIR_STATUS_INPUT_ERROR;
    } catch (const std::exception& e) {
        g_err = e.what();
        return NIR_STATUS_INTERNAL_ERROR;
    }
    *out = h.release();
    return 0;
}

int nir_pdhg_parallel_groups(const nir_lp_view* lp, int32_t* rep_of, double* lambda, int32_t* groups) {
    if (!groups) {
        g_err = "null output";
        return NIR_STATUS_INPUT_ERROR;
    }
    try {
        validate_lp(lp);
        const ParallelGroups g = find_parallel(lp);
        *groups = g.groups;
        if (rep_of) std::copy(g.rep_of.begin(), g.rep_of.end(), rep_of);
        if (lambda) std::copy(g.lam.begin(), g.lam.end(), lambda);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return NIR_STATUS_INPUT_ERROR;
    }
}

int nir_pdhg_update_vectors(nir_pdhg* h, const double* cost, const double* collo, const double* colup,
                            const double* rowlo, const double* rowup) {
    if (!h) {
        g_err = "null handle";
        return NIR_STATUS_INPUT_ERROR;
    }
    try {
        NIR_CUDA(cudaSetDevice(h->device));
        if (cost)
            for (int j = 0; j < h->n; ++j)
                if (!std::isfinite(cost[j])) throw std::invalid_argument("non-finite cost");
        std::vector<double> rl, ru;
        if (!h->row_orig.empty()) {
            if (rowlo) rows_in(h, rowlo, rl);
            if (rowup) rows_in(h, rowup, ru);
        }
        upload_vectors(h, cost, collo, colup, rowlo && !rl.empty() ? rl.data() : rowlo,
                       rowup && !ru.empty() ? ru.data() : rowup);
        if (h->inner) parallel_update_vectors(h);
        return 0;
    } catch (const std::invalid_argument& e) {
        g_err = e.what();
        return NIR_STATUS_INPUT_ERROR;
    } catch (const std::exception& e) {
        g_err = e.what();
        return NIR_STATUS_INTERNAL_ERROR;
    }
}

int nir_pdhg_solve(nir_pdhg* h, const nir_pdhg_params* p_in, int (*poll)(void*), void* poll_ctx, double* x_out,
                   double* y_out, nir_pdhg_info* info) {
    nir_pdhg_info dummy;
    if (!info) info = &dummy;
    std::memset(info, 0, sizeof(*info));
    if (!h) {
        g_err = "null handle";
        return info->status = NIR_STATUS_INPUT_ERROR;
    }
    nir_pdhg_params p;
    if (p_in) p = *p_in;
    else nir_pdhg_default_params(&p);
    if (p.algorithm < 0 || p.algorithm > 2 || p.precision < 0 || p.precision > 2 || !(p.tol >= 0.0) ||
        p.check_every < 1 || p.reflection < 0.0 || p.reflection > 1.0) {
        g_err = "invalid parameters";
        return info->status = NIR_STATUS_INPUT_ERROR;
    }
    try {
        NIR_CUDA(cudaSetDevice(h->device));
        const int before = h->launches;
        h->last_x = nullptr;  // out_x and x64 serve as scratch until the solve's end
        // the caller's row order <-> the engine's (row_order)
        const bool mapped = !h->row_orig.empty();
        std::vector<double> yin, yres, xdev, ydev;
        // the row order and the parallel columns remap a start on the host
        if (h->inner) p.x_init = host_readable(p.x_init, size_t(h->n), xdev);
        if (mapped || h->inner) p.y_init = host_readable(p.y_init, size_t(h->m), ydev);
        if (mapped && p.y_init) {
            rows_in(h, p.y_init, yin);
            p.y_init = yin.data();
        }
        if (mapped && y_out) yres.resize(size_t(h->m));
        double* y_eng = (mapped && y_out) ? yres.data() : y_out;
        int st;
        if (p.algorithm == NIR_ALGO_REFERENCE) st = solve_reference(h, p, poll, poll_ctx, x_out, y_eng, info);
        else if (h->inner) st = solve_parallel(h, p, poll, poll_ctx, x_out, y_eng, info);
        else st = solve_fast(h, p, poll, poll_ctx, x_out, y_eng, info);
        if (mapped && y_out) rows_out(h, yres.data(), y_out);
        info->kernel_launches = h->launches - before;
        return st;
    } catch (const std::invalid_argument& e) {
        g_err = e.what();
        return info->status = NIR_STATUS_INPUT_ERROR;
    } catch (const std::exception& e) {
        g_err = e.what();
        return info->status = NIR_STATUS_INTERNAL_ERROR;
    }
}

int nir_pdhg_solve_lp(const nir_lp_view* lp, int device, const nir_pdhg_params* p, int (*poll)(void*), void* ctx,
                      double* x_out, double* y_out, nir_pdhg_info* info) {
    nir_pdhg* h = nullptr;
    int rc = nir_pdhg_create(lp, device, &h);
    if (rc != 0) {
        if (info) {
            std::memset(info, 0, sizeof(*info));
            info->status = rc;
        }
        return rc;
    }
    const double t0 = now_sec();
    rc = nir_pdhg_solve(h, p, poll, ctx, x_out, y_out, info);
    (void)t0;
    nir_pdhg_free(h);
    return rc;
}

void nir_pdhg_free(nir_pdhg* h) { delete h; }

int nir_pdhg_spmv(nir_pdhg* h, int transpose, int kernel, const double* x, double* y) {
    if (!h || !x || !y || kernel < 0 || kernel > 2) {
        g_err = "invalid arguments";
        return NIR_STATUS_INPUT_ERROR;
    }
    try {
        NIR_CUDA(cudaSetDevice(h->device));
        cudaStream_t s = h->stream;
        Orient& o = transpose ? h->At : h->A;
        const int nin = o.cols, nout = o.rows;
        double* din = transpose ? h->tmp_m : h->tmp_n;
        double* dout = transpose ? h->tmp_n : h->tmp_m;
        // row-indexed vectors in the caller's order (row_order)
        std::vector<double> xin, yres;
        double* y_caller = y;
        if (!h->row_orig.empty()) {
            if (transpose) {
                rows_in(h, x, xin);
                x = xin.data();
            } else {
                yres.resize(size_t(h->m));
                y = yres.data();
            }
        }
        NIR_CUDA(cudaMemcpyAsync(din, x, nin * sizeof(double), cudaMemcpyHostToDevice, s));
        if (kernel == 0) {
            nir::k_ref_spmv<<<std::max(grid_for(nout), 1u), nir::kBlock, 0, s>>>(nout, o.rp, o.ci, o.v_orig, din, dout);
            NIR_LAUNCHED();
        } else {
            if (!o.blk) set_blocks(h, o, auto_cap(h->nnz, nout));
            if (kernel == 1) {
                const LaunchCfg lc = warp_cfg<double>(h, nir::k_spmv_adaptive<double, double, double>, o.nblk);
                nir::k_spmv_adaptive<double, double, double><<<lc.grid, nir::kBlock, lc.smem, s>>>(
                    o.blk, o.nblk, o.cap, o.rp, o.ci, o.v_orig, din, dout);
                NIR_LAUNCHED();
            } else {
                if (!o.v32_orig) {
                    o.v32_orig = h->allocz<float>(o.nnz);
                    nir::k_to_float<<<grid_for(o.nnz), nir::kBlock, 0, s>>>(o.nnz, o.v_orig, o.v32_orig);
                }
                float* fin = transpose ? h->tmp_m32 : h->tmp_n32;
                float* fout = transpose ? h->tmp_n32 : h->tmp_m32;
                nir::k_to_float<<<std::max(grid_for(nin), 1u), nir::kBlock, 0, s>>>(nin, din, fin);
                const LaunchCfg lc = warp_cfg<float>(h, nir::k_spmv_adaptive<float, float, float>, o.nblk);
                nir::k_spmv_adaptive<float, float, float><<<lc.grid, nir::kBlock, lc.smem, s>>>(
                    o.blk, o.nblk, o.cap, o.rp, o.ci, o.v32_orig, fin, fout);
                nir::k_to_double<<<std::max(grid_for(nout), 1u), nir::kBlock, 0, s>>>(nout, fout, dout);
                NIR_LAUNCHED();
            }
        }
        NIR_CUDA(cudaMemcpyAsync(y, dout, nout * sizeof(double), cudaMemcpyDeviceToHost, s));
        NIR_CUDA(cudaStreamSynchronize(s));
        if (!yres.empty()) rows_out(h, yres.data(), y_caller);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return NIR_STATUS_INTERNAL_ERROR;
    }
}

int nir_pdhg_time_spmv(nir_pdhg* h, int transpose, int kernel, int reps, int flush_l2, double* usec) {
    if (!h || !usec || reps < 1 || kernel < 0 || kernel > 2) {
        g_err = "invalid arguments";
        return NIR_STATUS_INPUT_ERROR;
    }
    try {
        NIR_CUDA(cudaSetDevice(h->device));
        cudaStream_t s = h->stream;
        Orient& o = transpose ? h->At : h->A;
        const int nin = o.cols, nout = o.rows;
        if (!o.blk) set_blocks(h, o, auto_cap(h->nnz, nout));
        if (kernel == 2 && !o.v32_orig) {
            o.v32_orig = h->allocz<float>(o.nnz);
            nir::k_to_float<<<grid_for(o.nnz), nir::kBlock, 0, s>>>(o.nnz, o.v_orig, o.v32_orig);
        }
        double* din = transpose ? h->tmp_m : h->tmp_n;
        double* dout = transpose ? h->tmp_n : h->tmp_m;
        float* fin = transpose ? h->tmp_m32 : h->tmp_n32;
        float* fout = transpose ? h->tmp_n32 : h->tmp_m32;
        nir::k_fill<<<std::max(grid_for(nin), 1u), nir::kBlock, 0, s>>>(nin, 1.0, din);
        nir::k_to_float<<<std::max(grid_for(nin), 1u), nir::kBlock, 0, s>>>(nin, din, fin);
        if (flush_l2 && !h->flush) {
            h->flush_bytes = size_t(512) << 20;
            h->flush = h->alloc<unsigned char>(h->flush_bytes);
        }
        const LaunchCfg l64 = warp_cfg<double>(h, nir::k_spmv_adaptive<double, double, double>, o.nblk);
        const LaunchCfg l32 = warp_cfg<float>(h, nir::k_spmv_adaptive<float, float, float>, o.nblk);
        cudaEvent_t a, b;
        NIR_CUDA(cudaEventCreate(&a));
        NIR_CUDA(cudaEventCreate(&b));
        double total_ms = 0.0;
        for (int r = 0; r < reps + 1; ++r) {
            if (flush_l2) NIR_CUDA(cudaMemsetAsync(h->flush, r & 0xff, h->flush_bytes, s));
            NIR_CUDA(cudaEventRecord(a, s));
            if (kernel == 0)
                nir::k_ref_spmv<<<std::max(grid_for(nout), 1u), nir::kBlock, 0, s>>>(nout, o.rp, o.ci, o.v_orig, din, dout);
            else if (kernel == 1)
                nir::k_spmv_adaptive<double, double, double><<<l64.grid, nir::kBlock, l64.smem, s>>>(
                    o.blk, o.nblk, o.cap, o.rp, o.ci, o.v_orig, din, dout);
            else
                nir::k_spmv_adaptive<float, float, float><<<l32.grid, nir::kBlock, l32.smem, s>>>(
                    o.blk, o.nblk, o.cap, o.rp, o.ci, o.v32_orig, fin, fout);
            NIR_LAUNCHED();
            NIR_CUDA(cudaEventRecord(b, s));
            NIR_CUDA(cudaEventSynchronize(b));
            float ms = 0.0f;
            NIR_CUDA(cudaEventElapsedTime(&ms, a, b));
            if (r > 0) total_ms += ms;  // the first launch is a warm-up
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        *usec = 1000.0 * total_ms / reps;
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return NIR_STATUS_INTERNAL_ERROR;
    }
}

}  // extern "C"

namespace {

// Launches k_spmv_cta for the run length of the layout with a persistent
// grid of the resident CTAs.
template <typename TA, typename TV, typename TX, int E>
void launch_spmv_cta_e(nir_pdhg* h, const Orient::Cta& c, const int* rp, const TV* val, const TX* x, TA* y) {
    auto* kern = nir::k_spmv_cta<TA, TV, TX, E>;
    const int grid = lay_grid<E, TA>(h, kern, c.nblk);
    kern<<<grid, nir::kBlock, 0, h->stream>>>(c.blk, c.nblk, rp, c.ci, val, x, y);
    NIR_LAUNCHED();
}

template <typename TA, typename TV, typename TX>
void launch_spmv_cta(nir_pdhg* h, const Orient::Cta& c, const int* rp, const TV* val, const TX* x, TA* y) {
    switch (c.cap) {
        case 256: launch_spmv_cta_e<TA, TV, TX, 1>(h, c, rp, val, x, y); break;
        case 512: launch_spmv_cta_e<TA, TV, TX, 2>(h, c, rp, val, x, y); break;
        case 1024: launch_spmv_cta_e<TA, TV, TX, 4>(h, c, rp, val, x, y); break;
        case 2048: launch_spmv_cta_e<TA, TV, TX, 8>(h, c, rp, val, x, y); break;
        default: throw std::invalid_argument("CTA block capacity must be 256, 512, 1024 or 2048");
    }
}

// One launch of a measured SpMV kind (nir_pdhg_time_kernel) on the
// handle's device vectors: din/fin inputs, dout/fout outputs.
void launch_kernel_kind(nir_pdhg* h, Orient& o, int kernel, int cap, const double* din, const float* fin, double* dout,
                        float* fout) {
    cudaStream_t s = h->stream;
    const int nout = o.rows;
    switch (kernel) {
        case 0:
            nir::k_ref_spmv<<<std::max(grid_for(nout), 1u), nir::kBlock, 0, s>>>(nout, o.rp, o.ci, o.v_orig, din, dout);
            NIR_LAUNCHED();
            return;
        case 1:
        case 2: {
            if (kernel == 1) {
                const LaunchCfg lc = warp_cfg<double>(h, nir::k_spmv_adaptive<double, double, double>, o.nblk);
                nir::k_spmv_adaptive<double, double, double><<<lc.grid, nir::kBlock, lc.smem, s>>>(
                    o.blk, o.nblk, o.cap, o.rp, o.ci, o.v_orig, din, dout);
            } else {
                const LaunchCfg lc = warp_cfg<float>(h, nir::k_spmv_adaptive<float, float, float>, o.nblk);
                nir::k_spmv_adaptive<float, float, float><<<lc.grid, nir::kBlock, lc.smem, s>>>(
                    o.blk, o.nblk, o.cap, o.rp, o.ci, o.v32_orig, fin, fout);
            }
            NIR_LAUNCHED();
            return;
        }
        case 3:
        case 4:
        case 5: {
            Orient::Cta& c = cta_layout(h, o, cap);
            cta_orig_values(h, o, c);
            if (kernel == 3) launch_spmv_cta<double, double, double>(h, c, o.rp, c.vorig, din, dout);
            else if (kernel == 4) launch_spmv_cta<float, float, float>(h, c, o.rp, c.v32orig, fin, fout);
            else launch_spmv_cta<double, float, double>(h, c, o.rp, c.v32orig, din, dout);
            return;
        }
        default: break;
    }
    // the row-less ceilings over the CSR stream itself (groups of 8 from 0)
    const int groups = int(o.nnz / 8);
    const unsigned grid = unsigned(8 * h->sms);
    if (!h->ceil_out) h->ceil_out = h->alloc<double>(size_t(grid) * nir::kBlock);
    double* out = h->ceil_out;
    switch (kernel) {
        case 6: nir::k_stream_ceiling<double, double, double, true><<<grid, nir::kBlock, 0, s>>>(groups, o.ci, o.v_orig, din, out); break;
        case 7: nir::k_stream_ceiling<float, float, float, true><<<grid, nir::kBlock, 0, s>>>(groups, o.ci, o.v32_orig, fin, reinterpret_cast<float*>(out)); break;
        case 8: nir::k_stream_ceiling<double, double, double, false><<<grid, nir::kBlock, 0, s>>>(groups, o.ci, o.v_orig, din, out); break;
        case 9: nir::k_stream_ceiling<float, float, float, false><<<grid, nir::kBlock, 0, s>>>(groups, o.ci, o.v32_orig, fin, reinterpret_cast<float*>(out)); break;
        default: throw std::invalid_argument("kernel kind out of range");
    }
    NIR_LAUNCHED();
}

// FP32 copy of the original values (the FP32 kernel kinds).
void ensure_v32_orig(nir_pdhg* h, Orient& o) {
    if (o.v32_orig) return;
    o.v32_orig = h->allocz<float>(o.nnz);
    nir::k_to_float<<<grid_for(o.nnz), nir::kBlock, 0, h->stream>>>(o.nnz, o.v_orig, o.v32_orig);
    NIR_LAUNCHED();
}

}  // namespace

extern "C" {

int nir_pdhg_spmv_kernel(nir_pdhg* h, int transpose, int kernel, int block_nnz, const double* x, double* y) {
    if (!h || !x || !y || kernel < 0 || kernel > 5) {
        g_err = "invalid arguments";
        return NIR_STATUS_INPUT_ERROR;
    }
    try {
        NIR_CUDA(cudaSetDevice(h->device));
        cudaStream_t s = h->stream;
        Orient& o = transpose ? h->At : h->A;
        const int nin = o.cols, nout = o.rows;
        if (!o.blk) set_blocks(h, o, auto_cap(h->nnz, nout));
        ensure_v32_orig(h, o);
        double* din = transpose ? h->tmp_m : h->tmp_n;
        double* dout = transpose ? h->tmp_n : h->tmp_m;
        float* fin = transpose ? h->tmp_m32 : h->tmp_n32;
        float* fout = transpose ? h->tmp_n32 : h->tmp_m32;
        // row-indexed vectors in the caller's order (row_order)
        std::vector<double> xin, yres;
        double* y_caller = y;
        if (!h->row_orig.empty()) {
            if (transpose) {
                rows_in(h, x, xin);
                x = xin.data();
            } else {
                yres.resize(size_t(h->m));
                y = yres.data();
            }
        }
        NIR_CUDA(cudaMemcpyAsync(din, x, nin * sizeof(double), cudaMemcpyHostToDevice, s));
        nir::k_to_float<<<std::max(grid_for(nin), 1u), nir::kBlock, 0, s>>>(nin, din, fin);
        NIR_LAUNCHED();
        launch_kernel_kind(h, o, kernel, block_nnz >= 256 ? block_nnz : kCtaCap, din, fin, dout, fout);
        if (kernel == 2 || kernel == 4) {
            nir::k_to_double<<<std::max(grid_for(nout), 1u), nir::kBlock, 0, s>>>(nout, fout, dout);
            NIR_LAUNCHED();
        }
        NIR_CUDA(cudaMemcpyAsync(y, dout, nout * sizeof(double), cudaMemcpyDeviceToHost, s));
        NIR_CUDA(cudaStreamSynchronize(s));
        if (!yres.empty()) rows_out(h, yres.data(), y_caller);
        return 0;
    } catch (const std::invalid_argument& e) {
        g_err = e.what();
        return NIR_STATUS_INPUT_ERROR;
    } catch (const std::exception& e) {
        g_err = e.what();
        return NIR_STATUS_INTERNAL_ERROR;
    }
}

int nir_pdhg_time_kernel(nir_pdhg* h, int transpose, int kernel, int block_nnz, int reps, int flush_l2,
                         double* usec) {
    if (!h || !usec || reps < 1 || kernel < 0 || kernel > 9) {
        g_err = "invalid arguments";
        return NIR_STATUS_INPUT_ERROR;
    }
    try {
        NIR_CUDA(cudaSetDevice(h->device));
        cudaStream_t s = h->stream;
        Orient& o = transpose ? h->At : h->A;
        const int nin = o.cols;
        // warp kinds: row blocks of capacity block_nnz (32..256), else the
        // current ones (or the automatic capacity); CTA kinds: blocks of
        // block_nnz (256..2048), else those of the iteration kernels (1024)
        if (kernel == 1 || kernel == 2) {
            if (block_nnz >= 32 && block_nnz <= nir::kWarpCapMax) set_blocks(h, o, block_nnz);
            else if (!o.blk) set_blocks(h, o, auto_cap(h->nnz, o.rows));
        }
        ensure_v32_orig(h, o);
        const int cap = block_nnz >= 256 ? block_nnz : kCtaCap;
        if (kernel >= 3 && kernel <= 5) cta_orig_values(h, o, cta_layout(h, o, cap));
        double* din = transpose ? h->tmp_m : h->tmp_n;
        double* dout = transpose ? h->tmp_n : h->tmp_m;
        float* fin = transpose ? h->tmp_m32 : h->tmp_n32;
        float* fout = transpose ? h->tmp_n32 : h->tmp_m32;
        nir::k_fill<<<std::max(grid_for(nin), 1u), nir::kBlock, 0, s>>>(nin, 1.0, din);
        nir::k_to_float<<<std::max(grid_for(nin), 1u), nir::kBlock, 0, s>>>(nin, din, fin);
        NIR_LAUNCHED();
        if (flush_l2 && !h->flush) {
            h->flush_bytes = size_t(512) << 20;
            h->flush = h->alloc<unsigned char>(h->flush_bytes);
        }
        cudaEvent_t a, b;
        NIR_CUDA(cudaEventCreate(&a));
        NIR_CUDA(cudaEventCreate(&b));
        double total_ms = 0.0;
        try {
            for (int r = 0; r < reps + 1; ++r) {
                if (flush_l2) NIR_CUDA(cudaMemsetAsync(h->flush, r & 0xff, h->flush_bytes, s));
                NIR_CUDA(cudaEventRecord(a, s));
                launch_kernel_kind(h, o, kernel, cap, din, fin, dout, fout);
                NIR_CUDA(cudaEventRecord(b, s));
                NIR_CUDA(cudaEventSynchronize(b));
                float ms = 0.0f;
                NIR_CUDA(cudaEventElapsedTime(&ms, a, b));
                if (r > 0) total_ms += ms;  // the first launch is a warm-up
            }
        } catch (...) {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
            throw;
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        *usec = 1000.0 * total_ms / reps;
        return 0;
    } catch (const std::invalid_argument& e) {
        g_err = e.what();
        return NIR_STATUS_INPUT_ERROR;
    } catch (const std::exception& e) {
        g_err = e.what();
        return NIR_STATUS_INTERNAL_ERROR;
    }
}

int nir_pdhg_set_profiling(nir_pdhg* h, int on) {
    if (!h) return NIR_STATUS_INPUT_ERROR;
    h->profiling = on != 0;
    return 0;
}

int nir_pdhg_kernel_times(nir_pdhg* h, nir_pdhg_kernel_time* out) {
    if (!h || !out) return NIR_STATUS_INPUT_ERROR;
    *out = h->ktime;
    for (int q = 0; q < 2; ++q) {
        if (out->samples[q] > 0) {
            out->primal_us[q] /= double(out->samples[q]);
            out->dual_us[q] /= double(out->samples[q]);
            out->iter_us[q] /= double(out->samples[q]);
        }
    }
    return 0;
}

}  // extern "C"

namespace {

// Steady-state timing of the fused iteration kernels of one precision on
// the handle's current state: `reps` back-to-back launches of k_primal
// alone, of k_dual alone, and of reps (k_primal, k_dual) pairs, each batch
// captured in a CUDA graph as the solve's chunks are, and its launch
// bracketed by CUDA events on the handle's stream (a warm-up launch first).  The kernels run against
// a copy of the solver state marked running, on the layout and scaled
// values of the last solve; they overwrite the iterates, which a finished
// solve no longer needs (its result is in out_x / out_y).
template <typename TV, typename TX, int LP, int LD>
void time_iteration_l(nir_pdhg* h, int reps, double* primal_us, double* dual_us, double* pair_us) {
    cudaStream_t s = h->stream;
    const PartLayout L = part_layout(h);
    if (!h->st_time) h->st_time = h->alloc<nir::DevState>(1);
    nir::DevState st;
    d2h(h, &st, h->st, sizeof(st));
    st.done = 0;
    st.phase = 0;
    h2d(h, h->st_time, &st, sizeof(st));
    const int gp = lay_grid<LP, TX>(h, nir::k_primal<LP, TV, TX, false>, lay_nblk(h->At));
    const int gd = lay_grid<LD, TX>(h, nir::k_dual<LD, TV, TX, false>, lay_nblk(h->A));
    const size_t sp = lay_smem<LP, TX>(), sd = lay_smem<LD, TX>();
    nir::IterArgs ap{lay_of(h->At), L.P, h->st_time, 1, 1, 0, 1.0};
    nir::IterArgs ad{lay_of(h->A), L.D, h->st_time, 1, 1, 0, 1.0};
    const TV* valAt = vals_of<TV>(h->At);
    const TV* valA = vals_of<TV>(h->A);
    auto primal = [&]() {
        nir::k_primal<LP, TV, TX, false><<<gp, nir::kBlock, sp, s>>>(
            ap, valAt, Vec<TX>::y(h), Vec<TX>::x(h), Vec<TX>::xb(h), Vec<TX>::xp(h), Vec<TX>::c(h), Vec<TX>::l(h),
            Vec<TX>::u(h), Vec<TX>::x0(h));
    };
    auto dual = [&]() {
        nir::k_dual<LD, TV, TX, false><<<gd, nir::kBlock, sd, s>>>(ad, valA, Vec<TX>::xb(h), Vec<TX>::y(h),
                                                                   Vec<TX>::yp(h), Vec<TX>::rl(h), Vec<TX>::ru(h),
                                                                   Vec<TX>::y0(h));
    };
    cudaEvent_t a, b;
    NIR_CUDA(cudaEventCreate(&a));
    NIR_CUDA(cudaEventCreate(&b));
    auto timed = [&](int which) {
        cudaGraph_t g = nullptr;
        cudaGraphExec_t ge = nullptr;
        NIR_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        for (int r = 0; r < reps; ++r) {
            if (which != 1) primal();
            if (which != 0) dual();
        }
        const cudaError_t launched = cudaGetLastError();
        const cudaError_t ended = cudaStreamEndCapture(s, &g);
        if (launched != cudaSuccess || ended != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            NIR_CUDA(launched != cudaSuccess ? launched : ended);
        }
        float ms = 0.0f;
        try {
            NIR_CUDA(cudaGraphInstantiate(&ge, g, 0));
            for (int w = 0; w < 2; ++w) {  // the first launch warms up
                NIR_CUDA(cudaEventRecord(a, s));
                NIR_CUDA(cudaGraphLaunch(ge, s));
                NIR_CUDA(cudaEventRecord(b, s));
                NIR_CUDA(cudaEventSynchronize(b));
            }
            NIR_CUDA(cudaEventElapsedTime(&ms, a, b));
        } catch (...) {
            if (ge) cudaGraphExecDestroy(ge);
            cudaGraphDestroy(g);
            throw;
        }
        cudaGraphExecDestroy(ge);
        cudaGraphDestroy(g);
        return 1000.0 * ms / reps;
    };
    *primal_us = timed(0);
    *dual_us = timed(1);
    *pair_us = timed(2);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    h->launches += 8 * reps;
}

}  // namespace

extern "C" {

int nir_pdhg_time_iteration(nir_pdhg* h, int precision, int reps, double* primal_us, double* dual_us,
                            double* pair_us) {
    if (!h || !primal_us || !dual_us || !pair_us || reps < 1 || precision < 0 || precision > 2) {
        g_err = "invalid arguments";
        return NIR_STATUS_INPUT_ERROR;
    }
    if (h->inner) h = h->inner.get();  // PDHG / PDLP solves ran on the equivalent LP
    try {
        NIR_CUDA(cudaSetDevice(h->device));
        if (h->A.lay < 0 || h->At.lay < 0)
            throw std::invalid_argument("no PDHG / PDLP solve has set up the iteration kernels yet");
        if (h->last_x == h->x64) h->last_x = nullptr;  // a reference-loop result the kernels would overwrite
        with_lays(h, [&](auto lp, auto ld) {
            constexpr int LP = decltype(lp)::value, LD = decltype(ld)::value;
            if (precision == NIR_PREC_FP64) time_iteration_l<double, double, LP, LD>(h, reps, primal_us, dual_us, pair_us);
            else if (precision == NIR_PREC_MIXED) time_iteration_l<float, double, LP, LD>(h, reps, primal_us, dual_us, pair_us);
            else time_iteration_l<float, float, LP, LD>(h, reps, primal_us, dual_us, pair_us);
        });
        return 0;
    } catch (const std::invalid_argument& e) {
        g_err = e.what();
        return NIR_STATUS_INPUT_ERROR;
    } catch (const std::exception& e) {
        g_err = e.what();
        return NIR_STATUS_INTERNAL_ERROR;
    }
}

int nir_pdhg_history(nir_pdhg* h, double* out, int max_entries) {
    if (!h || !out || max_entries < 0) return -1;
    if (h->inner) h = h->inner.get();  // PDHG / PDLP solves ran on the equivalent LP
    try {
        NIR_CUDA(cudaSetDevice(h->device));
        std::vector<double> ring(8 * nir::kHist);
        d2h(h, ring.data(), h->hist, ring.size() * sizeof(double));
        // entries carry their iteration count; keep those of the last solve
        std::vector<int> idx;
        for (int i = 0; i < nir::kHist; ++i)
            if (ring[8 * i] > 0.0 && ring[8 * i] <= double(h->last_iters)) idx.push_back(i);
        std::sort(idx.begin(), idx.end(), [&](int a, int b) { return ring[8 * a] < ring[8 * b]; });
        int cnt = 0;
        for (int i : idx) {
            if (cnt >= max_entries) break;
            std::memcpy(out + 8 * cnt, &ring[8 * i], 8 * sizeof(double));
            ++cnt;
        }
        return cnt;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

int nir_pdhg_get_layout(nir_pdhg* h, nir_pdhg_layout* out) {
    if (!h || !out) return NIR_STATUS_INPUT_ERROR;
    out->nrow = h->m;
    out->ncol = h->n;
    out->nnz = h->nnz;
    const nir_pdhg* src = h->inner ? h->inner.get() : h;  // PDHG / PDLP solves ran on the equivalent LP
    out->blocks_a = src->A.lay >= 0 ? lay_nblk(src->A) : 0;
    out->blocks_at = src->At.lay >= 0 ? lay_nblk(src->At) : 0;
    out->block_nnz = src->A.lay == nir::kLayCta ? kCtaCap : src->A.cap;
    out->block_nnz_at = src->At.lay == nir::kLayCta ? kCtaCap : src->At.cap;
    out->device_bytes = h->device_bytes;
    return 0;
}

}  // extern "C"

// ---------------------------------------------------------------- no-allocation entry point
//
// nir_pdhg_reference_solve_noalloc runs the reference PDHG loop (the same
// kernels as NIR_ALGO_REFERENCE) on an LP that the caller already holds in
// device memory, for callers that cannot allocate device memory themselves:
// a process whose whole device budget belongs to its own pool allocator, or
// a latency-critical caller that may not take cudaMalloc's implicit device
// synchronisation.  Its working memory (the extrapolated primal, the two
// power-iteration vectors, per-block maxima and the solver state) lives in
// the file-scope array below; every GPU that loads this library holds the
// array until the process exits.

namespace {

constexpr long long kNoAllocScratchDoubles = 1LL << 20;  // 8 MiB per device

__device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

// Device address of g_noalloc_scratch, resolved once per device with that
// device current.  In host code the symbol itself is only a host-side
// stand-in and must never be passed to a kernel.
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_addr[kMaxDevices] = {};

double* noalloc_scratch(int device) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            throw CudaError(std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
        g_noalloc_addr[device] = static_cast<double*>(p);
    }
    return g_noalloc_addr[device];
}

}  // namespace

extern "C" int nir_pdhg_reference_solve_noalloc(const nir_csr_dev* A, const nir_csr_dev* At, const double* cost,
                                                const double* collo, const double* colup, const double* rowlo,
                                                const double* rowup, int64_t max_iters, void* stream, double* x_out,
                                                double* y_out, int64_t* iterations, int32_t* status) {
    if (!A || !At || !cost || !collo || !colup || !rowlo || !rowup || !x_out || !y_out || !iterations || !status) {
        g_err = "null argument";
        return NIR_STATUS_INPUT_ERROR;
    }
    const long long m = A->rows, n = A->cols;
    if (m < 0 || n < 0 || At->rows != n || At->cols != m || max_iters < 0) {
        g_err = "inconsistent dimensions of A and A'";
        return NIR_STATUS_INPUT_ERROR;
    }
    // scratch: state (256 B) | xbar (n) | u (n) | v (m) | per-block maxima
    const long long state_d = 32;
    static_assert(sizeof(nir::DevState) <= 32 * sizeof(double),
                  "the solver state must fit the 32 doubles reserved for it ahead of xbar");
    const long long nblk = (m + nir::kBlock - 1) / nir::kBlock;
    const long long need = state_d + 2 * n + m + std::max(nblk, 1LL);
    if (need > kNoAllocScratchDoubles) {
        g_err = "LP too large for the no-allocation entry point: needs 32 + 2*ncol + nrow + ceil(nrow/256) = " +
                std::to_string(need) + " doubles of scratch, the limit is " + std::to_string(kNoAllocScratchDoubles);
        return NIR_STATUS_INPUT_ERROR;
    }
    try {
        int dev = 0;
        NIR_CUDA(cudaGetDevice(&dev));
        if (dev < 0 || dev >= kMaxDevices) throw std::invalid_argument("device ordinal beyond the supported range");
        double* base = noalloc_scratch(dev);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        nir::DevState* st = reinterpret_cast<nir::DevState*>(base);
        double* xbar = base + state_d;
        double* u = xbar + n;
        double* v = u + n;
        double* part = v + m;
        const int mi = int(m), ni = int(n);
        // every call starts from a cleared state: the array keeps the last call's contents
        nir::DevState st0{};
        st0.max_iters = max_iters;
        NIR_CUDA(cudaMemcpyAsync(st, &st0, sizeof(st0), cudaMemcpyHostToDevice, s));
        const unsigned gm = grid_for(m), gn = grid_for(n);
        nir::k_fill<<<gn, nir::kBlock, 0, s>>>(n, 1.0, u);
        for (int r = 0; r < 12; ++r) {
            nir::k_ref_spmv<<<gm, nir::kBlock, 0, s>>>(mi, A->row_ptr, A->col_idx, A->value, u, v);
            nir::k_ref_spmv<<<gn, nir::kBlock, 0, s>>>(ni, At->row_ptr, At->col_idx, At->value, v, u);
            nir::k_ref_norm<<<1, 32, 0, s>>>(ni, u, st);
            nir::k_ref_div<<<gn, nir::kBlock, 0, s>>>(ni, u, st);
        }
        nir::k_ref_steps<<<1, 32, 0, s>>>(st);
        nir::k_ref_init<<<grid_for(std::max(m, n)), nir::kBlock, 0, s>>>(ni, mi, collo, colup, x_out, y_out);
        NIR_LAUNCHED();
        const int K = 32;
        nir::DevState host{};
        for (long long done_it = 0; done_it < max_iters; done_it += K) {
            for (int i = 0; i < K; ++i) {
                nir::k_ref_primal<<<gn, nir::kBlock, 0, s>>>(ni, At->row_ptr, At->col_idx, At->value, y_out, cost, collo,
                                                            colup, x_out, xbar, st, i);
                nir::k_ref_dual<<<gm, nir::kBlock, 0, s>>>(mi, A->row_ptr, A->col_idx, A->value, xbar, rowlo, rowup,
                                                          y_out, part, st, i);
                nir::k_ref_stop<<<1, nir::kBlock, 0, s>>>(part, int(std::max(nblk, 1LL)), st, i, K);
            }
            NIR_LAUNCHED();
            NIR_CUDA(cudaMemcpyAsync(&host, st, sizeof(host), cudaMemcpyDeviceToHost, s));
            NIR_CUDA(cudaStreamSynchronize(s));
            if (host.done) break;
        }
        NIR_CUDA(cudaMemcpyAsync(&host, st, sizeof(host), cudaMemcpyDeviceToHost, s));
        NIR_CUDA(cudaStreamSynchronize(s));
        *iterations = max_iters > 0 ? host.ref_iterations : 0;
        *status = host.ref_stopped ? NIR_STATUS_OPTIMAL : NIR_STATUS_ITERATION_LIMIT;
        return *status;
    } catch (const std::invalid_argument& e) {
        g_err = e.what();
        return NIR_STATUS_INPUT_ERROR;
    } catch (const std::exception& e) {
        g_err = e.what();
        return NIR_STATUS_INTERNAL_ERROR;
    }
}

#include "engine_batch.cuh"
#include "engine_verify.cuh"
