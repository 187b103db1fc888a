// The C ABI (include/hfjk.h): context, shell upload, fitted-tensor build, J, K.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <future>
#include <mutex>
#include <thread>
#include <unordered_set>
#include <string>
#include <vector>

#include "../../include/hfjk.h"
#include "context.cuh"
#include "dgemm.cuh"
#include "integrals.cuh"
#include "jk.cuh"
#include "linalg.cuh"
#include "md.cuh"
#include "mp2.cuh"
#include "tc_exchange.cuh"

using namespace hf;

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

// State of hf_exchange_scheduled between calls (device buffers of n x n
// doubles each, allocated on first use).
struct ScheduleState {
    int phase = 0;           // 0: split-BF16 builds, 1: anchored increments
    bool has_prev = false;   // a previous density is held
    int64_t anchor_rank = 0;
    double* prev = nullptr;      // the previous call's density
    double* anchor_d = nullptr;  // D_a
    double* anchor_k = nullptr;  // K64(D_a)
    double* anchor_ft = nullptr; // F_a^T, [anchor_rank][n]
    double* dens = nullptr;      // this call's density (host input staged here)
    double* ft = nullptr;        // this call's factor, F^T [rank][n]
    double* overlap = nullptr;   // S
    double* work[10] = {};       // products and factors of the difference
    double* scalar = nullptr;    // device reduction results
    bool overlap_ready = false;
};

struct hf_ctx {
    int device = 0;
    std::unordered_set<void*> pooled;  // blocks from the stream-ordered pool (freed with cudaFreeAsync)
    cudaStream_t own = nullptr;
    cudaStream_t stream = nullptr;
    std::string err;
    hf_stats stats{};
    bool uploaded = false, built = false;
    // shells
    int n = 0, nt = 0, naux = 0;
    int64_t ntiles = 0;
    std::vector<DevShell> orb, aux;  // aux in internal order (sorted by l)
    std::vector<double> h_exps, h_coefs;  // host copies of the primitive data
    std::vector<int> aux_ref_fn;     // internal aux function -> reference index
    int aux_count[kMaxAuxL + 1] = {};
    DevShell* d_orb = nullptr;
    DevShell* d_aux = nullptr;
    double* d_exps = nullptr;
    double* d_coefs = nullptr;
    int* d_aux_by_l[kMaxAuxL + 1] = {};
    const double* d_btable = nullptr;  // shared by the device's contexts (shared_boys_table)
    // tensors
    double* d_metric = nullptr;  // N x N internal order
    double* d_B = nullptr;       // N x ntiles*4096
    // scratch
    double* d_work = nullptr;
    size_t work_bytes = 0;
    double* d_io = nullptr;  // host-transfer staging: 2 n x n
    size_t io_bytes = 0;
    double* d_kscratch = nullptr;  // K build: Kp | X | Xs
    size_t kscratch_bytes = 0;
    double* d_stage = nullptr;  // exchange staging: C, w, Ct, sign, D, Lc, K
    size_t stage_bytes = 0;
    size_t b_alloc_bytes = 0;  // size of the block holding d_B (retained blocks may be larger)
    void* d_bf16_b = nullptr;  // full BF16 hi/lo copies of B (split-BF16 exchange)
    size_t bf16_alloc_bytes = 0;
    double* d_tcwork = nullptr;  // split-BF16 exchange: factor and X chunk
    size_t tcwork_bytes = 0;
    double* d_ctc = nullptr;  // split-BF16 exchange: the padded FP64 factor
    size_t ctc_bytes = 0;
    int* d_info = nullptr;
    double* d_scalar = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // rows [row0, row1) of the fitted tensor held here (internal auxiliary order;
    // row1 < 0: all of them), for a tensor sharded over devices by auxiliary index
    int row0 = 0, row1 = -1;
    ScheduleState sched;
    // bounded device waits of the split-BF16 exchange (hf_set_wait_limit)
    uint64_t wait_ns = 2000000000ull;  // 2 s: far above any legitimate wait there
    int stall_next = 0;                // the next split-BF16 build runs the stall self-test
};

namespace {

int fail(hf_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

// Rows of the fitted tensor this context holds, and whether it holds them all.
int fitted_rows(const hf_ctx* c) { return (c->row1 < 0 ? c->naux : c->row1) - c->row0; }
bool holds_all_rows(const hf_ctx* c) { return c->row0 == 0 && fitted_rows(c) == c->naux; }

#define HF_CU(call)                                                                           \
    do {                                                                                      \
        cudaError_t _e = (call);                                                              \
        if (_e != cudaSuccess)                                                                \
            return fail(ctx, _e == cudaErrorMemoryAllocation ? HF_ERR_OOM : HF_ERR_CUDA,      \
                        std::string(#call) + ": " + cudaGetErrorString(_e));                  \
    } while (0)

// Device memory that a context keeps. Blocks below kPoolMaxBytes (shell
// tables, the metric, small scratch) come from the device's stream-ordered pool
// (cudaMallocAsync on the context's stream, then that stream is waited for, so
// the block can be used anywhere at once) and go back to it with cudaFreeAsync
// on that stream: unlike cudaMalloc and cudaFree, which may synchronise the
// whole device, neither waits for the work of other streams, which matters when
// many contexts are built and destroyed at once (the batched SCF's clusters,
// built on several host threads). Larger blocks are cudaMalloc'd (and
// retained, below) and freed with cudaFree: served from the pool, blocks of
// gigabytes were mapped afresh whenever a synchronisation trimmed the pool to
// its release threshold (a batched setup of 128 clusters took 11 s instead of
// 1.6 s). Every caller frees a block only after the work that used it on other
// streams has completed.
constexpr size_t kPoolMaxBytes = (size_t)256 << 20;
int alloc(hf_ctx* ctx, void** p, size_t bytes) {
    ctx->stats.device_allocations++;
    const size_t size = bytes ? bytes : 8;
    cudaError_t e = cudaErrorMemoryAllocation;
    if (size < kPoolMaxBytes && ctx->stream) {
        e = cudaMallocAsync(p, size, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e == cudaSuccess) {
            ctx->pooled.insert(*p);
        } else {
            if (*p) cudaFree(*p);
            *p = nullptr;
            cudaGetLastError();
        }
    }
    if (e != cudaSuccess) e = cudaMalloc(p, size);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(ctx, HF_ERR_OOM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed: " +
                                         cudaGetErrorString(e));
    }
    return HF_OK;
}

// Free a block of alloc(): stream-ordered for pool blocks, cudaFree otherwise.
void free_block(hf_ctx* ctx, void* q) {
    if (!q) return;
    if (ctx->pooled.erase(q) && ctx->stream)
        cudaFreeAsync(q, ctx->stream);
    else
        cudaFree(q);
}

template <class T>
void release(hf_ctx* ctx, T*& p) {
    free_block(ctx, (void*)p);
    p = nullptr;
}

// Free hf_exchange_scheduled's buffers and forget its state.
void schedule_release(hf_ctx* ctx) {
    ScheduleState& st = ctx->sched;
    for (double** q : {&st.prev, &st.anchor_d, &st.anchor_k, &st.anchor_ft, &st.dens, &st.ft, &st.overlap, &st.scalar})
        release(ctx, *q);
    for (auto& q : st.work) release(ctx, q);
    st = ScheduleState{};
}

// The Boys-function Taylor grid (boys_grid_host) on each device, uploaded once
// and shared by every context there: a constant of the library, like the c2s
// tables, so a context's creation needs no copy and no synchronisation for it.
// Resolved with that device current; kept until the process exits.
const double* shared_boys_table(int device) {
    static std::mutex mutex;
    static double* tables[64] = {};
    if (device < 0 || device >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(mutex);
    if (!tables[device]) {
        const auto grid = boys_grid_host();
        double* p = nullptr;
        if (cudaMalloc((void**)&p, sizeof(double) * grid.size()) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        // a copy from pageable memory may return before its DMA lands: wait for the
        // device, so kernels on any stream see the table
        if (cudaMemcpy(p, grid.data(), sizeof(double) * grid.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaDeviceSynchronize() != cudaSuccess) {
            cudaGetLastError();
            cudaFree(p);
            return nullptr;
        }
        tables[device] = p;
    }
    return tables[device];
}

// Retained device blocks: the fitted tensor and its BF16 copy (tens of GB at the
// largest clusters) and the J/K scratch areas. A context that is destroyed, or
// that rebuilds for another molecule, hands its blocks of at least
// kRetainMinBytes to a per-device cache instead of freeing them, and the next
// context on that device whose request fits takes one back: a run over many
// geometries of one size (a scan, a benchmark) then maps its large buffers
// once instead of once per geometry, and a cudaFree of tens of GB, which
// synchronises the device, is avoided. At most kRetainBlocks blocks are kept
// per device; a failed allocation empties the cache and retries;
// hf_release_retained frees it on request.
constexpr size_t kRetainMinBytes = kPoolMaxBytes;  // smaller blocks come from the pool
constexpr int kRetainBlocks = 8;
constexpr int kRetainDevices = 64;
struct Retained {
    void* p;
    size_t bytes;
};
std::mutex g_retain_mutex;
std::vector<Retained> g_retained[kRetainDevices];

void free_retained(int device) {
    std::vector<Retained> blocks;
    {
        std::lock_guard<std::mutex> lock(g_retain_mutex);
        if (device < 0 || device >= kRetainDevices) return;
        blocks.swap(g_retained[device]);
    }
    for (const Retained& r : blocks) cudaFree(r.p);
}

// A block of at least `bytes` for a fitted tensor: a retained one that wastes
// at most an eighth of its size, else a new allocation (after emptying the cache
// if the first attempt fails). *have is the block's size.
int big_alloc(hf_ctx* ctx, void** p, size_t bytes, size_t* have) {
    *p = nullptr;
    *have = 0;
    if (bytes >= kRetainMinBytes && ctx->device >= 0 && ctx->device < kRetainDevices) {
        std::lock_guard<std::mutex> lock(g_retain_mutex);
        auto& pool = g_retained[ctx->device];
        int best = -1;
        for (int i = 0; i < (int)pool.size(); ++i)
            if (pool[i].bytes >= bytes && pool[i].bytes - bytes <= pool[i].bytes / 8 &&
                (best < 0 || pool[i].bytes < pool[best].bytes))
                best = i;
        if (best >= 0) {
            *p = pool[best].p;
            *have = pool[best].bytes;
            pool.erase(pool.begin() + best);
            return HF_OK;
        }
    }
    if (alloc(ctx, p, bytes) != HF_OK) {
        free_retained(ctx->device);
        if (alloc(ctx, p, bytes) != HF_OK) return HF_ERR_OOM;
    }
    *have = bytes;
    return HF_OK;
}

// Return a fitted-tensor block: large blocks go to the device's cache (the
// oldest one is freed when it is full), small ones are freed.
template <class T>
void big_release(hf_ctx* ctx, T*& p, size_t& have) {
    if (!p) return;
    void* q = (void*)p;
    p = nullptr;
    const size_t bytes = have;
    have = 0;
    if (bytes < kRetainMinBytes || ctx->device < 0 || ctx->device >= kRetainDevices) {
        free_block(ctx, q);
        return;
    }
    // the block may still be read by work queued on this context's stream
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    void* evict = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_retain_mutex);
        auto& pool = g_retained[ctx->device];
        if ((int)pool.size() >= kRetainBlocks) {
            evict = pool.front().p;
            pool.erase(pool.begin());
        }
        pool.push_back({q, bytes});
    }
    if (evict) cudaFree(evict);
}

// The build's stream-ordered temporaries (several GB for large molecules) come
// from the device's default memory pool; by default the pool returns freed
// memory to the driver at every synchronisation, so each build would map its
// temporaries afresh. Keeping up to 8 GB in the pool makes them reusable.
void keep_pool_memory(int device) {
    static std::mutex mutex;
    static bool done[64] = {};
    if (device < 0 || device >= 64) return;
    std::lock_guard<std::mutex> lock(mutex);
    if (done[device]) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t threshold = (uint64_t)8 << 30;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
    }
    cudaGetLastError();
    done[device] = true;
}

// Stream-ordered temporaries of the build: allocation and release are ordered on
// the context's stream and, unlike cudaFree, do not synchronise the device, so
// contexts on other streams (other clusters) keep running.
int talloc(hf_ctx* ctx, void** p, size_t bytes) {
    ctx->stats.device_allocations++;
    cudaError_t e = cudaMallocAsync(p, bytes ? bytes : 8, ctx->stream);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(ctx, HF_ERR_OOM, "cudaMallocAsync of " + std::to_string(bytes) + " bytes failed: " +
                                         cudaGetErrorString(e));
    }
    return HF_OK;
}

template <class T>
void trelease(hf_ctx* ctx, T*& p) {
    if (p) cudaFreeAsync((void*)p, ctx->stream);
    p = nullptr;
}

int ensure_work(hf_ctx* ctx, size_t bytes) {
    if (ctx->work_bytes >= bytes) return HF_OK;
    big_release(ctx, ctx->d_work, ctx->work_bytes);
    return big_alloc(ctx, (void**)&ctx->d_work, bytes, &ctx->work_bytes);
}

int ensure_io(hf_ctx* ctx, size_t bytes) {
    if (ctx->io_bytes >= bytes) return HF_OK;
    big_release(ctx, ctx->d_io, ctx->io_bytes);
    return big_alloc(ctx, (void**)&ctx->d_io, bytes, &ctx->io_bytes);
}

// Validation of integrals/mod.rs:111-173 plus the device kernels' limits.
int check_table(hf_ctx* ctx, const hf_shell_table* t, const char* name, int max_l, bool aux) {
    if (!t || t->n_shells < 0) return fail(ctx, HF_ERR_ARG, std::string(name) + ": missing shell table");
    if (t->n_shells == 0) return fail(ctx, HF_ERR_ARG, std::string(name) + ": the shell table is empty");
    if (!t->angular_momenta || !t->centers || !t->primitive_offsets || !t->exponents || !t->coefficients ||
        !t->n_contractions)
        return fail(ctx, HF_ERR_ARG, std::string(name) + ": null array in the shell table");
    if (t->primitive_offsets[0] != 0)
        return fail(ctx, HF_ERR_ARG, std::string(name) + ": primitive offsets start at zero");
    for (int64_t s = 0; s < t->n_shells; ++s) {
        const int64_t l = t->angular_momenta[s];
        const int64_t np = t->primitive_offsets[s + 1] - t->primitive_offsets[s];
        const int64_t k = t->n_contractions[s];
        if (np < 1) return fail(ctx, HF_ERR_ARG, std::string(name) + ": every shell needs at least one primitive");
        if (k < 1) return fail(ctx, HF_ERR_ARG, std::string(name) + ": every shell needs at least one contraction");
        if (l < 0 || l > max_l)
            return fail(ctx, HF_ERR_ARG, std::string(name) + ": angular momentum " + std::to_string(l) +
                                             " exceeds the device kernels' maximum " + std::to_string(max_l));
        if (!aux && np > 16)
            return fail(ctx, HF_ERR_ARG, std::string(name) + ": more than 16 primitives in a shell");
        if (aux ? (k != 1) : (k > kMaxOrbContr[l]))
            return fail(ctx, HF_ERR_ARG, std::string(name) + ": too many general contractions (" + std::to_string(k) +
                                             ") for l = " + std::to_string(l));
        for (int x = 0; x < 3; ++x)
            if (!std::isfinite(t->centers[3 * s + x]))
                return fail(ctx, HF_ERR_ARG, std::string(name) + ": centres are finite");
    }
    int64_t ncoef = 0;
    for (int64_t s = 0; s < t->n_shells; ++s)
        ncoef += t->n_contractions[s] * (t->primitive_offsets[s + 1] - t->primitive_offsets[s]);
    for (int64_t i = 0; i < t->primitive_offsets[t->n_shells]; ++i)
        if (!(t->exponents[i] > 0.0) || !std::isfinite(t->exponents[i]))
            return fail(ctx, HF_ERR_ARG, std::string(name) + ": exponents are positive");
    for (int64_t i = 0; i < ncoef; ++i)
        if (!std::isfinite(t->coefficients[i]))
            return fail(ctx, HF_ERR_ARG, std::string(name) + ": coefficients are finite");
    return HF_OK;
}

void time_begin(hf_ctx* ctx) { cudaEventRecord(ctx->ev0, ctx->stream); }
double time_end(hf_ctx* ctx) {
    cudaEventRecord(ctx->ev1, ctx->stream);
    cudaEventSynchronize(ctx->ev1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    return ms;
}

// Ct[i][mu] = C[mu][i] * sqrt|w_i| (zero padded), sign[i] = sign(w_i).
__global__ void k_factor_transpose(const double* __restrict__ C, int64_t n, int64_t ncols,
                                   const double* __restrict__ w, double* __restrict__ Ct, int64_t npad, int64_t opad,
                                   double* __restrict__ sign) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= opad * npad) return;
    const int64_t i = e / npad, mu = e % npad;
    double v = 0.0, s = 1.0;
    if (i < ncols) {
        const double wi = w ? w[i] : 1.0;
        s = wi < 0.0 ? -1.0 : 1.0;
        if (mu < n) v = C[mu * ncols + i] * sqrt(fabs(wi));
    }
    Ct[e] = v;
    if (mu == 0) sign[i] = s;
}

int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

// Carves 256-byte aligned sub-buffers out of one allocation.
struct Carver {
    size_t used = 0;
    size_t take(size_t doubles) {
        const size_t at = used;
        used += (size_t)round_up((int64_t)doubles, 32);
        return at;
    }
};

// Grow-only scratch owned by the context: the K build's Kp/X chunks.
int ensure_scratch(hf_ctx* ctx, double** p, size_t* have, size_t bytes) {
    if (*have >= bytes) return HF_OK;
    big_release(ctx, *p, *have);
    return big_alloc(ctx, (void**)p, bytes, have);
}

int check_async(hf_ctx* ctx, const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return fail(ctx, HF_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return HF_OK;
}


// ---------------------------------------------------------------------------
// Kernels of hf_exchange_scheduled (small, memory-bound helpers).

// max |a - b| (b may be null: max |a|) into *out, which starts at 0: the bits of
// non-negative doubles order as unsigned integers, so atomicMax on them is a max.
__global__ void k_maxabs_diff(const double* __restrict__ a, const double* __restrict__ b, int64_t count,
                              unsigned long long* out) {
    double m = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        m = fmax(m, fabs(a[i] - (b ? b[i] : 0.0)));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ double wm[32];
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x + 31) / 32 ? wm[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (threadIdx.x == 0) atomicMax(out, (unsigned long long)__double_as_longlong(v));
    }
}

// max |Y - I| of an r x r matrix into *out (starting at 0).
__global__ void k_maxabs_minus_eye(const double* __restrict__ y, int64_t r, unsigned long long* out) {
    double m = 0.0;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < r * r; e += (int64_t)gridDim.x * blockDim.x)
        m = fmax(m, fabs(y[e] - ((e / r == e % r) ? 1.0 : 0.0)));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ double wm[32];
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x + 31) / 32 ? wm[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (threadIdx.x == 0) atomicMax(out, (unsigned long long)__double_as_longlong(v));
    }
}

// dst[c][r] = src[r][c] for a rows x cols row-major src.
__global__ void k_transpose_plain(const double* __restrict__ src, int64_t rows, int64_t cols, double* __restrict__ dst) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= rows * cols) return;
    const int64_t c = e / rows, r = e % rows;  // dst element (c, r), written in order
    dst[e] = src[r * cols + c];
}

// Z = 3 I - Y (r x r).
__global__ void k_three_minus(const double* __restrict__ y, int64_t r, double* __restrict__ z) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= r * r) return;
    z[e] = ((e / r == e % r) ? 3.0 : 0.0) - y[e];
}

// Rows k of A = F + G and B = F - G ([r][n] each) and their norms (one CTA per row).
__global__ void k_sum_diff_norms(const double* __restrict__ f, const double* __restrict__ g, int64_t n,
                                 double* __restrict__ a, double* __restrict__ b, double* __restrict__ na,
                                 double* __restrict__ nb) {
    const int64_t row = blockIdx.x;
    double sa = 0.0, sb = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const double x = f[row * n + i], y = g[row * n + i];
        const double s = x + y, d = x - y;
        a[row * n + i] = s;
        b[row * n + i] = d;
        sa += s * s;
        sb += d * d;
    }
    for (int o = 16; o > 0; o >>= 1) {
        sa += __shfl_xor_sync(0xffffffffu, sa, o);
        sb += __shfl_xor_sync(0xffffffffu, sb, o);
    }
    __shared__ double wa[32], wb[32];
    if ((threadIdx.x & 31) == 0) {
        wa[threadIdx.x >> 5] = sa;
        wb[threadIdx.x >> 5] = sb;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ta = 0.0, tb = 0.0;
        for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) {
            ta += wa[w];
            tb += wb[w];
        }
        na[row] = sqrt(ta);
        nb[row] = sqrt(tb);
    }
}

// V+-[i][k] = (alpha_k A[k][i] +- B[k][i] / alpha_k) / 2, alpha_k = sqrt(|b_k| / |a_k|):
// the factors of (A^T B + B^T A) / 2 = V+ V+^T - V- V-^T, written [n][r].
__global__ void k_difference_factors(const double* __restrict__ a, const double* __restrict__ b,
                                     const double* __restrict__ na, const double* __restrict__ nb, int64_t r,
                                     int64_t n, double* __restrict__ vp, double* __restrict__ vm) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= n * r) return;
    const int64_t i = e / r, k = e % r;
    const double alpha = sqrt(fmax(nb[k], 1e-300) / fmax(na[k], 1e-300));
    const double x = alpha * a[k * n + i], y = b[k * n + i] / alpha;
    vp[e] = 0.5 * (x + y);
    vm[e] = 0.5 * (x - y);
}

// K = Ka + Kp - Km.
__global__ void k_combine(const double* __restrict__ ka, const double* __restrict__ kp, const double* __restrict__ km,
                          int64_t count, double* __restrict__ k) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e < count) k[e] = ka[e] + kp[e] - km[e];
}

unsigned blocks_for(int64_t count, int threads = 256) { return (unsigned)((count + threads - 1) / threads); }

// max |a - b| (or max |Y - I| when eye) on the context's stream, read back.
int device_maxabs(hf_ctx* ctx, const double* a, const double* b, int64_t count, bool eye, int64_t r, double* out) {
    unsigned long long* slot = reinterpret_cast<unsigned long long*>(ctx->sched.scalar);
    HF_CU(cudaMemsetAsync(slot, 0, sizeof(unsigned long long), ctx->stream));
    if (eye) k_maxabs_minus_eye<<<std::min<unsigned>(1024, blocks_for(r * r)), 256, 0, ctx->stream>>>(a, r, slot);
    else k_maxabs_diff<<<std::min<unsigned>(4 * 148, blocks_for(count)), 256, 0, ctx->stream>>>(a, b, count, slot);
    unsigned long long bits = 0;
    HF_CU(cudaMemcpyAsync(&bits, slot, sizeof(bits), cudaMemcpyDeviceToHost, ctx->stream));
    HF_CU(cudaStreamSynchronize(ctx->stream));
    std::memcpy(out, &bits, sizeof(double));
    return HF_OK;
}

// C (M x N, row-major, ldc) = alpha A B^T with A M x K (lda) and B N x K (ldb), on the DMMA kernel.
cudaError_t gemm_nt(hf_ctx* ctx, int64_t M, int64_t N, int64_t K, const double* A, int64_t lda, const double* B,
                    int64_t ldb, double* C, int64_t ldc, double alpha) {
    GemmArgs g{};
    g.M = (int)M;
    g.N = (int)N;
    g.K = (int)K;
    g.A = A;
    g.lda = lda;
    g.B = B;
    g.ldb = ldb;
    g.C = C;
    g.ldc = ldc;
    g.alpha = alpha;
    g.beta = 0.0;
    g.tile = 1;  // 64 x 64: these products are at most n x r x n
    return dgemm_nt(g, 1, ctx->stream);
}
}  // namespace

namespace hf {
int context_view(const hf_ctx* ctx, TensorView* out) {
    if (!ctx || !out) return HF_ERR_ARG;
    if (!holds_all_rows(ctx)) return HF_ERR_STATE;
    out->device = ctx->device;
    out->B = ctx->d_B;
    out->n = ctx->n;
    out->nt = ctx->nt;
    out->ntiles = ctx->ntiles;
    out->naux = ctx->naux;
    out->built = ctx->built;
    return HF_OK;
}
}  // namespace hf

extern "C" {

int hf_ctx_create(int device, hf_ctx** out) {
    if (!out) return HF_ERR_ARG;
    *out = nullptr;
    hf_ctx* ctx = new (std::nothrow) hf_ctx();
    if (!ctx) return HF_ERR_OOM;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        delete ctx;
        return HF_ERR_CUDA;
    }
    if (device < 0 || device >= ndev) {
        delete ctx;
        return HF_ERR_ARG;
    }
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->own, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete ctx;
        return HF_ERR_CUDA;
    }
    ctx->stream = ctx->own;
    cudaEventCreate(&ctx->ev0);
    cudaEventCreate(&ctx->ev1);
    upload_c2s(ctx->stream);
    keep_pool_memory(device);
    ctx->d_btable = shared_boys_table(device);
    if (!ctx->d_btable || alloc(ctx, (void**)&ctx->d_info, 4 * sizeof(int)) != HF_OK ||
        alloc(ctx, (void**)&ctx->d_scalar, 4 * sizeof(double)) != HF_OK) {
        hf_ctx_destroy(ctx);
        return HF_ERR_OOM;
    }
    if (cudaGetLastError() != cudaSuccess) {
        hf_ctx_destroy(ctx);
        return HF_ERR_CUDA;
    }
    *out = ctx;
    return HF_OK;
}

static void free_shells(hf_ctx* ctx) {
    release(ctx, ctx->d_orb);
    release(ctx, ctx->d_aux);
    release(ctx, ctx->d_exps);
    release(ctx, ctx->d_coefs);
    for (auto& p : ctx->d_aux_by_l) release(ctx, p);
}

int hf_ctx_destroy(hf_ctx* ctx) {
    if (!ctx) return HF_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    free_shells(ctx);
    release(ctx, ctx->d_metric);
    big_release(ctx, ctx->d_B, ctx->b_alloc_bytes);
    big_release(ctx, ctx->d_work, ctx->work_bytes);
    big_release(ctx, ctx->d_io, ctx->io_bytes);
    big_release(ctx, ctx->d_kscratch, ctx->kscratch_bytes);
    big_release(ctx, ctx->d_stage, ctx->stage_bytes);
    big_release(ctx, ctx->d_bf16_b, ctx->bf16_alloc_bytes);
    big_release(ctx, ctx->d_tcwork, ctx->tcwork_bytes);
    big_release(ctx, ctx->d_ctc, ctx->ctc_bytes);
    schedule_release(ctx);
    release(ctx, ctx->d_info);
    release(ctx, ctx->d_scalar);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->own) cudaStreamDestroy(ctx->own);
    delete ctx;
    return HF_OK;
}

const char* hf_last_error(const hf_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

int hf_set_stream(hf_ctx* ctx, void* stream) {
    if (!ctx) return HF_ERR_ARG;
    cudaStream_t next = stream ? (cudaStream_t)stream : ctx->own;
    if (ctx->stream && next != ctx->stream) {
        // the context's pool blocks go back with cudaFreeAsync on its current stream, so
        // the work queued on the old stream finishes before the switch (unless that
        // stream is being captured, where the caller orders the work)
        cudaSetDevice(ctx->device);
        cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(ctx->stream, &capture) == cudaSuccess && capture == cudaStreamCaptureStatusNone)
            cudaStreamSynchronize(ctx->stream);
        cudaGetLastError();
    }
    ctx->stream = next;
    return HF_OK;
}

int hf_set_fitted_rows(hf_ctx* ctx, int64_t row0, int64_t row1) {
    if (!ctx) return HF_ERR_ARG;
    if (!ctx->uploaded) return fail(ctx, HF_ERR_STATE, "upload shells first");
    if (row0 < 0 || row1 <= row0 || row1 > ctx->naux)
        return fail(ctx, HF_ERR_ARG, "the rows lie in 0 <= row0 < row1 <= n_aux = " + std::to_string(ctx->naux) +
                                         " (got " + std::to_string(row0) + ", " + std::to_string(row1) + ")");
    cudaSetDevice(ctx->device);
    big_release(ctx, ctx->d_B, ctx->b_alloc_bytes);
    big_release(ctx, ctx->d_bf16_b, ctx->bf16_alloc_bytes);
    ctx->built = false;
    ctx->row0 = (int)row0;
    ctx->row1 = (int)row1;
    return HF_OK;
}

int hf_release_retained(int device) {
    if (device < 0 || device >= kRetainDevices) return HF_ERR_ARG;
    int previous = 0;
    cudaGetDevice(&previous);
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return HF_ERR_ARG;
    }
    free_retained(device);
    cudaSetDevice(previous);
    return HF_OK;
}

int hf_set_wait_limit(hf_ctx* ctx, int64_t wait_ns, int stall_next_build) {
    if (!ctx) return HF_ERR_ARG;
    if (wait_ns < 1000 || wait_ns > 60000000000ll)
        return fail(ctx, HF_ERR_ARG, "the wait limit lies between 1 us and 60 s (got " + std::to_string(wait_ns) + " ns)");
    ctx->wait_ns = (uint64_t)wait_ns;
    ctx->stall_next = stall_next_build ? 1 : 0;
    return HF_OK;
}

int hf_shells_upload(hf_ctx* ctx, const hf_shell_table* orbt, const hf_shell_table* auxt) {
    if (!ctx) return HF_ERR_ARG;
    cudaSetDevice(ctx->device);
    int s;
    if ((s = check_table(ctx, orbt, "orbital", kMaxOrbL, false)) != HF_OK) return s;
    if (auxt && (s = check_table(ctx, auxt, "auxiliary", kMaxAuxL, true)) != HF_OK) return s;
    free_shells(ctx);
    big_release(ctx, ctx->d_B, ctx->b_alloc_bytes);
    release(ctx, ctx->d_metric);
    big_release(ctx, ctx->d_bf16_b, ctx->bf16_alloc_bytes);
    ctx->built = false;
    ctx->row0 = 0;
    ctx->row1 = -1;
    schedule_release(ctx);
    std::vector<double> exps, coefs;
    auto add = [&](const hf_shell_table* t, int64_t sh, int fn) {
        DevShell d{};
        d.x = t->centers[3 * sh];
        d.y = t->centers[3 * sh + 1];
        d.z = t->centers[3 * sh + 2];
        d.l = (int)t->angular_momenta[sh];
        const int64_t p0 = t->primitive_offsets[sh], p1 = t->primitive_offsets[sh + 1];
        d.nprim = (int)(p1 - p0);
        d.ncontr = (int)t->n_contractions[sh];
        d.prim = (int)exps.size();
        d.coef = (int)coefs.size();
        d.fn = fn;
        int64_t coff = 0;
        for (int64_t q = 0; q < sh; ++q)
            coff += t->n_contractions[q] * (t->primitive_offsets[q + 1] - t->primitive_offsets[q]);
        for (int64_t i = p0; i < p1; ++i) exps.push_back(t->exponents[i]);
        for (int64_t i = 0; i < d.ncontr * d.nprim; ++i) coefs.push_back(t->coefficients[coff + i]);
        return d;
    };
    ctx->orb.clear();
    int fn = 0;
    for (int64_t sh = 0; sh < orbt->n_shells; ++sh) {
        ctx->orb.push_back(add(orbt, sh, fn));
        fn += ctx->orb.back().ncontr * nsph(ctx->orb.back().l);
    }
    ctx->n = fn;
    // auxiliary: reference function offsets, then internal order sorted by l
    static const hf_shell_table kNoShells{};
    if (!auxt) auxt = &kNoShells;
    std::vector<int> ref_off(auxt->n_shells);
    int rf = 0;
    for (int64_t sh = 0; sh < auxt->n_shells; ++sh) {
        ref_off[sh] = rf;
        rf += (int)auxt->n_contractions[sh] * nsph((int)auxt->angular_momenta[sh]);
    }
    ctx->aux.clear();
    ctx->aux_ref_fn.clear();
    std::vector<std::vector<int>> by_l(kMaxAuxL + 1);
    int q = 0;
    for (int l = 0; l <= kMaxAuxL; ++l)
        for (int64_t sh = 0; sh < auxt->n_shells; ++sh) {
            if (auxt->angular_momenta[sh] != l) continue;
            by_l[l].push_back((int)ctx->aux.size());
            ctx->aux.push_back(add(auxt, sh, q));
            for (int m = 0; m < nsph(l); ++m) ctx->aux_ref_fn.push_back(ref_off[sh] + m);
            q += nsph(l);
        }
    ctx->naux = q;
    ctx->nt = (ctx->n + 63) / 64;
    ctx->ntiles = (int64_t)ctx->nt * (ctx->nt + 1) / 2;
    if (alloc(ctx, (void**)&ctx->d_orb, sizeof(DevShell) * ctx->orb.size()) ||
        alloc(ctx, (void**)&ctx->d_aux, sizeof(DevShell) * std::max<size_t>(1, ctx->aux.size())) ||
        alloc(ctx, (void**)&ctx->d_exps, sizeof(double) * exps.size()) ||
        alloc(ctx, (void**)&ctx->d_coefs, sizeof(double) * coefs.size()))
        return HF_ERR_OOM;
    HF_CU(cudaMemcpyAsync(ctx->d_orb, ctx->orb.data(), sizeof(DevShell) * ctx->orb.size(), cudaMemcpyHostToDevice,
                          ctx->stream));
    if (!ctx->aux.empty())
        HF_CU(cudaMemcpyAsync(ctx->d_aux, ctx->aux.data(), sizeof(DevShell) * ctx->aux.size(), cudaMemcpyHostToDevice,
                              ctx->stream));
    HF_CU(cudaMemcpyAsync(ctx->d_exps, exps.data(), sizeof(double) * exps.size(), cudaMemcpyHostToDevice, ctx->stream));
    ctx->h_exps = exps;
    ctx->h_coefs = coefs;
    HF_CU(cudaMemcpyAsync(ctx->d_coefs, coefs.data(), sizeof(double) * coefs.size(), cudaMemcpyHostToDevice,
                          ctx->stream));
    for (int l = 0; l <= kMaxAuxL; ++l) {
        ctx->aux_count[l] = (int)by_l[l].size();
        if (alloc(ctx, (void**)&ctx->d_aux_by_l[l], sizeof(int) * std::max<size_t>(1, by_l[l].size()))) return HF_ERR_OOM;
        if (!by_l[l].empty())
            HF_CU(cudaMemcpyAsync(ctx->d_aux_by_l[l], by_l[l].data(), sizeof(int) * by_l[l].size(),
                                  cudaMemcpyHostToDevice, ctx->stream));
    }
    HF_CU(cudaStreamSynchronize(ctx->stream));
    ctx->stats.n_ao = ctx->n;
    ctx->stats.n_aux = ctx->naux;
    ctx->stats.n_tiles = ctx->ntiles;
    ctx->uploaded = true;
    return HF_OK;
}

int hf_dims(const hf_ctx* ctx, int64_t* n_ao, int64_t* n_aux) {
    if (!ctx || !ctx->uploaded) return HF_ERR_STATE;
    if (n_ao) *n_ao = ctx->n;
    if (n_aux) *n_aux = ctx->naux;
    return HF_OK;
}

// (P|Q) into d_metric (internal order).
static int build_metric(hf_ctx* ctx) {
    const size_t bytes = sizeof(double) * (size_t)ctx->naux * ctx->naux;
    if (!ctx->d_metric && alloc(ctx, (void**)&ctx->d_metric, bytes)) return HF_ERR_OOM;
    HF_CU(launch_metric(ctx->d_aux, ctx->d_exps, ctx->d_coefs, ctx->d_aux_by_l, ctx->aux_count, ctx->d_btable,
                        ctx->d_metric, ctx->naux, ctx->stream));
    ctx->stats.kernel_launches += 25;
    return check_async(ctx, "metric");
}

// The screening bound of integrals.cu for a whole shell pair: the largest
// |c_a c_b| exp(-mu R_AB^2) over its primitive pairs.
static double pair_bound(const hf_ctx* ctx, const DevShell& A, const DevShell& B, const std::vector<double>& exps,
                         const std::vector<double>& coefs) {
    const double dx = A.x - B.x, dy = A.y - B.y, dz = A.z - B.z;
    const double r2 = dx * dx + dy * dy + dz * dz;
    double best = 0.0;
    for (int i = 0; i < A.nprim; ++i)
        for (int j = 0; j < B.nprim; ++j) {
            const double a = exps[A.prim + i], b = exps[B.prim + j];
            const double e = std::exp(-a * b / (a + b) * r2);
            double cmax = 0.0;
            for (int ka = 0; ka < A.ncontr; ++ka)
                for (int kb = 0; kb < B.ncontr; ++kb)
                    cmax = std::max(cmax, std::fabs(coefs[A.coef + ka * A.nprim + i] * coefs[B.coef + kb * B.nprim + j]));
            best = std::max(best, cmax * e);
        }
    (void)ctx;
    return best;
}

// Every shell pair (a <= b) with at least one primitive pair above the screening
// bound, listed by its first shell; the host threads split the first shells.
static std::vector<std::vector<PairTask>> screen_pairs(const hf_ctx* ctx) {
    const int ns = (int)ctx->orb.size();
    std::vector<std::vector<PairTask>> by_a(ns);
    auto work = [&](int begin, int step) {
        for (int a = begin; a < ns; a += step) {
            const DevShell& A = ctx->orb[a];
            for (int b = a; b < ns; ++b) {
                const DevShell& B = ctx->orb[b];
                if (pair_bound(ctx, A, B, ctx->h_exps, ctx->h_coefs) < 1e-22) continue;
                by_a[a].push_back(PairTask{a, b, A.l > B.l ? 1 : 0, 0});
            }
        }
    };
    // a thread per 64 first shells, at most 16: small molecules are screened on the
    // calling thread (many of them are built at once by the batched SCF's threads)
    const int nthreads = std::max(1, std::min({16, (int)std::thread::hardware_concurrency(), ns / 64}));
    std::vector<std::thread> pool;
    for (int t = 1; t < nthreads; ++t) pool.emplace_back(work, t, nthreads);
    work(0, nthreads);
    for (auto& t : pool) t.join();
    return by_a;
}

// Pair tasks for tile rows [row0, row1): the screened pairs whose first shell
// touches those rows, bucketed by (la <= lb).
static void chunk_tasks_from(const hf_ctx* ctx, const std::vector<std::vector<PairTask>>& by_a, int row0, int row1,
                             std::vector<PairTask> (&tasks)[3][3], int (&max_npp)[3][3]) {
    for (auto& r : tasks)
        for (auto& v : r) v.clear();
    for (auto& r : max_npp)
        for (auto& v : r) v = 0;
    const int ns = (int)ctx->orb.size();
    for (int a = 0; a < ns; ++a) {
        const DevShell& A = ctx->orb[a];
        const int f0 = A.fn, f1 = A.fn + A.ncontr * nsph(A.l) - 1;
        if ((f1 >> 6) < row0 || (f0 >> 6) >= row1) continue;
        for (const PairTask& t : by_a[a]) {
            const DevShell& B = ctx->orb[t.second];
            const int la = std::min(A.l, B.l), lb = std::max(A.l, B.l);
            tasks[la][lb].push_back(t);
            max_npp[la][lb] = std::max(max_npp[la][lb], A.nprim * B.nprim);
        }
    }
}

static void chunk_tasks(const hf_ctx* ctx, int row0, int row1, std::vector<PairTask> (&tasks)[3][3],
                        int (&max_npp)[3][3]) {
    chunk_tasks_from(ctx, screen_pairs(ctx), row0, row1, tasks, max_npp);
}

// Three-centre integrals of tile rows [row0, row1) into T ([cols][naux]).
static int three_center_chunk(hf_ctx* ctx, int row0, int row1, double* T, PairTask* d_tasks, size_t task_cap) {
    std::vector<PairTask> tasks[3][3];
    int max_npp[3][3];
    chunk_tasks(ctx, row0, row1, tasks, max_npp);
    ChunkDesc cd{row0, row1, ctx->nt, tile_index(row0, row0, ctx->nt), ctx->naux};
    size_t off = 0;
    for (int la = 0; la <= 2; ++la)
        for (int lb = la; lb <= 2; ++lb) {
            auto& v = tasks[la][lb];
            if (v.empty()) continue;
            if (off + v.size() > task_cap) return fail(ctx, HF_ERR_STATE, "task buffer too small");
            HF_CU(cudaMemcpyAsync(d_tasks + off, v.data(), sizeof(PairTask) * v.size(), cudaMemcpyHostToDevice,
                                  ctx->stream));
            HF_CU(launch_three_center(la, lb, d_tasks + off, (int)v.size(), max_npp[la][lb], ctx->d_orb, ctx->d_aux,
                                      ctx->d_exps, ctx->d_coefs, ctx->d_aux_by_l, ctx->aux_count, ctx->d_btable, cd,
                                      T, ctx->stream));
            ctx->stats.kernel_launches += 5;
            off += v.size();
        }
    // the host task vectors must outlive the async copies
    HF_CU(cudaStreamSynchronize(ctx->stream));
    return HF_OK;
}

int hf_build_fitted_tensor(hf_ctx* ctx) {
    if (!ctx) return HF_ERR_ARG;
    if (!ctx->uploaded) return fail(ctx, HF_ERR_STATE, "upload shells first");
    if (ctx->naux == 0) return fail(ctx, HF_ERR_STATE, "no auxiliary shells were uploaded");
    cudaSetDevice(ctx->device);
    const int N = ctx->naux;
    int s;
    // the host screens the shell pairs while the device builds and factors the metric
    auto screened = std::async(std::launch::async, [ctx]() { return screen_pairs(ctx); });
    time_begin(ctx);
    if ((s = build_metric(ctx)) != HF_OK) return s;
    ctx->stats.ms_metric = time_end(ctx);

    // Cholesky + inverse of the factor.
    time_begin(ctx);
    double *L = nullptr, *Linv = nullptr, *LinvT = nullptr, *wk = nullptr;
    const size_t nn = (size_t)N * N;
    if (talloc(ctx, (void**)&L, nn * 8) || talloc(ctx, (void**)&Linv, nn * 8) || talloc(ctx, (void**)&LinvT, nn * 8) ||
        talloc(ctx, (void**)&wk, (size_t)N * 64 * 8)) {
        trelease(ctx, L);
        trelease(ctx, Linv);
        trelease(ctx, LinvT);
        trelease(ctx, wk);
        return HF_ERR_OOM;
    }
    HF_CU(cudaMemcpyAsync(L, ctx->d_metric, nn * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    HF_CU(cudaMemsetAsync(ctx->d_info, 0, sizeof(int), ctx->stream));
    const double big = 1e300;
    HF_CU(cudaMemcpyAsync(ctx->d_scalar, &big, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    HF_CU(cholesky_lower(L, N, N, ctx->d_info, ctx->d_scalar, ctx->stream));
    int info = 0;
    double pivmin = 0.0;
    HF_CU(cudaMemcpyAsync(&info, ctx->d_info, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    HF_CU(cudaMemcpyAsync(&pivmin, ctx->d_scalar, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    HF_CU(cudaStreamSynchronize(ctx->stream));
    if (info != 0) {
        trelease(ctx, L);
        trelease(ctx, Linv);
        trelease(ctx, LinvT);
        trelease(ctx, wk);
        return fail(ctx, HF_ERR_NUMERIC, "the Coulomb metric is not positive definite (pivot " + std::to_string(info - 1) +
                                             ")");
    }
    {
        std::vector<double> diag(N);
        HF_CU(cudaMemcpy2D(diag.data(), sizeof(double), ctx->d_metric, sizeof(double) * ((size_t)N + 1), sizeof(double),
                           N, cudaMemcpyDeviceToHost));
        const double dmax = *std::max_element(diag.begin(), diag.end());
        ctx->stats.min_pivot_ratio = pivmin * pivmin / dmax;
    }
    HF_CU(triangular_inverse(L, N, N, Linv, LinvT, wk, ctx->stream));
    if ((s = check_async(ctx, "inverse factor")) != HF_OK) return s;
    ctx->stats.ms_factor = time_end(ctx);
    trelease(ctx, L);
    trelease(ctx, LinvT);
    trelease(ctx, wk);

    // B = L^-1 (P|mu nu), chunked over tile rows.
    big_release(ctx, ctx->d_B, ctx->b_alloc_bytes);
    const int64_t ldb = ctx->ntiles * 4096;
    // the auxiliary rows [q_begin, q_end) this context holds
    const int rows = fitted_rows(ctx), q_begin = ctx->row0, q_end = q_begin + rows;
    if (big_alloc(ctx, (void**)&ctx->d_B, sizeof(double) * (size_t)rows * ldb, &ctx->b_alloc_bytes)) {
        trelease(ctx, Linv);
        return HF_ERR_OOM;
    }
    ctx->stats.b_bytes = (int64_t)sizeof(double) * rows * ldb;
    // Chunks of tile rows whose three-centre integrals fit one buffer; each chunk's
    // integrals, then its fit. (Running the integrals of the next chunk beside the
    // fit of this one, on a second stream, measured no faster at (H2O)64: both
    // need the FP64 units.)
    const size_t row_bytes = sizeof(double) * 4096 * (size_t)N * ctx->nt;  // the widest row
    size_t budget = std::max<size_t>(row_bytes, (size_t)4 << 30);
    budget = std::min<size_t>(budget, sizeof(double) * 4096 * (size_t)N * ctx->ntiles);
    size_t freeb = 0, totalb = 0;
    cudaMemGetInfo(&freeb, &totalb);
    if (budget > freeb / 2) budget = std::max(row_bytes, freeb / 2);
    std::vector<std::pair<int, int>> chunks;
    for (int row0 = 0; row0 < ctx->nt;) {
        int row1 = row0 + 1;
        while (row1 < ctx->nt &&
               sizeof(double) * 4096 * (size_t)N * (tile_index(row1 + 1, row1 + 1, ctx->nt) - tile_index(row0, row0, ctx->nt)) <= budget)
            ++row1;
        chunks.push_back({row0, row1});
        row0 = row1;
    }
    // every chunk's pair tasks, built on the host first and copied in one go
    struct Launch {
        int la, lb, max_npp;
        size_t off, count;
    };
    std::vector<std::vector<Launch>> launches(chunks.size());
    std::vector<PairTask> all_tasks;
    const std::vector<std::vector<PairTask>> by_a = screened.get();
    for (size_t c = 0; c < chunks.size(); ++c) {
        std::vector<PairTask> tasks[3][3];
        int max_npp[3][3];
        chunk_tasks_from(ctx, by_a, chunks[c].first, chunks[c].second, tasks, max_npp);
        for (int la = 0; la <= 2; ++la)
            for (int lb = la; lb <= 2; ++lb) {
                const auto& v = tasks[la][lb];
                if (v.empty()) continue;
                launches[c].push_back(Launch{la, lb, max_npp[la][lb], all_tasks.size(), v.size()});
                all_tasks.insert(all_tasks.end(), v.begin(), v.end());
            }
    }
    double* T = nullptr;
    PairTask* d_tasks = nullptr;
    if (talloc(ctx, (void**)&d_tasks, sizeof(PairTask) * std::max<size_t>(1, all_tasks.size())) ||
        talloc(ctx, (void**)&T, budget)) {
        trelease(ctx, T);
        trelease(ctx, d_tasks);
        trelease(ctx, Linv);
        return HF_ERR_OOM;
    }
    if (!all_tasks.empty())
        HF_CU(cudaMemcpyAsync(d_tasks, all_tasks.data(), sizeof(PairTask) * all_tasks.size(), cudaMemcpyHostToDevice,
                              ctx->stream));
    // per chunk: start, integrals done, fit done (timing only; one stream)
    const size_t nc = chunks.size();
    std::vector<cudaEvent_t> ev(3 * nc, nullptr);
    for (auto& x : ev) cudaEventCreate(&x);
    cudaError_t e = cudaSuccess;
    for (size_t c = 0; c < nc && e == cudaSuccess; ++c) {
        const int row0 = chunks[c].first, row1 = chunks[c].second;
        const int64_t t0 = tile_index(row0, row0, ctx->nt), t1 = tile_index(row1, row1, ctx->nt);
        const int64_t ncols = (t1 - t0) * 4096;
        cudaEventRecord(ev[3 * c], ctx->stream);
        e = cudaMemsetAsync(T, 0, sizeof(double) * (size_t)ncols * N, ctx->stream);
        const ChunkDesc cd{row0, row1, ctx->nt, t0, ctx->naux};
        for (const Launch& l : launches[c]) {
            if (e != cudaSuccess) break;
            e = launch_three_center(l.la, l.lb, d_tasks + l.off, (int)l.count, l.max_npp, ctx->d_orb, ctx->d_aux,
                                    ctx->d_exps, ctx->d_coefs, ctx->d_aux_by_l, ctx->aux_count, ctx->d_btable, cd, T,
                                    ctx->stream);
            ctx->stats.kernel_launches += 5;
        }
        cudaEventRecord(ev[3 * c + 1], ctx->stream);
        if (e == cudaSuccess)
            e = apply_inverse_factor(Linv, N, N, T, N, ncols, ctx->d_B + t0 * 4096, ldb, ctx->stream, q_begin, q_end);
        ++ctx->stats.kernel_launches;
        cudaEventRecord(ev[3 * c + 2], ctx->stream);
    }
    cudaError_t se = cudaStreamSynchronize(ctx->stream);  // the host task vector outlives its copy
    if (e == cudaSuccess) e = se;
    if (e == cudaSuccess) e = cudaGetLastError();
    double ms3c = 0.0, msfit = 0.0;
    if (e == cudaSuccess)
        for (size_t c = 0; c < nc; ++c) {
            float a = 0.f, b = 0.f;
            cudaEventElapsedTime(&a, ev[3 * c], ev[3 * c + 1]);
            cudaEventElapsedTime(&b, ev[3 * c + 1], ev[3 * c + 2]);
            ms3c += a;
            msfit += b;
        }
    for (auto& x : ev) cudaEventDestroy(x);
    trelease(ctx, T);
    trelease(ctx, d_tasks);
    trelease(ctx, Linv);
    if (e != cudaSuccess) return fail(ctx, HF_ERR_CUDA, std::string("fitted tensor: ") + cudaGetErrorString(e));
    HF_CU(cudaStreamSynchronize(ctx->stream));
    ctx->stats.ms_three_center = ms3c;
    ctx->stats.ms_fit = msfit;
    ctx->built = true;
    return HF_OK;
}

static JkPlan plan_of(const hf_ctx* ctx) {
    JkPlan p{};
    p.B = ctx->d_B;
    p.ldb = ctx->ntiles * 4096;
    p.n = ctx->n;
    p.nt = ctx->nt;
    p.ntiles = ctx->ntiles;
    p.naux = fitted_rows(ctx);
    return p;
}

int hf_coulomb(hf_ctx* ctx, const double* D, double* J, int on_device) {
    if (!ctx || !D || !J) return HF_ERR_ARG;
    if (!ctx->built) return fail(ctx, HF_ERR_STATE, "build the fitted tensor first");
    cudaSetDevice(ctx->device);
    const JkPlan p = plan_of(ctx);
    const size_t nn = (size_t)ctx->n * ctx->n;
    int s;
    if ((s = ensure_work(ctx, sizeof(double) * coulomb_work_doubles(p))) != HF_OK) return s;
    const double* dD = D;
    double* dJ = J;
    if (!on_device) {
        if ((s = ensure_io(ctx, 2 * nn * sizeof(double))) != HF_OK) return s;
        HF_CU(cudaMemcpyAsync(ctx->d_io, D, nn * 8, cudaMemcpyHostToDevice, ctx->stream));
        dD = ctx->d_io;
        dJ = ctx->d_io + nn;
    }
    time_begin(ctx);
    HF_CU(coulomb_build(p, dD, dJ, ctx->d_work, ctx->stream));
    ctx->stats.kernel_launches += 4;
    if (!on_device) HF_CU(cudaMemcpyAsync(J, dJ, nn * 8, cudaMemcpyDeviceToHost, ctx->stream));
    ctx->stats.ms_coulomb = time_end(ctx);
    return check_async(ctx, "hf_coulomb");
}

// K from Ct ([opad][npad], device) and sign ([opad]).
static int exchange_from_ct(hf_ctx* ctx, const double* Ct, int opad, const double* sign, bool any_negative,
                            double* dK, int precision) {
    if (precision != HF_PREC_FP64) return fail(ctx, HF_ERR_ARG, "unknown precision");
    const JkPlan p = plan_of(ctx);
    const int64_t npad = (int64_t)ctx->nt * 64;
    // X chunk: npad x qchunk x opad doubles, within a budget
    size_t freeb = 0, totalb = 0;
    cudaMemGetInfo(&freeb, &totalb);
    const size_t per_q = sizeof(double) * npad * opad * (any_negative ? 2 : 1);
    size_t budget = std::min<size_t>((size_t)4 << 30, freeb / 3);
    int qchunk = (int)std::max<size_t>(1, std::min<size_t>(budget / per_q, (size_t)p.naux));
    qchunk = std::min(qchunk, 65535);
    const size_t kp_doubles = (size_t)round_up(npad * npad, 32);
    const size_t part_doubles = (size_t)round_up(syrk_partial_doubles(npad, 1), 32);
    int st = ensure_scratch(ctx, &ctx->d_kscratch, &ctx->kscratch_bytes,
                            sizeof(double) * (kp_doubles + part_doubles) + per_q * qchunk);
    if (st != HF_OK) return st;
    double* Kp = ctx->d_kscratch;
    double* part = part_doubles ? Kp + kp_doubles : nullptr;
    double* X = Kp + kp_doubles + part_doubles;
    double* Xs = any_negative ? X + npad * (int64_t)qchunk * opad : nullptr;
    cudaError_t e = exchange_build_fp64(p, Ct, opad, any_negative ? sign : nullptr, dK, Kp, X, Xs, part, qchunk,
                                        ctx->stream);
    ctx->stats.kernel_launches += 3 * ((p.naux + qchunk - 1) / qchunk) + 2;
    if (e != cudaSuccess) return fail(ctx, HF_ERR_CUDA, std::string("exchange: ") + cudaGetErrorString(e));
    return check_async(ctx, "exchange");
}

// Split-BF16 exchange from Ct_tc ([t.opad][t.npad], FP64, zero padded) into dK (n x n);
// sign ([t.opad], device) for a signed factor, else null.
static int exchange_bf16(hf_ctx* ctx, const TcPlan& t, const double* Ct_tc, double* dK, const double* sign = nullptr) {
    const JkPlan p = plan_of(ctx);
    if (!ctx->d_bf16_b) {
        if (big_alloc(ctx, &ctx->d_bf16_b, tc_b_bytes(ctx->n, p.naux), &ctx->bf16_alloc_bytes))
            return fail(ctx, HF_ERR_OOM, "no room for the BF16 copies of the fitted tensor (" +
                                             std::to_string(tc_b_bytes(ctx->n, p.naux)) + " bytes)");
        HF_CU(tc_split_b(p, t.npad, ctx->d_bf16_b, ctx->stream));
        int s = check_async(ctx, "BF16 copy of B");
        if (s != HF_OK) {
            big_release(ctx, ctx->d_bf16_b, ctx->bf16_alloc_bytes);
            return s;
        }
    }
    size_t freeb = 0, totalb = 0;
    cudaMemGetInfo(&freeb, &totalb);
    const size_t ct_bytes = 2 * 2 * (size_t)t.opad * t.npad;
    const size_t per_q = (sign ? 4 : 2) * 2 * (size_t)t.npad * t.opad;
    const size_t kp_doubles = (size_t)round_up(t.npad * t.npad, 32);
    size_t budget = std::min<size_t>((size_t)2 << 30, freeb / 3);
    size_t want = round_up((int64_t)ct_bytes, 256) + tc_partial_bytes(t.npad) +
                  per_q * std::max<size_t>(1, std::min<size_t>(budget / per_q, (size_t)p.naux));
    want = round_up((int64_t)want, 256) + sizeof(double) * kp_doubles;
    int st = ensure_scratch(ctx, &ctx->d_tcwork, &ctx->tcwork_bytes, want);
    if (st != HF_OK) return st;
    double* Kp = ctx->d_tcwork;
    void* work = ctx->d_tcwork + kp_doubles;
    HF_CU(cudaMemsetAsync(ctx->d_info + 2, 0, sizeof(int), ctx->stream));
    const TcWait wait{ctx->d_info + 2, ctx->wait_ns, ctx->stall_next};
    ctx->stall_next = 0;
    cudaError_t e = exchange_build_bf16(t, ctx->d_bf16_b, Ct_tc, t.npad, dK, Kp, work, want - sizeof(double) * kp_doubles,
                                        wait, ctx->stream, ctx->n, sign);
    ctx->stats.kernel_launches += 3 * ((p.naux + 1023) / 1024) + 3;
    if (e != cudaSuccess) return fail(ctx, HF_ERR_CUDA, std::string("split-BF16 exchange: ") + cudaGetErrorString(e));
    int s = check_async(ctx, "split-BF16 exchange");
    if (s != HF_OK) return s;
    int flag = 0;
    HF_CU(cudaMemcpy(&flag, ctx->d_info + 2, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) return fail(ctx, HF_ERR_TIMEOUT, "split-BF16 exchange: a pipeline wait ran out (code " +
                                                   std::to_string(flag) + ")");
    return HF_OK;
}

int hf_exchange_factored(hf_ctx* ctx, const double* C, int64_t ncols, const double* w, double* K, int precision,
                         int on_device) {
    if (!ctx || !C || !K || ncols < 0) return HF_ERR_ARG;
    if (!ctx->built) return fail(ctx, HF_ERR_STATE, "build the fitted tensor first");
    cudaSetDevice(ctx->device);
    const int64_t n = ctx->n, npad = (int64_t)ctx->nt * 64;
    const int64_t opad = std::max<int64_t>(64, round_up(ncols, 64));
    bool neg = false;
    std::vector<double> wh;
    const double* dC = C;
    const double* dw = w;
    Carver cv;
    const size_t oC = cv.take(n * ncols), ow = cv.take(ncols), oCt = cv.take(opad * npad), osg = cv.take(opad),
                 oK = cv.take(n * n);
    int st = ensure_scratch(ctx, &ctx->d_stage, &ctx->stage_bytes, sizeof(double) * cv.used);
    if (st != HF_OK) return st;
    double* buf = ctx->d_stage;
    double* sC = buf + oC;
    double* sw = buf + ow;
    double* Ct = buf + oCt;
    double* sign = buf + osg;
    double* sK = buf + oK;
    if (w) {
        wh.resize(ncols);
        if (on_device) cudaMemcpy(wh.data(), w, sizeof(double) * ncols, cudaMemcpyDeviceToHost);
        else std::memcpy(wh.data(), w, sizeof(double) * ncols);
        for (double v : wh) neg = neg || v < 0.0;
    }
    if (!on_device) {
        cudaMemcpyAsync(sC, C, sizeof(double) * n * ncols, cudaMemcpyHostToDevice, ctx->stream);
        if (w) cudaMemcpyAsync(sw, w, sizeof(double) * ncols, cudaMemcpyHostToDevice, ctx->stream);
        dC = sC;
        dw = w ? sw : nullptr;
    }
    if (precision == HF_PREC_BF16X3) {
        const TcPlan t = tc_plan(n, fitted_rows(ctx), ncols);
        int sc = ensure_scratch(ctx, &ctx->d_ctc, &ctx->ctc_bytes, sizeof(double) * ((size_t)t.opad * t.npad + t.opad));
        if (sc != HF_OK) return sc;
        double* Ct_tc = ctx->d_ctc;
        time_begin(ctx);
        k_factor_transpose<<<(unsigned)((t.opad * t.npad + 255) / 256), 256, 0, ctx->stream>>>(
            dC, n, ncols, dw, Ct_tc, t.npad, t.opad, Ct_tc + (size_t)t.opad * t.npad);
        double* dK = on_device ? K : sK;
        int s = exchange_bf16(ctx, t, Ct_tc, dK, neg ? Ct_tc + (size_t)t.opad * t.npad : nullptr);
        if (s == HF_OK && !on_device) cudaMemcpyAsync(K, sK, sizeof(double) * n * n, cudaMemcpyDeviceToHost, ctx->stream);
        ctx->stats.ms_exchange = time_end(ctx);
        ctx->stats.exchange_rank = ncols;
        if (s == HF_OK) s = check_async(ctx, "hf_exchange_factored");
        return s;
    }
    time_begin(ctx);
    k_factor_transpose<<<(unsigned)((opad * npad + 255) / 256), 256, 0, ctx->stream>>>(dC, n, ncols, dw, Ct, npad, opad,
                                                                                        sign);
    double* dK = on_device ? K : sK;
    int s = exchange_from_ct(ctx, Ct, (int)opad, sign, neg, dK, precision);
    if (s == HF_OK && !on_device) cudaMemcpyAsync(K, sK, sizeof(double) * n * n, cudaMemcpyDeviceToHost, ctx->stream);
    ctx->stats.ms_exchange = time_end(ctx);
    ctx->stats.exchange_rank = ncols;
    if (s == HF_OK) s = check_async(ctx, "hf_exchange_factored");
    return s;
}

int hf_schedule_reset(hf_ctx* ctx) {
    if (!ctx) return HF_ERR_ARG;
    ScheduleState& st = ctx->sched;
    st.phase = 0;
    st.has_prev = false;
    st.anchor_rank = 0;
    return HF_OK;
}

int hf_exchange_scheduled(hf_ctx* ctx, const double* D, double* K, int on_device, const hf_schedule* sc, int* kind) {
    if (!ctx || !D || !K || !sc) return HF_ERR_ARG;
    if (!ctx->built) return fail(ctx, HF_ERR_STATE, "build the fitted tensor first");
    if (sc->mode == HF_SCHEDULE_FP64) {
        if (kind) *kind = HF_BUILD_FP64;
        return hf_exchange(ctx, D, K, HF_PREC_FP64, on_device);
    }
    if (sc->mode != HF_SCHEDULE_MIXED) return fail(ctx, HF_ERR_ARG, "unknown schedule mode");
    if (!(sc->anchor_change > 0.0) || !(sc->final_change > 0.0) || sc->final_change > sc->anchor_change)
        return fail(ctx, HF_ERR_ARG, "the schedule needs 0 < final_change <= anchor_change");
    cudaSetDevice(ctx->device);
    const int64_t n = ctx->n;
    const size_t nn = (size_t)n * n, bytes = sizeof(double) * nn;
    ScheduleState& st = ctx->sched;
    for (double** q : {&st.prev, &st.anchor_d, &st.anchor_k, &st.anchor_ft, &st.dens, &st.ft, &st.overlap})
        if (!*q && alloc(ctx, (void**)q, bytes)) return HF_ERR_OOM;
    for (auto& q : st.work)
        if (!q && alloc(ctx, (void**)&q, bytes)) return HF_ERR_OOM;
    if (!st.scalar && alloc(ctx, (void**)&st.scalar, sizeof(double) * (2 * (size_t)n + 8))) return HF_ERR_OOM;
    int s;
    if (!st.overlap_ready) {
        if ((s = hf_one_electron(ctx, 0, nullptr, nullptr, 0, st.overlap, 1)) != HF_OK) return s;
        st.overlap_ready = true;
    }
    const double* dD = D;
    if (!on_device) {
        HF_CU(cudaMemcpyAsync(st.dens, D, bytes, cudaMemcpyHostToDevice, ctx->stream));
        dD = st.dens;
    }
    // the largest element change from the previous call's density
    double delta = INFINITY;
    if (st.has_prev && (s = device_maxabs(ctx, dD, st.prev, (int64_t)nn, false, 0, &delta)) != HF_OK) return s;
    HF_CU(cudaMemcpyAsync(st.prev, dD, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    st.has_prev = true;
    if (delta >= sc->anchor_change) st.phase = 0;
    // D ~= F F^T, F^T in st.ft ([rank][n])
    int64_t rank = 0;
    if ((s = hf_density_factor(ctx, dD, st.ft, n, &rank, 1)) != HF_OK) return s;
    double* const* w = st.work;
    double* kout = on_device ? K : w[9];
    if (rank == 0) {  // D = 0: K = 0 exactly
        HF_CU(cudaMemsetAsync(kout, 0, bytes, ctx->stream));
        if (kind) *kind = HF_BUILD_FP64;
        if (!on_device) HF_CU(cudaMemcpyAsync(K, kout, bytes, cudaMemcpyDeviceToHost, ctx->stream));
        return check_async(ctx, "hf_exchange_scheduled");
    }
    const unsigned tb = blocks_for(rank * n);
    auto build_from_factor = [&](int precision) -> int {
        k_transpose_plain<<<tb, 256, 0, ctx->stream>>>(st.ft, rank, n, w[0]);  // F, [n][rank]
        return hf_exchange_factored(ctx, w[0], rank, nullptr, kout, precision, 1);
    };
    auto anchor = [&]() -> int {
        int r2 = build_from_factor(HF_PREC_FP64);
        if (r2 != HF_OK) return r2;
        HF_CU(cudaMemcpyAsync(st.anchor_d, dD, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
        HF_CU(cudaMemcpyAsync(st.anchor_ft, st.ft, sizeof(double) * rank * n, cudaMemcpyDeviceToDevice, ctx->stream));
        HF_CU(cudaMemcpyAsync(st.anchor_k, kout, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
        st.anchor_rank = rank;
        st.phase = 1;
        if (kind) *kind = HF_BUILD_ANCHOR;
        return HF_OK;
    };
    // K64(D_a) + K16(V+) - K16(V-) for D - D_a = V+ V+^T - V- V-^T; an anchor when the
    // rotation of the anchor's factor onto this one does not converge
    auto increment = [&]() -> int {
        const int64_t r = std::max(rank, st.anchor_rank);
        double *fnt = w[1], *fat = w[2], *t1t = w[3], *x = w[4], *xt = w[5], *y = w[6], *z = w[7], *xn = w[8];
        // the two factors' transposes, zero padded to r rows
        HF_CU(cudaMemsetAsync(fnt, 0, sizeof(double) * r * n, ctx->stream));
        HF_CU(cudaMemsetAsync(fat, 0, sizeof(double) * r * n, ctx->stream));
        HF_CU(cudaMemcpyAsync(fnt, st.ft, sizeof(double) * rank * n, cudaMemcpyDeviceToDevice, ctx->stream));
        HF_CU(cudaMemcpyAsync(fat, st.anchor_ft, sizeof(double) * st.anchor_rank * n, cudaMemcpyDeviceToDevice,
                              ctx->stream));
        // M = F_a^T S F: T1^T = F^T S (S symmetric), then M = F_a^T (T1^T)^T
        HF_CU(gemm_nt(ctx, r, n, n, fnt, n, st.overlap, n, t1t, n, 1.0));
        HF_CU(gemm_nt(ctx, r, r, n, fat, n, t1t, n, x, r, 1.0));
        // its orthogonal polar factor: X <- X (3 I - X^T X) / 2
        const unsigned rb = blocks_for(r * r);
        for (int it = 0; it < 8; ++it) {
            k_transpose_plain<<<rb, 256, 0, ctx->stream>>>(x, r, r, xt);
            HF_CU(gemm_nt(ctx, r, r, r, xt, r, xt, r, y, r, 1.0));  // X^T X
            k_three_minus<<<rb, 256, 0, ctx->stream>>>(y, r, z);
            HF_CU(gemm_nt(ctx, r, r, r, x, r, z, r, xn, r, 0.5));   // X Z / 2 (Z symmetric)
            std::swap(x, xn);
        }
        k_transpose_plain<<<rb, 256, 0, ctx->stream>>>(x, r, r, xt);
        HF_CU(gemm_nt(ctx, r, r, r, xt, r, xt, r, y, r, 1.0));
        double orth = INFINITY;
        int r2 = device_maxabs(ctx, y, nullptr, 0, true, r, &orth);
        if (r2 != HF_OK) return r2;
        if (!(orth < 1e-13)) return anchor();
        // F_a X: with F_a = (F_a^T)^T in t1t ([n][r]), (F_a X)^T = X^T F_a^T -> [r][n]
        k_transpose_plain<<<blocks_for(r * n), 256, 0, ctx->stream>>>(fat, r, n, t1t);
        double* frt = y;  // [r][n]
        HF_CU(gemm_nt(ctx, r, n, r, xt, r, t1t, r, frt, n, 1.0));
        double* at = z;   // A^T = F^T + (F_a X)^T
        double* bt = xt;  // B^T = F^T - (F_a X)^T
        double* norms = st.scalar + 8;
        k_sum_diff_norms<<<(unsigned)r, 256, 0, ctx->stream>>>(fnt, frt, n, at, bt, norms, norms + r);
        double *vp = w[0], *vm = w[1];
        k_difference_factors<<<blocks_for(n * r), 256, 0, ctx->stream>>>(at, bt, norms, norms + r, r, n, vp, vm);
        double *kp = w[2], *km = w[3];
        if ((r2 = hf_exchange_factored(ctx, vp, r, nullptr, kp, HF_PREC_BF16X3, 1)) != HF_OK) return r2;
        if ((r2 = hf_exchange_factored(ctx, vm, r, nullptr, km, HF_PREC_BF16X3, 1)) != HF_OK) return r2;
        k_combine<<<blocks_for((int64_t)nn), 256, 0, ctx->stream>>>(st.anchor_k, kp, km, (int64_t)nn, kout);
        if (kind) *kind = HF_BUILD_INCREMENTAL;
        return HF_OK;
    };
    if (st.phase == 0) {
        if (delta < sc->anchor_change) {
            s = anchor();
        } else {
            s = build_from_factor(HF_PREC_BF16X3);
            if (s == HF_OK && kind) *kind = HF_BUILD_BF16;
        }
    } else {
        double distance = 0.0;
        if ((s = device_maxabs(ctx, dD, st.anchor_d, (int64_t)nn, false, 0, &distance)) != HF_OK) return s;
        s = (delta < sc->final_change && distance > sc->final_change) ? anchor() : increment();
    }
    if (s != HF_OK) return s;
    if (!on_device) HF_CU(cudaMemcpyAsync(K, kout, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    return check_async(ctx, "hf_exchange_scheduled");
}

int hf_density_factor(hf_ctx* ctx, const double* D, double* F, int64_t max_rank, int64_t* rank, int on_device) {
    if (!ctx || !D || !F || !rank || max_rank < 1) return HF_ERR_ARG;
    if (!ctx->uploaded) return fail(ctx, HF_ERR_STATE, "upload shells first");
    cudaSetDevice(ctx->device);
    const int64_t n = ctx->n;
    const size_t nn = (size_t)n * n;
    const int64_t cap = std::min<int64_t>(max_rank, n);
    Carver cv;
    const size_t oD = cv.take(nn), oL = cv.take((size_t)cap * n),
                 oW = cv.take(pivoted_cholesky_work_doubles((int)n));
    int st = ensure_scratch(ctx, &ctx->d_stage, &ctx->stage_bytes, sizeof(double) * cv.used);
    if (st != HF_OK) return st;
    double* sD = ctx->d_stage + oD;
    double* Lc = on_device ? F : ctx->d_stage + oL;
    const double* dD = D;
    if (!on_device) {
        HF_CU(cudaMemcpyAsync(sD, D, sizeof(double) * nn, cudaMemcpyHostToDevice, ctx->stream));
        dD = sD;
    }
    time_begin(ctx);
    HF_CU(cudaMemsetAsync(ctx->d_info, 0, 2 * sizeof(int), ctx->stream));
    HF_CU(pivoted_cholesky_blocked(dD, (int)n, 1e-14, (int)cap, Lc, ctx->d_info, ctx->d_stage + oW, ctx->stream));
    ++ctx->stats.kernel_launches;
    int res[2] = {0, 0};
    HF_CU(cudaMemcpyAsync(res, ctx->d_info, sizeof(res), cudaMemcpyDeviceToHost, ctx->stream));
    HF_CU(cudaStreamSynchronize(ctx->stream));
    ctx->stats.ms_factorize_density = time_end(ctx);
    if (res[1])
        return fail(ctx, HF_ERR_NUMERIC, "the density is not positive semidefinite");
    *rank = res[0];
    if (!on_device) {
        HF_CU(cudaMemcpyAsync(F, Lc, sizeof(double) * (size_t)res[0] * n, cudaMemcpyDeviceToHost, ctx->stream));
        return check_async(ctx, "hf_density_factor");
    }
    return HF_OK;
}

int hf_exchange(hf_ctx* ctx, const double* D, double* K, int precision, int on_device) {
    if (!ctx || !D || !K) return HF_ERR_ARG;
    if (!ctx->built) return fail(ctx, HF_ERR_STATE, "build the fitted tensor first");
    cudaSetDevice(ctx->device);
    const int64_t n = ctx->n, npad = (int64_t)ctx->nt * 64;
    const size_t nn = (size_t)n * n;
    const int64_t opad_max = std::max<int64_t>(64, round_up(n, 64));
    Carver cv;
    const size_t oD = cv.take(nn), oL = cv.take(nn), oK = cv.take(nn), oCt = cv.take(opad_max * npad),
                 osg = cv.take(opad_max), oW = cv.take(pivoted_cholesky_work_doubles((int)n));
    int st = ensure_scratch(ctx, &ctx->d_stage, &ctx->stage_bytes, sizeof(double) * cv.used);
    if (st != HF_OK) return st;
    double* buf = ctx->d_stage;
    double* sD = buf + oD;
    double* Lc = buf + oL;
    double* sK = buf + oK;
    const double* dD = D;
    if (!on_device) {
        cudaMemcpyAsync(sD, D, sizeof(double) * nn, cudaMemcpyHostToDevice, ctx->stream);
        dD = sD;
    }
    time_begin(ctx);
    cudaMemsetAsync(ctx->d_info, 0, 2 * sizeof(int), ctx->stream);
    HF_CU(pivoted_cholesky_blocked(dD, (int)n, 1e-14, (int)n, Lc, ctx->d_info, buf + oW, ctx->stream));
    int res[2] = {0, 0};
    cudaMemcpyAsync(res, ctx->d_info, sizeof(res), cudaMemcpyDeviceToHost, ctx->stream);
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    ctx->stats.ms_factorize_density = time_end(ctx);
    if (e != cudaSuccess) return fail(ctx, HF_ERR_CUDA, std::string("pivoted Cholesky: ") + cudaGetErrorString(e));
    if (res[1])
        return fail(ctx, HF_ERR_NUMERIC, "the density is not positive semidefinite; pass a signed factor to "
                                         "hf_exchange_factored");
    const int64_t rank = res[0];
    if (precision == HF_PREC_BF16X3) {
        const TcPlan t = tc_plan(n, fitted_rows(ctx), rank);
        int sc = ensure_scratch(ctx, &ctx->d_ctc, &ctx->ctc_bytes, sizeof(double) * ((size_t)t.opad * t.npad + t.opad));
        if (sc != HF_OK) return sc;
        double* Ct_tc = ctx->d_ctc;
        time_begin(ctx);
        const cudaError_t fe = factor_pad(Lc, 0, n, ctx->d_info, Ct_tc, 0, t.npad, t.opad,
                                          Ct_tc + (size_t)t.opad * t.npad, 1, nullptr, ctx->stream);
        double* dK = on_device ? K : sK;
        int s = fe == cudaSuccess ? exchange_bf16(ctx, t, Ct_tc, dK)
                                  : fail(ctx, HF_ERR_CUDA, std::string("factor_pad: ") + cudaGetErrorString(fe));
        if (s == HF_OK && !on_device) cudaMemcpyAsync(K, sK, sizeof(double) * nn, cudaMemcpyDeviceToHost, ctx->stream);
        ctx->stats.ms_exchange = time_end(ctx);
        ctx->stats.exchange_rank = rank;
        if (s == HF_OK) s = check_async(ctx, "hf_exchange");
        return s;
    }
    const int64_t opad = std::max<int64_t>(64, round_up(rank, 64));
    double* Ct = buf + oCt;
    double* sign = buf + osg;
    time_begin(ctx);
    HF_CU(factor_pad(Lc, 0, n, ctx->d_info, Ct, 0, npad, opad, sign, 1, nullptr, ctx->stream));
    double* dK = on_device ? K : sK;
    int s = exchange_from_ct(ctx, Ct, (int)opad, sign, false, dK, precision);
    if (s == HF_OK && !on_device) cudaMemcpyAsync(K, sK, sizeof(double) * nn, cudaMemcpyDeviceToHost, ctx->stream);
    ctx->stats.ms_exchange = time_end(ctx);
    ctx->stats.exchange_rank = rank;
    if (s == HF_OK) s = check_async(ctx, "hf_exchange");
    return s;
}

int hf_metric(hf_ctx* ctx, double* out) {
    if (!ctx || !out) return HF_ERR_ARG;
    if (!ctx->uploaded) return fail(ctx, HF_ERR_STATE, "upload shells first");
    cudaSetDevice(ctx->device);
    int s;
    if (!ctx->d_metric && (s = build_metric(ctx)) != HF_OK) return s;
    const int N = ctx->naux;
    std::vector<double> m((size_t)N * N);
    HF_CU(cudaStreamSynchronize(ctx->stream));
    HF_CU(cudaMemcpy(m.data(), ctx->d_metric, sizeof(double) * m.size(), cudaMemcpyDeviceToHost));
    for (int a = 0; a < N; ++a)
        for (int b = 0; b < N; ++b)
            out[(size_t)ctx->aux_ref_fn[a] * N + ctx->aux_ref_fn[b]] = m[(size_t)a * N + b];
    return HF_OK;
}

int hf_three_center(hf_ctx* ctx, double* out) {
    if (!ctx || !out) return HF_ERR_ARG;
    if (!ctx->uploaded) return fail(ctx, HF_ERR_STATE, "upload shells first");
    cudaSetDevice(ctx->device);
    const int N = ctx->naux, n = ctx->n, nt = ctx->nt;
    const int64_t ncols = ctx->ntiles * 4096;
    double* T = nullptr;
    PairTask* d_tasks = nullptr;
    const size_t ns = ctx->orb.size(), task_cap = ns * (ns + 1) / 2 + 16;
    if (alloc(ctx, (void**)&T, sizeof(double) * (size_t)ncols * N) ||
        alloc(ctx, (void**)&d_tasks, sizeof(PairTask) * task_cap)) {
        release(ctx, T);
        return HF_ERR_OOM;
    }
    HF_CU(cudaMemsetAsync(T, 0, sizeof(double) * (size_t)ncols * N, ctx->stream));
    int s = three_center_chunk(ctx, 0, nt, T, d_tasks, task_cap);
    std::vector<double> h;
    if (s == HF_OK) {
        h.resize((size_t)ncols * N);
        cudaMemcpy(h.data(), T, sizeof(double) * h.size(), cudaMemcpyDeviceToHost);
    }
    release(ctx, T);
    release(ctx, d_tasks);
    if (s != HF_OK) return s;
    for (int mu = 0; mu < n; ++mu)
        for (int nu = 0; nu < n; ++nu) {
            int a = mu, b = nu;
            if ((a >> 6) > (b >> 6)) std::swap(a, b);
            const int64_t col = tile_index(a >> 6, b >> 6, nt) * 4096 + (a & 63) * 64 + (b & 63);
            for (int q = 0; q < N; ++q)
                out[((size_t)ctx->aux_ref_fn[q] * n + mu) * n + nu] = h[(size_t)col * N + q];
        }
    return HF_OK;
}

int hf_fitted_eri(hf_ctx* ctx, double* out) {
    if (!ctx || !out) return HF_ERR_ARG;
    if (!ctx->built) return fail(ctx, HF_ERR_STATE, "build the fitted tensor first");
    if (!holds_all_rows(ctx)) return fail(ctx, HF_ERR_STATE, "this needs every row of the fitted tensor; the context holds a shard");
    cudaSetDevice(ctx->device);
    const int N = ctx->naux, n = ctx->n, nt = ctx->nt;
    const int64_t ldb = ctx->ntiles * 4096;
    std::vector<double> b((size_t)N * ldb);
    HF_CU(cudaStreamSynchronize(ctx->stream));
    HF_CU(cudaMemcpy(b.data(), ctx->d_B, sizeof(double) * b.size(), cudaMemcpyDeviceToHost));
    std::vector<double> full((size_t)N * n * n);
    for (int q = 0; q < N; ++q)
        for (int mu = 0; mu < n; ++mu)
            for (int nu = 0; nu < n; ++nu) {
                int a = mu, c = nu;
                if ((a >> 6) > (c >> 6)) std::swap(a, c);
                full[((size_t)q * n + mu) * n + nu] = b[(size_t)q * ldb + tile_index(a >> 6, c >> 6, nt) * 4096 + (a & 63) * 64 + (c & 63)];
            }
    const size_t n2 = (size_t)n * n;
    for (size_t i = 0; i < n2; ++i)
        for (size_t j = 0; j < n2; ++j) {
            double s = 0.0;
            for (int q = 0; q < N; ++q) s += full[q * n2 + i] * full[q * n2 + j];
            out[i * n2 + j] = s;
        }
    return HF_OK;
}

int hf_one_electron(hf_ctx* ctx, int kind, const double* charges, const double* positions, int64_t natoms, double* out,
                    int on_device) {
    if (!ctx || !out || kind < 0 || kind > 2) return HF_ERR_ARG;
    if (!ctx->uploaded) return fail(ctx, HF_ERR_STATE, "upload shells first");
    if (kind == 2 && (natoms < 0 || (natoms > 0 && (!charges || !positions))))
        return fail(ctx, HF_ERR_ARG, "attraction needs charges and positions");
    cudaSetDevice(ctx->device);
    const int64_t n = ctx->n;
    const size_t nn = (size_t)n * n;
    double* buf = nullptr;
    const int ns = (int)ctx->orb.size();
    std::vector<int2> tasks[3][3];
    for (int a = 0; a < ns; ++a)
        for (int b = 0; b < ns; ++b) tasks[ctx->orb[a].l][ctx->orb[b].l].push_back(make_int2(a, b));
    const size_t need = sizeof(double) * (nn + 4 * (size_t)std::max<int64_t>(natoms, 1)) + sizeof(int2) * ns * ns + 64;
    if (talloc(ctx, (void**)&buf, need)) return HF_ERR_OOM;
    double* sOut = buf;
    double* sq = sOut + nn;
    double* spos = sq + std::max<int64_t>(natoms, 1);
    int2* dt = (int2*)(spos + 3 * std::max<int64_t>(natoms, 1));
    if (kind == 2 && natoms > 0) {
        cudaMemcpyAsync(sq, charges, sizeof(double) * natoms,
                        on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx->stream);
        cudaMemcpyAsync(spos, positions, sizeof(double) * 3 * natoms,
                        on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx->stream);
    }
    double* dOut = on_device ? out : sOut;
    size_t off = 0;
    cudaError_t e = cudaSuccess;
    for (int la = 0; la <= 2 && e == cudaSuccess; ++la)
        for (int lb = 0; lb <= 2 && e == cudaSuccess; ++lb) {
            auto& v = tasks[la][lb];
            if (v.empty()) continue;
            cudaMemcpyAsync(dt + off, v.data(), sizeof(int2) * v.size(), cudaMemcpyHostToDevice, ctx->stream);
            e = launch_one_electron(kind, la, lb, dt + off, (int)v.size(), ctx->d_orb, ctx->d_exps, ctx->d_coefs, sq,
                                    spos, (int)natoms, ctx->d_btable, dOut, n, ctx->stream);
            ++ctx->stats.kernel_launches;
            off += v.size();
        }
    if (e == cudaSuccess && !on_device)
        e = cudaMemcpyAsync(out, sOut, sizeof(double) * nn, cudaMemcpyDeviceToHost, ctx->stream);
    trelease(ctx, buf);
    const cudaError_t se = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess) e = se;
    if (e != cudaSuccess) return fail(ctx, HF_ERR_CUDA, std::string("one-electron: ") + cudaGetErrorString(e));
    return HF_OK;
}

int hf_four_center(hf_ctx* ctx, double* out, int on_device) {
    if (!ctx || !out) return HF_ERR_ARG;
    if (!ctx->uploaded) return fail(ctx, HF_ERR_STATE, "upload shells first");
    cudaSetDevice(ctx->device);
    const int64_t n = ctx->n;
    if (n > 128) return fail(ctx, HF_ERR_ARG, "the exact four-centre kernel serves atoms and small molecules (n <= 128)");
    const size_t bytes = sizeof(double) * (size_t)n * n * n * n;
    double* dst = out;
    double* tmp = nullptr;
    if (!on_device) {
        if (alloc(ctx, (void**)&tmp, bytes)) return HF_ERR_OOM;
        dst = tmp;
    }
    cudaError_t e = launch_four_center(ctx->d_orb, (int)ctx->orb.size(), ctx->d_exps, ctx->d_coefs, ctx->d_btable, dst,
                                       (int)n, ctx->stream);
    ++ctx->stats.kernel_launches;
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess && !on_device) e = cudaMemcpy(out, tmp, bytes, cudaMemcpyDeviceToHost);
    release(ctx, tmp);
    if (e != cudaSuccess) return fail(ctx, HF_ERR_CUDA, std::string("four-centre: ") + cudaGetErrorString(e));
    return HF_OK;
}

int hf_mp2_energy(hf_ctx* ctx, const double* mo_coefficients, const double* mo_energies, int64_t n_mo, int64_t n_occ,
                  double* correlation, int on_device) {
    if (!ctx || !mo_coefficients || !mo_energies || !correlation || n_mo < 1 || n_occ < 1 || n_occ > n_mo)
        return HF_ERR_ARG;
    if (!ctx->built) return fail(ctx, HF_ERR_STATE, "build the fitted tensor first");
    if (!holds_all_rows(ctx)) return fail(ctx, HF_ERR_STATE, "this needs every row of the fitted tensor; the context holds a shard");
    if (n_mo > ctx->n) return fail(ctx, HF_ERR_ARG, "more orbitals than basis functions");
    cudaSetDevice(ctx->device);
    const JkPlan p = plan_of(ctx);
    const double* dC = mo_coefficients;
    const double* de = mo_energies;
    double* staged = nullptr;
    if (!on_device) {
        const size_t cbytes = sizeof(double) * (size_t)ctx->n * n_mo, ebytes = sizeof(double) * (size_t)n_mo;
        HF_CU(cudaMallocAsync((void**)&staged, cbytes + ebytes, ctx->stream));
        HF_CU(cudaMemcpyAsync(staged, mo_coefficients, cbytes, cudaMemcpyHostToDevice, ctx->stream));
        HF_CU(cudaMemcpyAsync(staged + (size_t)ctx->n * n_mo, mo_energies, ebytes, cudaMemcpyHostToDevice, ctx->stream));
        dC = staged;
        de = staged + (size_t)ctx->n * n_mo;
    }
    cudaError_t e = mp2_energy(p, dC, n_mo, de, n_occ, correlation, ctx->stream);
    if (staged) cudaFreeAsync(staged, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess)
        return fail(ctx, e == cudaErrorMemoryAllocation ? HF_ERR_OOM : HF_ERR_CUDA,
                    std::string("hf_mp2_energy: ") + cudaGetErrorString(e));
    return HF_OK;
}

int hf_mo_fitted_tensor(hf_ctx* ctx, const double* c_bra, int64_t n_bra, const double* c_ket, int64_t n_ket,
                        double* out, int on_device) {
    if (!ctx || !c_bra || !c_ket || !out || n_bra < 1 || n_ket < 1) return HF_ERR_ARG;
    if (!ctx->built) return fail(ctx, HF_ERR_STATE, "build the fitted tensor first");
    if (!holds_all_rows(ctx)) return fail(ctx, HF_ERR_STATE, "this needs every row of the fitted tensor; the context holds a shard");
    cudaSetDevice(ctx->device);
    const JkPlan p = plan_of(ctx);
    const int64_t n = ctx->n, N = ctx->naux;
    const size_t out_doubles = (size_t)N * n_bra * n_ket;
    double *staged = nullptr, *dout = out;
    const double *db = c_bra, *dk = c_ket;
    if (!on_device) {
        const size_t cb = (size_t)n * n_bra, ck = (size_t)n * n_ket;
        if (cudaMallocAsync((void**)&staged, sizeof(double) * (cb + ck + out_doubles), ctx->stream) != cudaSuccess) {
            cudaGetLastError();
            return fail(ctx, HF_ERR_OOM, "no room to stage the orbital-basis tensor");
        }
        cudaError_t ec = cudaMemcpyAsync(staged, c_bra, sizeof(double) * cb, cudaMemcpyHostToDevice, ctx->stream);
        if (ec == cudaSuccess)
            ec = cudaMemcpyAsync(staged + cb, c_ket, sizeof(double) * ck, cudaMemcpyHostToDevice, ctx->stream);
        if (ec != cudaSuccess) {
            cudaFreeAsync(staged, ctx->stream);
            return fail(ctx, HF_ERR_CUDA, std::string("hf_mo_fitted_tensor: ") + cudaGetErrorString(ec));
        }
        db = staged;
        dk = staged + cb;
        dout = staged + cb + ck;
    }
    cudaError_t e = mo_fitted_tensor(p, db, n_bra, dk, n_ket, nullptr, dout, ctx->stream);
    ctx->stats.kernel_launches += 2 + 3 * ((N + 63) / 64);
    if (e == cudaSuccess && !on_device)
        e = cudaMemcpyAsync(out, dout, sizeof(double) * out_doubles, cudaMemcpyDeviceToHost, ctx->stream);
    if (staged) cudaFreeAsync(staged, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess)
        return fail(ctx, e == cudaErrorMemoryAllocation ? HF_ERR_OOM : HF_ERR_CUDA,
                    std::string("hf_mo_fitted_tensor: ") + cudaGetErrorString(e));
    return HF_OK;
}

// The atom of every shell: the one at its centre.
static int shell_atoms(hf_ctx* ctx, const std::vector<DevShell>& shells, const double* positions, int64_t natoms,
                       std::vector<int>& out, const char* what) {
    out.assign(shells.size(), -1);
    for (size_t s = 0; s < shells.size(); ++s) {
        double best = 1e300;
        for (int64_t a = 0; a < natoms; ++a) {
            const double dx = shells[s].x - positions[3 * a], dy = shells[s].y - positions[3 * a + 1],
                         dz = shells[s].z - positions[3 * a + 2];
            const double d2 = dx * dx + dy * dy + dz * dz;
            if (d2 < best) {
                best = d2;
                out[s] = (int)a;
            }
        }
        if (out[s] < 0 || best > 1e-20)
            return fail(ctx, HF_ERR_ARG, std::string(what) + " shell " + std::to_string(s) + " sits on no atom");
    }
    return HF_OK;
}

int hf_nuclear_gradient(hf_ctx* ctx, const double* C, int64_t nocc, const double* W, const double* charges,
                        const double* positions, int64_t natoms, double* terms, int on_device) {
    if (!ctx || !C || !W || !charges || !positions || !terms || nocc < 1 || natoms < 1) return HF_ERR_ARG;
    if (!ctx->built) return fail(ctx, HF_ERR_STATE, "build the fitted tensor first");
    if (!holds_all_rows(ctx)) return fail(ctx, HF_ERR_STATE, "this needs every row of the fitted tensor; the context holds a shard");
    if (nocc > ctx->n) return fail(ctx, HF_ERR_ARG, "more occupied orbitals than basis functions");
    if ((int64_t)nocc * nocc > INT32_MAX / 2) return fail(ctx, HF_ERR_ARG, "too many occupied orbitals");
    cudaSetDevice(ctx->device);
    std::vector<int> orb_atom, aux_atom;
    int st;
    if ((st = shell_atoms(ctx, ctx->orb, positions, natoms, orb_atom, "orbital")) != HF_OK) return st;
    if ((st = shell_atoms(ctx, ctx->aux, positions, natoms, aux_atom, "auxiliary")) != HF_OK) return st;
    upload_gradient_tables(ctx->stream);
    const JkPlan p = plan_of(ctx);
    const int64_t n = ctx->n, N = ctx->naux, o = nocc, oo = nocc * nocc;
    const size_t nn = (size_t)n * n, NN = (size_t)N * N;
    {
        // the split-BF16 copy of B is not needed here: its room goes to the
        // gradient when the intermediates (and 2 GB of exchange weights) do not fit
        size_t freeb = 0, totalb = 0;
        cudaMemGetInfo(&freeb, &totalb);
        const size_t need = sizeof(double) * (2 * (size_t)oo * N + 5 * NN + 4 * nn) + ((size_t)2 << 30);
        if (ctx->d_bf16_b && freeb < need) {
            big_release(ctx, ctx->d_bf16_b, ctx->bf16_alloc_bytes);
            free_retained(ctx->device);
        }
    }
    const int nso = (int)ctx->orb.size(), nsa = (int)ctx->aux.size();
    struct Temps {
        hf_ctx* c;
        std::vector<void*> ptrs;
        ~Temps() {
            for (void* q : ptrs) cudaFreeAsync(q, c->stream);
        }
        double* take(size_t doubles) {
            void* q = nullptr;
            if (cudaMallocAsync(&q, sizeof(double) * std::max<size_t>(doubles, 1), c->stream) != cudaSuccess) {
                cudaGetLastError();
                return nullptr;
            }
            ptrs.push_back(q);
            return static_cast<double*>(q);
        }
    } tmp{ctx, {}};
    const double* dC = C;
    const double* dW = W;
    if (!on_device) {
        double* sC = tmp.take((size_t)n * o);
        double* sW = tmp.take(nn);
        if (!sC || !sW) return fail(ctx, HF_ERR_OOM, "no room for the gradient's inputs");
        HF_CU(cudaMemcpyAsync(sC, C, sizeof(double) * n * o, cudaMemcpyHostToDevice, ctx->stream));
        HF_CU(cudaMemcpyAsync(sW, W, sizeof(double) * nn, cudaMemcpyHostToDevice, ctx->stream));
        dC = sC;
        dW = sW;
    }
    double* Dt = tmp.take(nn);
    double* dfit = tmp.take(N);
    double* cfit = tmp.take(N);
    double* work = tmp.take((size_t)coulomb_work_doubles(p));
    double* L = tmp.take(NN);
    double* Linv = tmp.take(NN);
    double* LinvT = tmp.take(NN);
    double* wk = tmp.take((size_t)N * 64);
    double* Gt = tmp.take((size_t)oo * N);
    double* G = tmp.take((size_t)oo * N);
    double* WJ = tmp.take(NN);
    double* WK = tmp.take(NN);
    double* acc = tmp.take((size_t)(2 * nso + nsa) * 6 + 3 * natoms);
    double* dq = tmp.take(natoms);
    double* dpos = tmp.take(3 * natoms);
    if (!Dt || !dfit || !cfit || !work || !L || !Linv || !LinvT || !wk || !Gt || !G || !WJ || !WK || !acc || !dq ||
        !dpos)
        return fail(ctx, HF_ERR_OOM, "no room for the gradient's intermediates");
    double* gorb = acc;
    double* gorb1 = gorb + (size_t)nso * 6;
    double* gaux = gorb1 + (size_t)nso * 6;
    double* gatom = gaux + (size_t)nsa * 6;
    HF_CU(cudaMemsetAsync(acc, 0, sizeof(double) * ((size_t)(2 * nso + nsa) * 6 + 3 * natoms), ctx->stream));
    HF_CU(cudaMemcpyAsync(dq, charges, sizeof(double) * natoms, cudaMemcpyHostToDevice, ctx->stream));
    HF_CU(cudaMemcpyAsync(dpos, positions, sizeof(double) * 3 * natoms, cudaMemcpyHostToDevice, ctx->stream));
    auto gemm = [&](int M, int Ncol, int K, const double* A, int64_t lda, const double* B, int64_t ldb, double* Cm,
                    int64_t ldc, double alpha, int kmode, int epi) {
        GemmArgs g{};
        g.M = M;
        g.N = Ncol;
        g.K = K;
        g.A = A;
        g.lda = lda;
        g.B = B;
        g.ldb = ldb;
        g.C = Cm;
        g.ldc = ldc;
        g.alpha = alpha;
        g.beta = 0.0;
        g.kmode = kmode;
        g.epi = epi;
        ++ctx->stats.kernel_launches;
        return dgemm_nt(g, 1, ctx->stream);
    };
    // total density D = 2 C C^T and the fitted charges d = L^-1 (P|uv) D
    ctx->stats.ms_gradient_weights = 0.0;
    time_begin(ctx);
    HF_CU(gemm((int)n, (int)n, (int)o, dC, o, dC, o, Dt, n, 2.0, 0, 0));
    HF_CU(fitted_charges(p, Dt, dfit, work, ctx->stream));
    // the metric's factor M = L L^T and its inverse
    HF_CU(cudaMemcpyAsync(L, ctx->d_metric, NN * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    HF_CU(cudaMemsetAsync(ctx->d_info, 0, sizeof(int), ctx->stream));
    const double big = 1e300;
    HF_CU(cudaMemcpyAsync(ctx->d_scalar, &big, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    HF_CU(cholesky_lower(L, N, N, ctx->d_info, ctx->d_scalar, ctx->stream));
    int info = 0;
    HF_CU(cudaMemcpyAsync(&info, ctx->d_info, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    HF_CU(cudaStreamSynchronize(ctx->stream));
    if (info != 0) return fail(ctx, HF_ERR_NUMERIC, "the Coulomb metric is not positive definite");
    HF_CU(triangular_inverse(L, N, N, Linv, LinvT, wk, ctx->stream));
    // c = M^-1 q = L^-T d
    HF_CU(gemm(1, (int)N, (int)N, dfit, N, LinvT, N, cfit, N, 1.0, 1, 0));
    // Gamma_P = C^T (sum_Q M^-1_PQ (Q|uv)) C = L^-T applied to C^T B_Q C
    HF_CU(occupied_pair_tensor_t(p, dC, o, o, Gt, ctx->stream));
    HF_CU(gemm((int)oo, (int)N, (int)N, Gt, N, LinvT, N, G, oo, 1.0, 1, 1));
    // metric weights: W^J = -c c^T / 2, W^K = Gamma Gamma^T (gradient.py:127-145)
    HF_CU(gemm((int)N, (int)N, 1, cfit, 1, cfit, 1, WJ, N, -0.5, 0, 0));
    HF_CU(gemm((int)N, (int)N, (int)oo, G, oo, G, oo, WK, N, 1.0, 0, 3));  // upper tiles only
    ctx->stats.ms_gradient_weights += time_end(ctx);
    time_begin(ctx);
    HF_CU(launch_metric_grad(ctx->d_aux, ctx->d_exps, ctx->d_coefs, ctx->d_aux_by_l, ctx->aux_count, ctx->d_btable,
                             WJ, WK, N, gaux, ctx->stream));
    ctx->stats.kernel_launches += 25;
    ctx->stats.ms_gradient_metric = time_end(ctx);
    time_begin(ctx);
    // three-centre derivatives over blocks of auxiliary functions, with the
    // exchange weight GK_P = -2 C Gamma_P C^T of the block formed by two GEMMs
    std::vector<PairTask> tasks[3][3];
    int max_npp[3][3];
    chunk_tasks(ctx, 0, ctx->nt, tasks, max_npp);
    size_t ntask = 0;
    for (int la = 0; la <= 2; ++la)
        for (int lb = la; lb <= 2; ++lb) {
            ntask += tasks[la][lb].size();
            if (!tasks[la][lb].empty() && three_center_grad_smem(la, lb, max_npp[la][lb]) > 200 * 1024)
                return fail(ctx, HF_ERR_ARG, "a shell pair has too many primitive pairs for the gradient kernel");
        }
    PairTask* d_tasks = reinterpret_cast<PairTask*>(tmp.take((ntask * sizeof(PairTask) + 7) / 8 + 1));
    // every pair's Hermite data, built once for all auxiliary classes and blocks
    std::vector<int64_t> pair_off(ntask + 1, 0);
    {
        size_t t = 0;
        for (int la = 0; la <= 2; ++la)
            for (int lb = la; lb <= 2; ++lb) {
                const int64_t stride = (int64_t)(three_center_grad_smem(la, lb, 1) / sizeof(double));
                for (const PairTask& pt : tasks[la][lb]) {
                    pair_off[t + 1] = pair_off[t] + (int64_t)ctx->orb[pt.first].nprim * ctx->orb[pt.second].nprim * stride;
                    ++t;
                }
            }
    }
    int64_t* d_pair_off = reinterpret_cast<int64_t*>(tmp.take(ntask + 1));
    int* d_npps = reinterpret_cast<int*>(tmp.take(ntask / 2 + 1));
    double* pair_data = tmp.take((size_t)pair_off[ntask]);
    if (!d_tasks || !d_pair_off || !d_npps || !pair_data)
        return fail(ctx, HF_ERR_OOM, "no room for the gradient's pair list and pair data");
    HF_CU(cudaMemcpyAsync(d_pair_off, pair_off.data(), sizeof(int64_t) * (ntask + 1), cudaMemcpyHostToDevice,
                          ctx->stream));
    {
        size_t off = 0;
        for (int la = 0; la <= 2; ++la)
            for (int lb = la; lb <= 2; ++lb) {
                auto& v = tasks[la][lb];
                if (v.empty()) continue;
                HF_CU(cudaMemcpyAsync(d_tasks + off, v.data(), sizeof(PairTask) * v.size(), cudaMemcpyHostToDevice,
                                      ctx->stream));
                HF_CU(launch_grad_pair_data(la, lb, d_tasks + off, (int)v.size(), max_npp[la][lb], ctx->d_orb,
                                            ctx->d_exps, ctx->d_coefs, Dt, n,
                                            GradPairData{d_pair_off + off, pair_data, d_npps + off}, ctx->stream));
                ++ctx->stats.kernel_launches;
                off += v.size();
            }
    }
    size_t freeb = 0, totalb = 0;
    cudaMemGetInfo(&freeb, &totalb);
    const size_t per_p = sizeof(double) * (nn + (size_t)n * o);
    const size_t budget = std::min<size_t>((size_t)8 << 30, freeb / 3);
    const int64_t pb_max = std::max<int64_t>(16, (int64_t)(budget / per_p));
    double* Zt = tmp.take((size_t)n * o * (pb_max + 8));
    double* GK = tmp.take(nn * (pb_max + 8));
    if (!Zt || !GK) return fail(ctx, HF_ERR_OOM, "no room for the exchange weights of a block");
    int class_start[kMaxAuxL + 1];
    for (int l = 0, c = 0; l <= kMaxAuxL; ++l) {
        class_start[l] = c;
        c += ctx->aux_count[l];
    }
    auto nfun = [&](int s) { return ctx->aux[s].ncontr * nsph(ctx->aux[s].l); };
    for (int s0 = 0; s0 < nsa;) {
        const int P0 = ctx->aux[s0].fn;
        int s1 = s0 + 1;
        while (s1 < nsa && ctx->aux[s1].fn + nfun(s1) - P0 <= pb_max) ++s1;
        const int64_t Pb = ctx->aux[s1 - 1].fn + nfun(s1 - 1) - P0;
        HF_CU(gemm((int)n, (int)(Pb * o), (int)o, dC, o, G + (size_t)P0 * oo, o, Zt, Pb * o, 1.0, 0, 0));
        HF_CU(gemm((int)n, (int)(n * Pb), (int)o, dC, o, Zt, o, GK, n * Pb, -2.0, 0, 0));
        const int* alist[kMaxAuxL + 1];
        int count[kMaxAuxL + 1];
        for (int l = 0; l <= kMaxAuxL; ++l) {
            const int lo = std::max(s0, class_start[l]), hi = std::min(s1, class_start[l] + ctx->aux_count[l]);
            alist[l] = ctx->d_aux_by_l[l] + std::max(0, lo - class_start[l]);
            count[l] = std::max(0, hi - lo);
        }
        const GradWeights gw{Dt, cfit, GK, n, P0, Pb};
        size_t off = 0;
        for (int la = 0; la <= 2; ++la)
            for (int lb = la; lb <= 2; ++lb) {
                const auto& v = tasks[la][lb];
                if (v.empty()) continue;
                HF_CU(launch_three_center_grad(la, lb, d_tasks + off, (int)v.size(), max_npp[la][lb], ctx->d_orb,
                                               ctx->d_aux, ctx->d_exps, ctx->d_coefs, alist, count, ctx->d_btable, gw,
                                               GradPairData{d_pair_off + off, pair_data, d_npps + off}, gorb, gaux,
                                               ctx->stream));
                ctx->stats.kernel_launches += 5;
                off += v.size();
            }
        s0 = s1;
    }
    ctx->stats.ms_gradient_three_center = time_end(ctx);
    // one-electron terms over all ordered shell pairs
    time_begin(ctx);
    std::vector<int2> pairs1[3][3];
    for (int a = 0; a < nso; ++a)
        for (int b = 0; b < nso; ++b) pairs1[ctx->orb[a].l][ctx->orb[b].l].push_back(make_int2(a, b));
    int2* d_pairs1 = reinterpret_cast<int2*>(tmp.take(((size_t)nso * nso * sizeof(int2) + 7) / 8 + 1));
    if (!d_pairs1) return fail(ctx, HF_ERR_OOM, "no room for the one-electron pair list");
    {
        size_t off = 0;
        for (int la = 0; la <= 2; ++la)
            for (int lb = 0; lb <= 2; ++lb) {
                auto& v = pairs1[la][lb];
                if (v.empty()) continue;
                HF_CU(cudaMemcpyAsync(d_pairs1 + off, v.data(), sizeof(int2) * v.size(), cudaMemcpyHostToDevice,
                                      ctx->stream));
                HF_CU(launch_one_electron_grad(la, lb, d_pairs1 + off, (int)v.size(), ctx->d_orb, ctx->d_exps,
                                               ctx->d_coefs, dq, dpos, (int)natoms, ctx->d_btable, Dt, dW, n, gorb1,
                                               gatom, ctx->stream));
                ctx->stats.kernel_launches += 2;
                off += v.size();
            }
    }
    ctx->stats.ms_gradient_one_electron = time_end(ctx);
    std::vector<double> h((size_t)(2 * nso + nsa) * 6 + 3 * natoms);
    HF_CU(cudaMemcpyAsync(h.data(), acc, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, ctx->stream));
    HF_CU(cudaStreamSynchronize(ctx->stream));
    if ((st = check_async(ctx, "hf_nuclear_gradient")) != HF_OK) return st;
    // per-shell sums to atoms in a fixed order; the nuclear repulsion on the host
    std::vector<double> out((size_t)5 * natoms * 3, 0.0);
    auto at = [&](int term, int atom, int d) -> double& { return out[((size_t)term * natoms + atom) * 3 + d]; };
    for (int64_t k = 0; k < natoms; ++k)
        for (int64_t l = 0; l < natoms; ++l) {
            if (k == l) continue;
            double r[3], r2 = 0.0;
            for (int d = 0; d < 3; ++d) {
                r[d] = positions[3 * k + d] - positions[3 * l + d];
                r2 += r[d] * r[d];
            }
            const double w = charges[k] * charges[l] / (r2 * std::sqrt(r2));
            for (int d = 0; d < 3; ++d) at(0, (int)k, d) -= w * r[d];
        }
    const double* hg = h.data();
    const double* hg1 = hg + (size_t)nso * 6;
    const double* hga = hg1 + (size_t)nso * 6;
    const double* hat = hga + (size_t)nsa * 6;
    for (int s = 0; s < nso; ++s)
        for (int d = 0; d < 3; ++d) {
            at(1, orb_atom[s], d) += hg1[s * 6 + d];
            at(2, orb_atom[s], d) += hg1[s * 6 + 3 + d];
            at(3, orb_atom[s], d) += hg[s * 6 + d];
            at(4, orb_atom[s], d) += hg[s * 6 + 3 + d];
        }
    for (int s = 0; s < nsa; ++s)
        for (int d = 0; d < 3; ++d) {
            at(3, aux_atom[s], d) += hga[s * 6 + d];
            at(4, aux_atom[s], d) += hga[s * 6 + 3 + d];
        }
    for (int64_t c = 0; c < natoms; ++c)
        for (int d = 0; d < 3; ++d) at(1, (int)c, d) += hat[c * 3 + d];
    if (on_device) {
        HF_CU(cudaMemcpyAsync(terms, out.data(), sizeof(double) * out.size(), cudaMemcpyHostToDevice, ctx->stream));
        HF_CU(cudaStreamSynchronize(ctx->stream));
    } else {
        std::memcpy(terms, out.data(), sizeof(double) * out.size());
    }
    return HF_OK;
}

int hf_get_stats(const hf_ctx* ctx, hf_stats* out) {
    if (!ctx || !out) return HF_ERR_ARG;
    *out = ctx->stats;
    return HF_OK;
}

int hf_boys(hf_ctx* ctx, const double* t, int64_t count, int n_max, double* out) {
    if (!ctx || count < 0 || (count > 0 && (!t || !out))) return HF_ERR_ARG;
    if (n_max < 0 || n_max > kBoysMaxOrder)
        return fail(ctx, HF_ERR_ARG, "the device Boys function covers orders 0.." + std::to_string(kBoysMaxOrder) +
                                         " (got " + std::to_string(n_max) + ")");
    for (int64_t i = 0; i < count; ++i)
        if (!(t[i] >= 0.0) || !std::isfinite(t[i])) return fail(ctx, HF_ERR_ARG, "the Boys function argument is non-negative");
    if (count == 0) return HF_OK;
    cudaSetDevice(ctx->device);
    const size_t in_bytes = sizeof(double) * (size_t)count, out_bytes = in_bytes * (size_t)(n_max + 1);
    double* dt = nullptr;
    if (talloc(ctx, (void**)&dt, in_bytes + out_bytes)) return HF_ERR_OOM;
    double* dout = dt + count;
    cudaError_t e = cudaMemcpyAsync(dt, t, in_bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = launch_boys_values(dt, count, n_max, ctx->d_btable, dout, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, out_bytes, cudaMemcpyDeviceToHost, ctx->stream);
    trelease(ctx, dt);
    ctx->stats.kernel_launches += 1;
    if (e != cudaSuccess) return fail(ctx, HF_ERR_CUDA, std::string("hf_boys: ") + cudaGetErrorString(e));
    return check_async(ctx, "hf_boys");
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Coulomb build that allocates nothing.
//
// Some callers cannot call cudaMalloc: an application whose device memory is
// already fully reserved by its own pool allocator (a cudaMalloc would fail or
// fragment that pool), or a latency-critical loop in which a cudaMalloc /
// cudaFree pair, which can synchronise the device, is not allowed. For them
// hf_coulomb_static runs the same J build as hf_coulomb but takes its scratch
// (the weighted packed density, the fitting charges and the packed J) from the
// file-scope array below instead of from an allocation. The caller still passes
// the density and J as device pointers.
//
// Limits: n_ao <= kStaticMaxAo (1536, 24 tiles of 64) and n_aux <= kStaticMaxAux
// (8192). The array is 2 * 300 * 4096 + 8192 doubles, about 19.7 MB, and every
// GPU that loads this library holds it until the process exits. All calls on a
// device share it: calls whose work overlaps on the GPU (different streams or
// contexts at the same time) race on it and must be serialised by the caller.
// The first call on a device resolves the array's device address
// (cudaGetSymbolAddress, with that device current); make that first call before
// any stream capture. The address is kept for the life of the process: after a
// reset of the device (cudaDeviceReset) it is stale, so no call may follow one.
// The call returns once J is complete (it waits for the context's stream).
namespace {
constexpr int64_t kStaticMaxAo = 1536;
constexpr int64_t kStaticMaxAux = 8192;
constexpr int64_t kStaticMaxTiles = (kStaticMaxAo / 64) * (kStaticMaxAo / 64 + 1) / 2;
constexpr int64_t kStaticScratchDoubles = 2 * kStaticMaxTiles * 4096 + kStaticMaxAux;
static __device__ __align__(256) double g_coulomb_scratch[kStaticScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
double* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_coulomb_scratch on `device` (current), resolved once.
int static_scratch(hf_ctx* ctx, double** out) {
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (ctx->device < 0 || ctx->device >= kMaxDevices) return fail(ctx, HF_ERR_ARG, "device index out of range");
    if (!g_scratch_ptr[ctx->device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_coulomb_scratch);
        if (e != cudaSuccess || p == nullptr)
            return fail(ctx, HF_ERR_CUDA, std::string("cudaGetSymbolAddress(g_coulomb_scratch): ") +
                                              cudaGetErrorString(e));
        g_scratch_ptr[ctx->device] = static_cast<double*>(p);
    }
    *out = g_scratch_ptr[ctx->device];
    return HF_OK;
}
}  // namespace

extern "C" int hf_coulomb_static(hf_ctx* ctx, const double* density, double* coulomb) {
    if (!ctx || !density || !coulomb) return HF_ERR_ARG;
    if (ctx->uploaded && (ctx->n > kStaticMaxAo || ctx->naux > kStaticMaxAux))
        return fail(ctx, HF_ERR_ARG, "hf_coulomb_static supports n_ao <= " + std::to_string(kStaticMaxAo) +
                                         " and n_aux <= " + std::to_string(kStaticMaxAux) + " (got " +
                                         std::to_string(ctx->n) + " and " + std::to_string(ctx->naux) +
                                         "); use hf_coulomb");
    if (!ctx->built) return fail(ctx, HF_ERR_STATE, "build the fitted tensor first");
    cudaSetDevice(ctx->device);
    double* scratch = nullptr;
    int s = static_scratch(ctx, &scratch);
    if (s != HF_OK) return s;
    const JkPlan p = plan_of(ctx);
    if (coulomb_work_doubles(p) > kStaticScratchDoubles) return fail(ctx, HF_ERR_ARG, "scratch size exceeded");
    cudaError_t e = coulomb_build(p, density, coulomb, scratch, ctx->stream);
    if (e != cudaSuccess) return fail(ctx, HF_ERR_CUDA, std::string("hf_coulomb_static: ") + cudaGetErrorString(e));
    ctx->stats.kernel_launches += 4;
    return check_async(ctx, "hf_coulomb_static");
}
