// FP64 DMMA GEMM (see dgemm.cuh for the contract).
//
// Warps of 32 x 32 output (2 x 4 mma.sync.m16n8k8 FP64 tiles), a cp.async
// pipeline from global memory into shared tiles stored row-major with a row
// pitch of BK + 4 doubles (conflict-free fragment loads): 3 stages of BK = 16,
// or for the 64 x 64 tile of the large products 2 stages of BK = 32 (half the
// barriers per k; 34.0 against 33.5 TF/s on a 7232 x 16384 x 7232 product). Operands are
// K-contiguous rows (A[m][k], B[n][k]); copies are 8 bytes so any row stride and
// offset is legal, and out-of-range elements are zero-filled.
#include <mutex>

#include "dgemm.cuh"

namespace hf {

namespace {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// 8-byte asynchronous copy; an invalid element copies nothing and zero-fills
// (the source then points at the matrix base, which is never read).
__device__ __forceinline__ void cp_async8(double* dst, const double* src, const double* base, bool valid) {
    const int bytes = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(smem_addr(dst)), "l"(valid ? src : base),
                 "r"(bytes));
}

// 16-byte asynchronous copy of (up to) two doubles: `bytes` of 16, 8 or 0 are
// read and the rest of the 16 zero-filled. Both addresses 16-byte aligned.
__device__ __forceinline__ void cp_async16(double* dst, const double* src, const double* base, int bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_addr(dst)), "l"(bytes ? src : base),
                 "r"(bytes));
}

__device__ __forceinline__ void mma16x8x8(double (&c)[4], const double (&a)[4], const double (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

template <int BM, int BN>
__host__ __device__ constexpr int threads_of() {
    return (BM / 32) * (BN / 32) * 32;
}

template <int BM, int BN, int BK, int STAGES>
__host__ __device__ constexpr int smem_of() {
    return STAGES * (BM + BN) * (BK + 4) * (int)sizeof(double);
}

// CTAs per SM the register budget is sized for: up to 16 warps, as many as the
// shared memory of the pipeline lets reside.
template <int BM, int BN, int BK, int STAGES>
__host__ __device__ constexpr int min_ctas_of() {
    const int by_warps = 512 / threads_of<BM, BN>();
    const int by_smem = (227 * 1024) / smem_of<BM, BN, BK, STAGES>();
    const int m = by_warps < by_smem ? by_warps : by_smem;
    return m < 1 ? 1 : m;
}

// VEC: operands 16-byte aligned with even row strides, copied two doubles at a time.
template <int BM, int BN, int BK, int STAGES, bool VEC>
__global__ void __launch_bounds__(threads_of<BM, BN>(), (min_ctas_of<BM, BN, BK, STAGES>()))
    k_dgemm_nt(GemmArgs g) {
    constexpr int THREADS = threads_of<BM, BN>();
    constexpr int LD = BK + 4;
    constexpr int WARPS_N = BN / 32;
    const int zz = blockIdx.z;
    int z = zz, sp = 0;
    if (g.splits > 1) {
        z = zz / g.splits;
        sp = zz - z * g.splits;
    }
    if (g.active && g.active[z] == 0) return;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    if (g.epi == 2 && n0 > m0 + BM - 1) return;
    if (g.epi == 3 && m0 > n0 + BN - 1) return;
    const double alpha = g.alpha_v ? g.alpha_v[z] : g.alpha;
    const double beta = g.beta_v ? g.beta_v[z] : g.beta;
    const double* A = g.A + (int64_t)z * g.strideA;
    const double* B = g.B + (int64_t)z * g.strideB;
    double* C = g.C + (int64_t)zz * g.strideC;
    int kb = 0, ke = g.K;
    if (g.kmode == 1) kb = n0;
    if (g.kmode == 2) ke = min(g.K, g.koff + m0 + BM);
    kb = (kb / BK) * BK;
    if (g.splits > 1) {
        const int span = ((ke - kb + g.splits - 1) / g.splits + BK - 1) / BK * BK;
        kb = kb + sp * span;
        ke = min(ke, kb + span);
    }
    const int nk = ke > kb ? (ke - kb + BK - 1) / BK : 0;

    extern __shared__ double smem[];
    double* As = smem;                     // [STAGES][BM][LD]
    double* Bs = smem + STAGES * BM * LD;  // [STAGES][BN][LD]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int gq = lane >> 2, tq = lane & 3;
    const int wm = (warp / WARPS_N) * 32, wn = (warp % WARPS_N) * 32;

    auto load = [&](int stage, int k0) {
        double* as = As + stage * BM * LD;
        double* bs = Bs + stage * BN * LD;
        if constexpr (VEC) {
            auto piece = [&](int gk) { return gk < ke ? (gk + 1 < ke ? 16 : 8) : 0; };
#pragma unroll
            for (int i = 0; i < (BM * BK) / (2 * THREADS); ++i) {
                const int e = tid + i * THREADS;
                const int r = e / (BK / 2), k = (e % (BK / 2)) * 2;
                const int gm = m0 + r, gk = k0 + k;
                cp_async16(as + r * LD + k, A + (int64_t)gm * g.lda + gk, A, gm < g.M ? piece(gk) : 0);
            }
#pragma unroll
            for (int i = 0; i < (BN * BK) / (2 * THREADS); ++i) {
                const int e = tid + i * THREADS;
                const int r = e / (BK / 2), k = (e % (BK / 2)) * 2;
                const int gn = n0 + r, gk = k0 + k;
                cp_async16(bs + r * LD + k, B + (int64_t)gn * g.ldb + gk, B, gn < g.N ? piece(gk) : 0);
            }
            return;
        }
#pragma unroll
        for (int i = 0; i < (BM * BK) / THREADS; ++i) {
            const int e = tid + i * THREADS;
            const int r = e / BK, k = e % BK;
            const int gm = m0 + r, gk = k0 + k;
            cp_async8(as + r * LD + k, A + (int64_t)gm * g.lda + gk, A, gm < g.M && gk < ke);
        }
#pragma unroll
        for (int i = 0; i < (BN * BK) / THREADS; ++i) {
            const int e = tid + i * THREADS;
            const int r = e / BK, k = e % BK;
            const int gn = n0 + r, gk = k0 + k;
            cp_async8(bs + r * LD + k, B + (int64_t)gn * g.ldb + gk, B, gn < g.N && gk < ke);
        }
    };

    double acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[i][j][v] = 0.0;

#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
        if (s < nk) load(s, kb + s * BK);
        asm volatile("cp.async.commit_group;\n" ::);
    }
    for (int it = 0; it < nk; ++it) {
        asm volatile("cp.async.wait_group %0;\n" ::"n"(STAGES - 2));
        __syncthreads();
        const int nxt = it + STAGES - 1;
        if (nxt < nk) load(nxt % STAGES, kb + nxt * BK);
        asm volatile("cp.async.commit_group;\n" ::);
        const double* as = As + (it % STAGES) * BM * LD;
        const double* bs = Bs + (it % STAGES) * BN * LD;
#pragma unroll
        for (int kk = 0; kk < BK; kk += 8) {
            double af[2][4], bf[4][2];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const double* r0 = as + (wm + i * 16 + gq) * LD + kk + tq;
                af[i][0] = r0[0];
                af[i][1] = r0[8 * LD];
                af[i][2] = r0[4];
                af[i][3] = r0[8 * LD + 4];
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const double* c0 = bs + (wn + j * 8 + gq) * LD + kk + tq;
                bf[j][0] = c0[0];
                bf[j][1] = c0[4];
            }
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) mma16x8x8(acc[i][j], af[i], bf[j]);
        }
    }
    asm volatile("cp.async.wait_group 0;\n" ::);

#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const int m = m0 + wm + i * 16 + gq + (v >> 1) * 8;
                const int n = n0 + wn + j * 8 + 2 * tq + (v & 1);
                if (m >= g.M || n >= g.N) continue;
                double* dst = (g.epi == 1) ? &C[(int64_t)n * g.ldc + m] : &C[(int64_t)m * g.ldc + n];
                const double val = alpha * acc[i][j][v];
                *dst = (beta == 0.0) ? val : val + beta * *dst;
            }
}

template <int BM, int BN, int BK = 16, int STAGES = 3>
cudaError_t configure_one() {
    cudaError_t e = cudaFuncSetAttribute(k_dgemm_nt<BM, BN, BK, STAGES, false>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem_of<BM, BN, BK, STAGES>());
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_dgemm_nt<BM, BN, BK, STAGES, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                smem_of<BM, BN, BK, STAGES>());
}

bool aligned16(const GemmArgs& g) {
    auto ok = [](const void* p, int64_t ld, int64_t stride) {
        return (reinterpret_cast<uintptr_t>(p) & 15) == 0 && (ld & 1) == 0 && (stride & 1) == 0;
    };
    return ok(g.A, g.lda, g.strideA) && ok(g.B, g.ldb, g.strideB);
}

template <int BM, int BN, int BK = 16, int STAGES = 3>
cudaError_t launch(const GemmArgs& g, int batch, cudaStream_t stream) {
    dim3 grid((g.N + BN - 1) / BN, (g.M + BM - 1) / BM, batch * (g.splits > 1 ? g.splits : 1));
    constexpr int smem = smem_of<BM, BN, BK, STAGES>();
    if (aligned16(g))
        k_dgemm_nt<BM, BN, BK, STAGES, true><<<grid, threads_of<BM, BN>(), smem, stream>>>(g);
    else
        k_dgemm_nt<BM, BN, BK, STAGES, false><<<grid, threads_of<BM, BN>(), smem, stream>>>(g);
    return cudaGetLastError();
}

constexpr int kMaxDevices = 64;
std::mutex g_config_mutex;
bool g_configured[kMaxDevices] = {};
}  // namespace

cudaError_t dgemm_configure() {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_config_mutex);
    if (g_configured[dev]) return cudaSuccess;
    if ((e = configure_one<128, 64>()) != cudaSuccess) return e;
    if ((e = configure_one<64, 64>()) != cudaSuccess) return e;
    if ((e = configure_one<64, 32>()) != cudaSuccess) return e;
    if ((e = configure_one<32, 32>()) != cudaSuccess) return e;
    if ((e = configure_one<128, 128>()) != cudaSuccess) return e;
    if ((e = configure_one<64, 64, 32, 2>()) != cudaSuccess) return e;
    g_configured[dev] = true;
    return cudaSuccess;
}

cudaError_t dgemm_nt(const GemmArgs& g, int batch, cudaStream_t stream) {
    if (g.M <= 0 || g.N <= 0 || batch <= 0) return cudaSuccess;
    if ((int64_t)batch * (g.splits > 1 ? g.splits : 1) > 65535) return cudaErrorInvalidValue;
    cudaError_t e = dgemm_configure();
    if (e != cudaSuccess) return e;
    switch (g.tile) {
        case 0: return launch<128, 64>(g, batch, stream);
        case 1: return launch<64, 64>(g, batch, stream);
        case 2: return launch<64, 32>(g, batch, stream);
        case 3: return launch<32, 32>(g, batch, stream);
        case 4: return launch<128, 128>(g, batch, stream);
        case 5: return launch<64, 64, 32, 2>(g, batch, stream);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace hf
