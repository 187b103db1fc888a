// FP64 DMMA GEMM (see dgemm.cuh for the contract).
#include "dgemm.cuh"

namespace hf {

namespace {
constexpr int BM = 64, BN = 64, BK = 16, LDS = 72;  // LDS: padded row of the k-major tile

__global__ void __launch_bounds__(128) k_dgemm_nt(GemmArgs g) {
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    if (g.epi == 2 && n0 > m0 + BM - 1) return;
    if (g.epi == 3 && m0 > n0 + BN - 1) return;
    const double* A = g.A + (int64_t)blockIdx.z * g.strideA;
    const double* B = g.B + (int64_t)blockIdx.z * g.strideB;
    double* C = g.C + (int64_t)blockIdx.z * g.strideC;
    int kb = 0, ke = g.K;
    if (g.kmode == 1) kb = n0;
    if (g.kmode == 2) ke = min(g.K, m0 + BM);
    kb = (kb / BK) * BK;

    __shared__ double As[2][BK][LDS];
    __shared__ double Bs[2][BK][LDS];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g8 = lane >> 2, t4 = lane & 3;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;

    // Loader mapping: 64 rows x 16 k per operand = 1024 values, 8 per thread:
    // thread -> row r = tid >> 1, k half h = (tid & 1) * 8.
    const int lr = tid >> 1, lk = (tid & 1) * 8;
    double ra[8], rb[8];
    auto load = [&](int k0) {
        const int am = m0 + lr, bn = n0 + lr;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int k = k0 + lk + j;
            ra[j] = (am < g.M && k < ke) ? A[(int64_t)am * g.lda + k] : 0.0;
            rb[j] = (bn < g.N && k < ke) ? B[(int64_t)bn * g.ldb + k] : 0.0;
        }
    };
    auto store = [&](int buf) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            As[buf][lk + j][lr] = ra[j];
            Bs[buf][lk + j][lr] = rb[j];
        }
    };

    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    int buf = 0;
    if (kb < ke) {
        load(kb);
        store(0);
    }
    __syncthreads();
    for (int k0 = kb; k0 < ke; k0 += BK) {
        const bool more = k0 + BK < ke;
        if (more) load(k0 + BK);
#pragma unroll
        for (int kk = 0; kk < BK; kk += 4) {
            double af[4], bf[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) af[i] = As[buf][kk + t4][wm + i * 8 + g8];
#pragma unroll
            for (int j = 0; j < 4; ++j) bf[j] = Bs[buf][kk + t4][wn + j * 8 + g8];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
        }
        if (more) store(buf ^ 1);
        __syncthreads();
        buf ^= 1;
    }

#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int m = m0 + wm + i * 8 + g8;
                const int n = n0 + wn + j * 8 + 2 * t4 + h;
                if (m >= g.M || n >= g.N) continue;
                double* dst = (g.epi == 1) ? &C[(int64_t)n * g.ldc + m] : &C[(int64_t)m * g.ldc + n];
                const double v = g.alpha * acc[i][j][h];
                *dst = (g.beta == 0.0) ? v : v + g.beta * *dst;
            }
}
}  // namespace

cudaError_t dgemm_nt(const GemmArgs& g, int batch, cudaStream_t stream) {
    if (g.M <= 0 || g.N <= 0 || batch <= 0) return cudaSuccess;
    dim3 grid((g.N + BN - 1) / BN, (g.M + BM - 1) / BM, batch);
    k_dgemm_nt<<<grid, 128, 0, stream>>>(g);
    return cudaGetLastError();
}

}  // namespace hf
