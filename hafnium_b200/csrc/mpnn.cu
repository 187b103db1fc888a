// Kernels of the learned initial-guess network (forward, backward, Adam).
//
// The network (no counterpart in the reference; see hafnium_b200/learned/model.py)
// is a message-passing net over the waters of a cluster. Its layers are dense
// maps over rows of nodes or edges, gathers of node rows onto edges, and
// scatter-adds of edge rows onto nodes; these kernels implement those pieces
// in FP32 and are driven from Python through the C ABI of include/hfnn.h.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/hfnn.h"

namespace {

constexpr int TS = 64, TK = 16;

// C[M][N] = op(A) op(B) (+ bias[N]) (+= when accumulate); op(A) is A[M][K] or
// A^T with A stored [K][M]; op(B) is B[K][N] or B^T with B stored [N][K].
__global__ void __launch_bounds__(256) k_sgemm(int M, int N, int K, const float* __restrict__ A, int ta,
                                               const float* __restrict__ B, int tb, const float* __restrict__ bias,
                                               float* __restrict__ C, int accumulate) {
    __shared__ float As[TK][TS + 4];
    __shared__ float Bs[TK][TS + 4];
    const int m0 = blockIdx.y * TS, n0 = blockIdx.x * TS;
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;  // 16 x 16 threads, 4 x 4 outputs each
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += TK) {
        for (int e = threadIdx.x; e < TS * TK; e += blockDim.x) {
            const int mm = e / TK, kk = e % TK;
            const int m = m0 + mm, k = k0 + kk;
            float av = 0.f;
            if (m < M && k < K) av = ta ? A[(int64_t)k * M + m] : A[(int64_t)m * K + k];
            As[kk][mm] = av;
            const int n = n0 + mm;
            float bv = 0.f;
            if (n < N && k < K) bv = tb ? B[(int64_t)n * K + k] : B[(int64_t)k * N + n];
            Bs[kk][mm] = bv;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < TK; ++kk) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] += a[i] * b[j];
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int m = m0 + ty * 4 + i, n = n0 + tx * 4 + j;
            if (m >= M || n >= N) continue;
            float v = acc[i][j] + (bias ? bias[n] : 0.f);
            float* dst = C + (int64_t)m * N + n;
            *dst = accumulate ? *dst + v : v;
        }
}

__device__ __forceinline__ float sigm(float x) { return 1.f / (1.f + __expf(-x)); }

// Y = silu(Z) * (scale[row] or 1); optionally Y += (residual add).
__global__ void k_silu(int64_t rows, int cols, const float* __restrict__ Z, const float* __restrict__ scale,
                       float* __restrict__ Y, int add) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= rows * cols) return;
    const float z = Z[e];
    float y = z * sigm(z);
    if (scale) y *= scale[e / cols];
    Y[e] = add ? Y[e] + y : y;
}

// dZ = dY * silu'(Z) * (scale[row] or 1)
__global__ void k_dsilu(int64_t rows, int cols, const float* __restrict__ dY, const float* __restrict__ Z,
                        const float* __restrict__ scale, float* __restrict__ dZ) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= rows * cols) return;
    const float z = Z[e];
    const float s = sigm(z);
    float g = dY[e] * s * (1.f + z * (1.f - s));
    if (scale) g *= scale[e / cols];
    dZ[e] = g;
}

// out[r][col0 + c] = in[idx ? idx[r] : r][c] for c < width (out row stride ldo)
__global__ void k_gather(int64_t rows, int width, const float* __restrict__ in, const int* __restrict__ idx,
                         float* __restrict__ out, int ldo, int col0) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= rows * width) return;
    const int64_t r = e / width;
    const int c = (int)(e % width);
    const int64_t src = idx ? idx[r] : r;
    out[r * ldo + col0 + c] = in[src * width + c];
}

// out[idx ? idx[r] : r][c] += in[r][col0 + c] * (scale ? scale[r] : 1) (in row stride ldi)
__global__ void k_scatter_add(int64_t rows, int width, const float* __restrict__ in, int ldi, int col0,
                              const int* __restrict__ idx, const float* __restrict__ scale, float* __restrict__ out) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= rows * width) return;
    const int64_t r = e / width;
    const int c = (int)(e % width);
    float v = in[r * ldi + col0 + c];
    if (scale) v *= scale[r];
    const int64_t dst = idx ? idx[r] : r;
    atomicAdd(out + dst * width + c, v);
}

// out[c] = sum_r in[r][c]
__global__ void k_colsum(int64_t rows, int cols, const float* __restrict__ in, float* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float s = 0.f;
    for (int64_t r = 0; r < rows; ++r) s += in[r * cols + c];
    out[c] = s;
}

// g = 2 w (y - t); loss += w |y - t|^2
__global__ void k_sq_loss(int64_t count, const float* __restrict__ y, const float* __restrict__ t, float w,
                          float* __restrict__ g, float* __restrict__ loss) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.f;
    if (e < count) {
        const float r = y[e] - t[e];
        g[e] = 2.f * w * r;
        l = w * r * r;
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l);
}

__global__ void k_adam(int64_t count, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count) return;
    const float gi = g[e];
    const float mi = b1 * m[e] + (1.f - b1) * gi;
    const float vi = b2 * v[e] + (1.f - b2) * gi * gi;
    m[e] = mi;
    v[e] = vi;
    p[e] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

unsigned blocks(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

int status() { return cudaGetLastError() == cudaSuccess ? 0 : 3; }

}  // namespace

extern "C" {

int hfnn_sgemm(int m, int n, int k, const float* a, int ta, const float* b, int tb, const float* bias, float* c,
               int accumulate, void* stream) {
    if (m <= 0 || n <= 0) return 0;
    dim3 grid((n + TS - 1) / TS, (m + TS - 1) / TS);
    k_sgemm<<<grid, 256, 0, (cudaStream_t)stream>>>(m, n, k, a, ta, b, tb, bias, c, accumulate);
    return status();
}

int hfnn_silu(int64_t rows, int cols, const float* z, const float* scale, float* y, int add, void* stream) {
    if (rows * cols == 0) return 0;
    k_silu<<<blocks(rows * cols), 256, 0, (cudaStream_t)stream>>>(rows, cols, z, scale, y, add);
    return status();
}

int hfnn_dsilu(int64_t rows, int cols, const float* dy, const float* z, const float* scale, float* dz, void* stream) {
    if (rows * cols == 0) return 0;
    k_dsilu<<<blocks(rows * cols), 256, 0, (cudaStream_t)stream>>>(rows, cols, dy, z, scale, dz);
    return status();
}

int hfnn_gather(int64_t rows, int width, const float* in, const int* idx, float* out, int ldo, int col0,
                void* stream) {
    if (rows * width == 0) return 0;
    k_gather<<<blocks(rows * width), 256, 0, (cudaStream_t)stream>>>(rows, width, in, idx, out, ldo, col0);
    return status();
}

int hfnn_scatter_add(int64_t rows, int width, const float* in, int ldi, int col0, const int* idx, const float* scale,
                     float* out, void* stream) {
    if (rows * width == 0) return 0;
    k_scatter_add<<<blocks(rows * width), 256, 0, (cudaStream_t)stream>>>(rows, width, in, ldi, col0, idx, scale,
                                                                         out);
    return status();
}

int hfnn_colsum(int64_t rows, int cols, const float* in, float* out, void* stream) {
    if (cols == 0) return 0;
    k_colsum<<<blocks(cols), 256, 0, (cudaStream_t)stream>>>(rows, cols, in, out);
    return status();
}

int hfnn_sq_loss(int64_t count, const float* y, const float* t, float w, float* g, float* loss, void* stream) {
    if (count == 0) return 0;
    k_sq_loss<<<blocks(count), 256, 0, (cudaStream_t)stream>>>(count, y, t, w, g, loss);
    return status();
}

int hfnn_adam(int64_t count, float* p, const float* g, float* m, float* v, float lr, float b1, float b2, float eps,
              int step, void* stream) {
    if (count == 0) return 0;
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    k_adam<<<blocks(count), 256, 0, (cudaStream_t)stream>>>(count, p, g, m, v, lr, b1, b2, eps, c1, c2);
    return status();
}

}  // extern "C"
