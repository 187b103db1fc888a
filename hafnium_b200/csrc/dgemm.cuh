// FP64 tensor-core GEMM for sm_100a: C = alpha * A * Bop^T + beta * C.
//
// Both operands are K-contiguous ("NT"): A[m][k] with row stride lda, Bop[n][k]
// with row stride ldb. 64x64x16 CTA tiles, 4 warps of 32x32, DMMA
// mma.sync.m8n8k4.f64 (the FP64 tensor path; tcgen05 has no FP64 kind).
// Global tiles are staged through registers into shared memory stored
// k-major ([k][m], padded so a fragment load touches every bank once per
// half-warp), double-buffered across k-steps.
//
// kmode restricts the k range per output tile (triangular operands):
//   0: [0, K)   1: [n0, K) (Bop upper: Bop[n][k] = 0 for k < n)
//   2: [0, min(K, m0 + 64)) (A lower: A[m][k] = 0 for k > m)
// epi selects the store:
//   0: C[m][n] (row stride ldc)      1: C[n][m] (transposed store)
//   2: as 0, only tiles touching the lower triangle (n0 <= m0 + 63)
//   3: as 0, only tiles touching the upper triangle (m0 <= n0 + 63)
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace hf {

struct GemmArgs {
    int M, N, K;
    const double* A;
    int64_t lda;
    const double* B;
    int64_t ldb;
    double* C;
    int64_t ldc;
    double alpha, beta;
    int kmode, epi;
    // Optional batching over blockIdx.z: pointer strides per batch.
    int64_t strideA, strideB, strideC;
};

cudaError_t dgemm_nt(const GemmArgs& g, int batch, cudaStream_t stream);

__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

}  // namespace hf
