// FP64 tensor-core GEMM for sm_100a: C = alpha * A * Bop^T + beta * C.
//
// Both operands are K-contiguous ("NT"): A[m][k] with row stride lda, Bop[n][k]
// with row stride ldb. DMMA mma.sync.m16n8k8.f64 (the FP64 tensor path;
// tcgen05 has no FP64 kind), warps of 32x32 output, a cp.async pipeline of
// 3 stages of BK = 16 slices (tile 5: 2 stages of BK = 32). The CTA tile is one
// of kTileShapes (selected by `tile`): an autotuner picks the shape per problem
// size for the batched products; the fit of B and the FP64 exchange's SYRK use
// tile 5.
//
// kmode restricts the k range per output tile (triangular operands):
//   0: [0, K)   1: [n0, K) (Bop upper: Bop[n][k] = 0 for k < n)
//   2: [0, min(K, koff + m0 + BM)) (A lower: A[m][k] = 0 for k > koff + m, koff the
//      row of the full triangle that A's first row is)
// epi selects the store:
//   0: C[m][n] (row stride ldc)      1: C[n][m] (transposed store)
//   2: as 0, only tiles touching the lower triangle (n0 <= m0 + BM - 1)
//   3: as 0, only tiles touching the upper triangle (m0 <= n0 + BN - 1)
//
// Batching runs over blockIdx.z with per-batch pointer strides. Optional
// per-batch arrays: `active` (a batch whose entry is 0 is skipped and its C is
// left untouched), `alpha_v` / `beta_v` (replace alpha / beta for that batch).
// With splits > 1 each batch's k range is cut into `splits` parts whose
// products go to separate C matrices (C + (batch * splits + split) * strideC),
// for the caller to reduce: deterministic split-K.
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
    const int* active;
    const double* alpha_v;
    const double* beta_v;
    int tile;    // index into kTileShapes
    int splits;  // > 1: split-K; blockIdx.z = batch * splits + split, C + blockIdx.z * strideC
    int koff;    // kmode 2: the first row of A within its triangle
};

// CTA tile shapes (BM x BN); warps = (BM / 32) * (BN / 32).
constexpr int kTileCount = 6;
constexpr int kTileShapes[kTileCount][2] = {{128, 64}, {64, 64}, {64, 32}, {32, 32}, {128, 128}, {64, 64}};

cudaError_t dgemm_nt(const GemmArgs& g, int batch, cudaStream_t stream);  // batch: matrices (not counting splits)

// Sets the shared-memory attributes of every tile instance on the current
// device (done lazily by dgemm_nt; call it before a stream capture).
cudaError_t dgemm_configure();

}  // namespace hf
