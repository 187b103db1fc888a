#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace hf {

// In-place lower Cholesky factor of the n x n matrix A (row stride lda); the
// strict upper triangle is zeroed. *d_info becomes 1 + the first non-positive
// pivot's index; *d_piv_min tracks the smallest pivot sqrt(d).
cudaError_t cholesky_lower(double* A, int n, int64_t lda, int* d_info, double* d_piv_min, cudaStream_t stream);

// Linv = L^{-1} (row-major lower) and LinvT = its transpose. work: n x 64.
cudaError_t triangular_inverse(const double* L, int n, int64_t ld, double* Linv, double* LinvT, double* work,
                               cudaStream_t stream);

// B[q - row0][c] = sum_{q' <= q} Linv[q][q'] T[c][q'] for c < ncols and the rows
// row0 <= q < row1 of the triangle (all n rows by default; T needs columns q' < row1).
cudaError_t apply_inverse_factor(const double* Linv, int n, int64_t ld, const double* T, int64_t ldt, int64_t ncols,
                                 double* B, int64_t ldb, cudaStream_t stream, int row0 = 0, int row1 = -1);

}  // namespace hf
