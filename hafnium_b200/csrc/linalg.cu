// FP64 Cholesky of the Coulomb metric, the inverse of its factor, and the
// formation of the fitted tensor B = L^{-1} (P|mu nu).
//
// The reference forms B = M^{-1/2} (P|mu nu) from an eigendecomposition,
// dropping eigenvalues below 1e-10 of the largest
// (hafnium/integrals/density_fitting.py:97-107, 181-197). Any factor with
// L L^T = M gives the same fitted integrals B^T B when nothing is dropped
// (the invariance the reference tests at tests/unit/test_density_fitting.py:177-195),
// so a Cholesky factor replaces the inverse square root. The smallest pivot
// relative to the largest diagonal is reported so the caller can see how close
// the metric is to the reference's drop threshold.
#include <cmath>

#include "dgemm.cuh"
#include "linalg.cuh"

namespace hf {

namespace {
constexpr int NB = 64;

// Factor the nb x nb diagonal block at (k0, k0) in place (lower), unblocked, by
// 256 threads (a 16 x 16 grid over the trailing triangle). Per column every
// thread takes the pivot's square root itself, so a column needs two barriers:
// after its scaling and after the trailing update (during which thread 0 stores
// the pivot, which no thread reads then).
__global__ void __launch_bounds__(256) k_potrf_diag(double* A, int64_t lda, int k0, int nb, int* info,
                                                    double* piv_min) {
    __shared__ double a[NB][NB + 1];
    const int tid = threadIdx.x;
    for (int e = tid; e < nb * nb; e += blockDim.x) {
        const int i = e / nb, j = e % nb;
        a[i][j] = (j <= i) ? A[(int64_t)(k0 + i) * lda + k0 + j] : 0.0;
    }
    __syncthreads();
    for (int j = 0; j < nb; ++j) {
        const double d = a[j][j];
        const bool bad = !(d > 0.0);
        const double r = bad ? 1.0 : sqrt(d);
        for (int i = j + 1 + tid; i < nb; i += blockDim.x) a[i][j] /= r;
        __syncthreads();
        if (tid == 0) {
            if (bad) atomicExch(info, k0 + j + 1);
            else if (r < *piv_min) *piv_min = r;
            a[j][j] = r;
        }
        // trailing update of the lower triangle, threads as a 16 x 16 grid over (i, l)
        for (int i = j + 1 + (tid >> 4); i < nb; i += 16) {
            const double aij = a[i][j];
            for (int l = j + 1 + (tid & 15); l <= i; l += 16) a[i][l] -= aij * a[l][j];
        }
        __syncthreads();
    }
    for (int e = tid; e < nb * nb; e += blockDim.x) {
        const int i = e / nb, j = e % nb;
        A[(int64_t)(k0 + i) * lda + k0 + j] = (j <= i) ? a[i][j] : 0.0;
    }
}

// Rows below the diagonal block: L_ik = A_ik L_kk^{-T}, one thread per row, by
// forward substitution in right-looking order: once x[q] is known it is
// subtracted from every later entry, so the 64 entries' updates are independent
// of one another (the same operations, in the same order per entry, as summing
// each entry's terms before its division).
__global__ void __launch_bounds__(128) k_trsm_panel(double* A, int64_t lda, int k0, int nb, int n) {
    __shared__ double l[NB][NB + 1];
    for (int e = threadIdx.x; e < NB * NB; e += blockDim.x) {
        const int i = e / NB, j = e % NB;
        l[i][j] = (i < nb && j < nb) ? A[(int64_t)(k0 + i) * lda + k0 + j] : 0.0;
    }
    __syncthreads();
    const int row = k0 + nb + blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n) return;
    double* r = A + (int64_t)row * lda + k0;
    double x[NB];
#pragma unroll
    for (int j = 0; j < NB; ++j) x[j] = (j < nb) ? r[j] : 0.0;
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        if (q < nb) {
            x[q] = x[q] / l[q][q];
#pragma unroll
            for (int j = q + 1; j < NB; ++j) x[j] -= x[q] * l[j][q];
        }
    }
#pragma unroll
    for (int j = 0; j < NB; ++j)
        if (j < nb) r[j] = x[j];
}

__global__ void k_zero_upper(double* A, int64_t lda, int n) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)n * n) return;
    const int i = (int)(e / n), j = (int)(e % n);
    if (j > i) A[(int64_t)i * lda + j] = 0.0;
}

// Inverse of the lower-triangular diagonal blocks (k0, k0), k0 = 64 blockIdx.x,
// all at once (they are independent): one CTA per block, one thread per column,
// forward substitution. Writes Linv (row-major) and LinvT.
__global__ void __launch_bounds__(64) k_trtri_diag(const double* L, int64_t ld, int n, double* Linv,
                                                   double* LinvT) {
    const int k0 = blockIdx.x * NB;
    const int nb = (n - k0 < NB) ? n - k0 : NB;
    __shared__ double l[NB][NB + 1];
    for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
        const int i = e / nb, j = e % nb;
        l[i][j] = L[(int64_t)(k0 + i) * ld + k0 + j];
    }
    __syncthreads();
    const int c = threadIdx.x;
    if (c >= nb) return;
    double x[NB];
#pragma unroll
    for (int r = 0; r < NB; ++r) {
        if (r >= nb) continue;
        double v;
        if (r < c) v = 0.0;
        else if (r == c) v = 1.0 / l[c][c];
        else {
            double s = 0.0;
#pragma unroll
            for (int q = 0; q < r; ++q)
                if (q >= c) s += l[r][q] * x[q];
            v = -s / l[r][r];
        }
        x[r] = v;
    }
#pragma unroll
    for (int r = 0; r < NB; ++r) {
        if (r >= nb) continue;
        Linv[(int64_t)(k0 + r) * ld + k0 + c] = x[r];
        LinvT[(int64_t)(k0 + c) * ld + k0 + r] = x[r];
    }
}

__global__ void k_transpose(const double* in, double* out, int n, int64_t ld) {
    __shared__ double t[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int r = by + j, c = bx + threadIdx.x;
        t[j][threadIdx.x] = (r < n && c < n) ? in[(int64_t)r * ld + c] : 0.0;
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int r = bx + j, c = by + threadIdx.x;
        if (r < n && c < n) out[(int64_t)r * ld + c] = t[threadIdx.x][j];
    }
}
}  // namespace

cudaError_t cholesky_lower(double* A, int n, int64_t lda, int* d_info, double* d_piv_min, cudaStream_t stream) {
    for (int k0 = 0; k0 < n; k0 += NB) {
        const int nb = (n - k0 < NB) ? n - k0 : NB;
        k_potrf_diag<<<1, 256, 0, stream>>>(A, lda, k0, nb, d_info, d_piv_min);
        const int rem = n - k0 - nb;
        if (rem > 0) {
            k_trsm_panel<<<(rem + 127) / 128, 128, 0, stream>>>(A, lda, k0, nb, n);
            GemmArgs g{};
            g.M = g.N = rem;
            g.K = nb;
            g.A = g.B = A + (int64_t)(k0 + nb) * lda + k0;
            g.lda = g.ldb = lda;
            g.C = A + (int64_t)(k0 + nb) * lda + k0 + nb;
            g.ldc = lda;
            g.alpha = -1.0;
            g.beta = 1.0;
            g.kmode = 0;
            g.epi = 2;
            cudaError_t e = dgemm_nt(g, 1, stream);
            if (e != cudaSuccess) return e;
        }
    }
    const int64_t total = (int64_t)n * n;
    k_zero_upper<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(A, lda, n);
    return cudaGetLastError();
}

cudaError_t triangular_inverse(const double* L, int n, int64_t ld, double* Linv, double* LinvT, double* work,
                               cudaStream_t stream) {
    cudaMemsetAsync(Linv, 0, sizeof(double) * (size_t)n * ld, stream);
    cudaMemsetAsync(LinvT, 0, sizeof(double) * (size_t)n * ld, stream);
    k_trtri_diag<<<(n + NB - 1) / NB, 64, 0, stream>>>(L, ld, n, Linv, LinvT);
    for (int k0 = NB; k0 < n; k0 += NB) {
        const int nb = (n - k0 < NB) ? n - k0 : NB;
        // Wt[c][m] = sum_{k in [c, k0)} L[k0 + m][k] Linv[k][c]   (c < k0)
        GemmArgs g{};
        g.M = nb;
        g.N = k0;
        g.K = k0;
        g.A = L + (int64_t)k0 * ld;
        g.lda = ld;
        g.B = LinvT;
        g.ldb = ld;
        g.C = work;
        g.ldc = NB;
        g.alpha = 1.0;
        g.beta = 0.0;
        g.kmode = 1;
        g.epi = 1;
        cudaError_t e = dgemm_nt(g, 1, stream);
        if (e != cudaSuccess) return e;
        // Linv[k0 + m][c] = -sum_j Linv_kk[m][j] W[j][c]; stored transposed into LinvT.
        GemmArgs h{};
        h.M = nb;
        h.N = k0;
        h.K = nb;
        h.A = Linv + (int64_t)k0 * ld + k0;
        h.lda = ld;
        h.B = work;
        h.ldb = NB;
        h.C = LinvT + k0;
        h.ldc = ld;
        h.alpha = -1.0;
        h.beta = 0.0;
        h.kmode = 0;
        h.epi = 1;
        e = dgemm_nt(h, 1, stream);
        if (e != cudaSuccess) return e;
    }
    dim3 grid((n + 31) / 32, (n + 31) / 32);
    k_transpose<<<grid, dim3(32, 8), 0, stream>>>(LinvT, Linv, n, ld);
    return cudaGetLastError();
}

cudaError_t apply_inverse_factor(const double* Linv, int n, int64_t ld, const double* T, int64_t ldt, int64_t ncols,
                                 double* B, int64_t ldb, cudaStream_t stream, int row0, int row1) {
    if (row1 < 0) row1 = n;
    GemmArgs g{};
    g.M = row1 - row0;
    g.N = (int)ncols;
    g.K = row1;  // L^-1 is lower triangular: rows below row1 need columns below row1
    g.koff = row0;
    g.A = Linv + (int64_t)row0 * ld;
    g.lda = ld;
    g.B = T;
    g.ldb = ldt;
    g.C = B;
    g.ldc = ldb;
    g.alpha = 1.0;
    g.beta = 0.0;
    g.kmode = 2;
    g.epi = 0;
    g.tile = 5;  // 64 x 64 with 2 stages of 32-wide k slices: the fastest tile for this product
    return dgemm_nt(g, 1, stream);
}

}  // namespace hf
