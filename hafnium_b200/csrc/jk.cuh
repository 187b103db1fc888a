#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace hf {

// The packed fitted tensor as the J and K builds see it. One cluster, or a
// batch of `count` clusters of equal shape whose tensors are listed in the
// device table Btab (B is then ignored).
struct JkPlan {
    const double* B;  // [naux][ntiles][64][64]
    int64_t ldb;      // ntiles * 4096
    int64_t n;        // orbital functions
    int nt;           // 64-wide tiles per side (n padded to 64 nt)
    int64_t ntiles;   // nt (nt + 1) / 2
    int naux;
    const double* const* Btab = nullptr;  // [count] per-cluster tensors (device)
    int count = 1;
    const int* active = nullptr;  // [count]: clusters whose entry is 0 are skipped
};

// J = scale * sum_q (B_q . D) B_q for a full symmetric n x n D (device), J full
// n x n; per cluster c: D + c strideD, J + c strideJ, work + c coulomb_work_doubles.
cudaError_t coulomb_build(const JkPlan& p, const double* D, int64_t strideD, double scale, double* J, int64_t strideJ,
                          double* work, cudaStream_t stream);
inline cudaError_t coulomb_build(const JkPlan& p, const double* D, double* J, double* work, cudaStream_t stream) {
    return coulomb_build(p, D, 0, 1.0, J, 0, work, stream);
}
int64_t coulomb_work_doubles(const JkPlan& p);  // per cluster

// d[q] = sum_{mu nu} B_q[mu][nu] D[mu][nu] for a full symmetric n x n D (one
// cluster): the fitted charges, the first half of the J build; work holds
// coulomb_work_doubles(p) doubles.
cudaError_t fitted_charges(const JkPlan& p, const double* D, double* d, double* work, cudaStream_t stream);

// K = sum_q (B_q C) diag(sign) (B_q C)^T. Ct: [opad][npad] (C^T, zero padded,
// opad a multiple of 64). sign: [opad] or null for all +1 (single cluster only).
// Kp: npad x npad scratch; X, Xs: npad x (qchunk * opad) scratch (Xs only when
// sign != null); partial: syrk_partial_doubles(npad, count) doubles (may be null
// when that is 0). Per cluster c: Ct + c strideCt, K + c strideK, Kp + c npad^2,
// X + c npad qchunk opad.
cudaError_t exchange_build_fp64(const JkPlan& p, const double* Ct, int64_t strideCt, int opad, const double* sign,
                                double* K, int64_t strideK, double* Kp, double* X, double* Xs, double* partial,
                                int qchunk, cudaStream_t stream);
inline cudaError_t exchange_build_fp64(const JkPlan& p, const double* Ct, int opad, const double* sign, double* K,
                                       double* Kp, double* X, double* Xs, double* partial, int qchunk,
                                       cudaStream_t stream) {
    return exchange_build_fp64(p, Ct, 0, opad, sign, K, 0, Kp, X, Xs, partial, qchunk, stream);
}

// Split-K factor of the K = X X^T product for `count` clusters of padded size
// npad (enough CTAs for about twelve per SM, at most 32 splits), and the
// partial-product scratch it needs.
int syrk_splits(int64_t npad, int count);
int64_t syrk_partial_doubles(int64_t npad, int count);

// Pivoted Cholesky of `count` symmetric PSD n x n matrices (D + c strideD), one
// CTA each: rows of Lc + c strideL ([rank][n]) with D ~= Lc^T Lc, stopping after
// maxr rows or when the largest remaining diagonal entry falls to tol times the
// largest initial one. info[2c] = rank, info[2c + 1] = 1 when D is indefinite.
// n <= 22000 (the pivot state lives in shared memory).
cudaError_t pivoted_cholesky(const double* D, int64_t strideD, int n, double tol, int maxr, double* Lc,
                             int64_t strideL, int* info, int count, const int* active, cudaStream_t stream);

// The same factorisation of one matrix, blocked: a working copy of D in `work`
// (pivoted_cholesky_work_doubles(n) doubles, device) is updated by a DMMA
// product once per panel of 32 pivots; the pivots and the factor are those of
// pivoted_cholesky up to rounding. info[0] = rank, info[1] = 1 when indefinite.
size_t pivoted_cholesky_work_doubles(int n);
cudaError_t pivoted_cholesky_blocked(const double* D, int n, double tol, int maxr, double* Lc, int* info,
                                     double* work, cudaStream_t stream);

// Ct[i][mu] = Lc[i][mu] (i < info[2c], mu < n), zero padded to [opad][npad] per
// cluster; sign[i] = 1 when sign is given.
cudaError_t factor_pad(const double* Lc, int64_t strideL, int64_t n, const int* info, double* Ct, int64_t strideCt,
                       int64_t npad, int64_t opad, double* sign, int count, const int* active, cudaStream_t stream);

// Xt[(ql, i)][p] = sum_r B_{q0+ql}[p][r] Ct[i][r] for ql < qc, i < opad (one
// cluster): the half-transform with the orbital index outermost, row stride npad.
cudaError_t half_transform_t(const JkPlan& p, const double* Ct, int opad, int q0, int qc, double* Xt,
                             cudaStream_t stream);

// Sets the kernel attributes on the current device (done lazily by the builds;
// call it before a stream capture).
cudaError_t jk_configure();

}  // namespace hf
