#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace hf {

// The packed fitted tensor as the J and K builds see it.
struct JkPlan {
    const double* B;  // [naux][ntiles][64][64]
    int64_t ldb;      // ntiles * 4096
    int64_t n;        // orbital functions
    int nt;           // 64-wide tiles per side (n padded to 64 nt)
    int64_t ntiles;   // nt (nt + 1) / 2
    int naux;
};

// J = sum_q (B_q . D) B_q for a full symmetric n x n D (device), J full n x n.
cudaError_t coulomb_build(const JkPlan& p, const double* D, double* J, double* work, cudaStream_t stream);
int64_t coulomb_work_doubles(const JkPlan& p);

// K = sum_q (B_q C) diag(sign) (B_q C)^T. Ct: [opad][npad] (C^T, zero padded,
// opad a multiple of 64). sign: [opad] or null for all +1. Kp: npad x npad
// scratch; X, Xs: npad x (qchunk * opad) scratch (Xs only when sign != null).
cudaError_t exchange_build_fp64(const JkPlan& p, const double* Ct, int opad, const double* sign, double* K,
                                double* Kp, double* X, double* Xs, int qchunk, cudaStream_t stream);

}  // namespace hf
