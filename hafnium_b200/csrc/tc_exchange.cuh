#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "jk.cuh"

namespace hf {

// Shapes of the split-BF16 exchange: n padded to 128 (npad), the factor's
// columns padded to opad = n_tiles1 * bn1 (bn1 a multiple of 16, <= 256).
struct TcPlan {
    int64_t npad;
    int opad, bn1, n_tiles1;
    int naux;
};

TcPlan tc_plan(int64_t n, int naux, int64_t ncols);
// Bytes of the full BF16 hi/lo copies of B.
size_t tc_b_bytes(int64_t n, int naux);
// Bytes of stage 2's per-split partial sums, carved from exchange_build_bf16's
// work area ahead of the X chunk (a multiple of 256).
size_t tc_partial_bytes(int64_t npad);
// Fill the BF16 hi/lo copies ([naux][npad][npad] each, hi first) from the FP64 tiles.
cudaError_t tc_split_b(const JkPlan& p, int64_t npad, void* bf16_b, cudaStream_t stream);
// The pipeline's bounded waits: err (device int, zeroed by the caller) is set to
// 1 when a wait runs out after wait_ns; stall makes the first stage-1 launch
// wait once on a barrier that nothing completes (a self-test of that path).
struct TcWait {
    int* err;
    uint64_t wait_ns;
    int stall;
};

// K = sum_q (B_q C) diag(sign) (B_q C)^T with split-BF16 products; Ct_fp64 is
// [opad][npad] (zero padded), sign [opad] device or null for all +1. work (256-byte
// aligned) holds the BF16 factor, stage 2's per-split FP32 partial sums
// (tc_partial_bytes) and one chunk of X (and of X diag(sign)); Kp is npad x npad
// scratch. The sum over k splits runs in a fixed order, so K is reproducible.
cudaError_t exchange_build_bf16(const TcPlan& t, const void* bf16_b, const double* Ct_fp64, int64_t ct_ld, double* K,
                                double* Kp, void* work, size_t work_bytes, const TcWait& wait, cudaStream_t stream, int64_t n,
                                const double* sign = nullptr);

}  // namespace hf
