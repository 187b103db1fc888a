#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "jk.cuh"

namespace hf {

// DF-MP2 correlation energy of a closed-shell reference from the packed fitted
// tensor of one cluster: C [n][nmo] device (orbitals in increasing energy, the
// first nocc occupied), eps [nmo] device. Synchronises `stream`.
cudaError_t mp2_energy(const JkPlan& p, const double* C, int64_t nmo, const double* eps, int64_t nocc,
                       double* correlation, cudaStream_t stream);

// The fitted tensor in the occupied orbital basis with the auxiliary index
// contiguous: Gt[(i * nocc + j)][Q] = sum_{pq} C[p][i] B_Q[p][q] C[q][j] for
// the first nocc columns of C [n][ncol] (device). Temporaries are stream-ordered.
cudaError_t occupied_pair_tensor_t(const JkPlan& p, const double* C, int64_t ncol, int64_t nocc, double* Gt,
                                   cudaStream_t stream);

}  // namespace hf
