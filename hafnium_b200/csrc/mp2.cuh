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
// The fitted tensor in an orbital basis (hafnium/orbitals/integrals.py:73-157,
// transform_df_tensor, restricted real orbitals): out[P][p][q] =
// sum_uv Cb[u][p] B_P[u][v] Ck[v][q] with Cb [n][nb], Ck [n][nk] (device); row P
// goes to out row ref[P] (device array) or P when ref is null.
cudaError_t mo_fitted_tensor(const JkPlan& p, const double* Cb, int64_t nb, const double* Ck, int64_t nk,
                             const int* ref, double* out, cudaStream_t stream);

cudaError_t occupied_pair_tensor_t(const JkPlan& p, const double* C, int64_t ncol, int64_t nocc, double* Gt,
                                   cudaStream_t stream);

}  // namespace hf
