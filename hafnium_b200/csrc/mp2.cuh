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

}  // namespace hf
