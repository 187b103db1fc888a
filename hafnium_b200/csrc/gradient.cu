// The DF-RHF nuclear gradient's derivative-integral kernels
// (gradient_kernels.cuh), in their own translation unit with their own copy of
// the constant tables the integral kernels read.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

#include "integrals.cuh"
#include "md.cuh"

namespace hf {

namespace {
__constant__ double c_c2s[kC2sSize];
__constant__ int c_tet_t[ntet(8)];
__constant__ int c_tet_u[ntet(8)];
__constant__ int c_tet_v[ntet(8)];
__constant__ int c_cart[kMaxAuxL + 1][15][3];
}  // namespace

void upload_gradient_tables(cudaStream_t stream) {
    static std::mutex mutex;
    static bool done[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
    std::lock_guard<std::mutex> lock(mutex);
    if (done[dev]) return;
    const ConstantTables t = constant_tables_host();
    cudaMemcpyToSymbolAsync(c_c2s, t.c2s, sizeof(t.c2s), 0, cudaMemcpyHostToDevice, stream);
    cudaMemcpyToSymbolAsync(c_tet_t, t.tet_t, sizeof(t.tet_t), 0, cudaMemcpyHostToDevice, stream);
    cudaMemcpyToSymbolAsync(c_tet_u, t.tet_u, sizeof(t.tet_u), 0, cudaMemcpyHostToDevice, stream);
    cudaMemcpyToSymbolAsync(c_tet_v, t.tet_v, sizeof(t.tet_v), 0, cudaMemcpyHostToDevice, stream);
    cudaMemcpyToSymbolAsync(c_cart, t.cart, sizeof(t.cart), 0, cudaMemcpyHostToDevice, stream);
    done[dev] = cudaStreamSynchronize(stream) == cudaSuccess;
}

}  // namespace hf

#include "gradient_kernels.cuh"
