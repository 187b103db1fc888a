// DF-MP2 correlation energy of a restricted reference from the packed fitted
// tensor (hafnium/mp/mp2.py:68-176, second_order for a closed shell):
//
//   E2 = sum_ij sum_ab (ia|jb) [2 (ia|jb) - (ib|ja)] / (e_i + e_j - e_a - e_b),
//   (ia|jb) = sum_Q B_Q,ia B_Q,jb,  B_Q,ia = sum_pq C_pi B_Q,pq C_qa.
//
// 1. Xt[(Q, i)][p] = (B_Q C_occ)^T, the exchange half-transform (DMMA) with
//    the occupied index outermost, over chunks of Q.
// 2. W[(Q, i)][a] = Xt C_vir (DMMA GEMM), then a transpose into
//    Bt[i][a][Q] so that Q is the contiguous (reduction) index.
// 3. For each i, V_j = Bt[i] Bt[j]^T for all j >= i in one batched DMMA GEMM,
//    and one CTA per pair reduces V against the denominators.
// Pair energies are summed on the host in a fixed order.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "dgemm.cuh"
#include "jk.cuh"
#include "mp2.cuh"

namespace hf {

namespace {

// Bt[(i * nv + a) * naux + q0 + ql] = W[(ql * opad + i) * vld + a]
__global__ void k_transpose_ov(const double* __restrict__ W, int64_t vld, int opad, int qc, int no, int nv,
                               int64_t naux, int q0, double* __restrict__ Bt) {
    __shared__ double tile[32][33];
    const int64_t f0 = (int64_t)blockIdx.x * 32;  // flat (i, a)
    const int ql0 = blockIdx.y * 32;
    const int64_t nflat = (int64_t)no * nv;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int ql = ql0 + r;
        const int64_t f = f0 + threadIdx.x;
        double v = 0.0;
        if (ql < qc && f < nflat) {
            const int i = (int)(f / nv), a = (int)(f % nv);
            v = W[((int64_t)ql * opad + i) * vld + a];
        }
        tile[r][threadIdx.x] = v;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int64_t f = f0 + r;
        const int ql = ql0 + threadIdx.x;
        if (ql < qc && f < nflat) Bt[f * naux + q0 + ql] = tile[threadIdx.x][r];
    }
}

// e[j] = sum_ab V_j[a][b] (2 V_j[a][b] - V_j[b][a]) / (e_i + e_{i+j} - e_a - e_b)
__global__ void __launch_bounds__(256) k_mp2_pairs(const double* __restrict__ V, int nv, int i,
                                                   const double* __restrict__ eo, const double* __restrict__ ev,
                                                   double* __restrict__ pair) {
    __shared__ double red[32];
    const int j = i + blockIdx.x;
    const double* v = V + (int64_t)blockIdx.x * nv * nv;
    const double eij = eo[i] + eo[j];
    double s = 0.0;
    for (int64_t e = threadIdx.x; e < (int64_t)nv * nv; e += blockDim.x) {
        const int a = (int)(e / nv), b = (int)(e % nv);
        const double x = v[e];
        s += x * (2.0 * x - v[(int64_t)b * nv + a]) / (eij - ev[a] - ev[b]);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        pair[j] = t;
    }
}

// Ct[i][p] = C[p][col0 + i] (i < cols, p < n), zero padded to [rows][npad].
__global__ void k_columns_t(const double* __restrict__ C, int64_t n, int64_t ncol, int64_t col0, int64_t cols,
                            double* __restrict__ Ct, int64_t rows, int64_t npad) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= rows * npad) return;
    const int64_t i = e / npad, p = e % npad;
    Ct[e] = (i < cols && p < n) ? C[p * ncol + col0 + i] : 0.0;
}

int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

}  // namespace

cudaError_t occupied_pair_tensor_t(const JkPlan& p, const double* C, int64_t ncol, int64_t nocc, double* Gt,
                                   cudaStream_t stream) {
    const int64_t n = p.n, npad = (int64_t)p.nt * 64, naux = p.naux;
    if (nocc < 1) return cudaSuccess;
    const int opad = (int)std::max<int64_t>(64, round_up(nocc, 64));
    const int64_t per_q = (int64_t)opad * (npad + opad) * 8;
    const int qc_max = (int)std::max<int64_t>(1, std::min<int64_t>(naux, ((int64_t)1 << 30) / per_q));
    double *Cot = nullptr, *Xt = nullptr, *W = nullptr;
    cudaError_t e;
    if ((e = cudaMallocAsync((void**)&Cot, sizeof(double) * (size_t)opad * npad, stream)) != cudaSuccess) return e;
    if ((e = cudaMallocAsync((void**)&Xt, sizeof(double) * (size_t)qc_max * opad * npad, stream)) != cudaSuccess ||
        (e = cudaMallocAsync((void**)&W, sizeof(double) * (size_t)qc_max * opad * opad, stream)) != cudaSuccess) {
        cudaFreeAsync(Cot, stream);
        if (Xt) cudaFreeAsync(Xt, stream);
        return e;
    }
    k_columns_t<<<(unsigned)((opad * npad + 255) / 256), 256, 0, stream>>>(C, n, ncol, 0, nocc, Cot, opad, npad);
    for (int q0 = 0; q0 < naux && e == cudaSuccess; q0 += qc_max) {
        const int qc = (int)std::min<int64_t>(qc_max, naux - q0);
        e = half_transform_t(p, Cot, opad, q0, qc, Xt, stream);
        if (e != cudaSuccess) break;
        GemmArgs g{};
        g.M = qc * opad;
        g.N = (int)nocc;
        g.K = (int)npad;
        g.A = Xt;
        g.lda = npad;
        g.B = Cot;
        g.ldb = npad;
        g.C = W;
        g.ldc = opad;
        g.alpha = 1.0;
        g.beta = 0.0;
        e = dgemm_nt(g, 1, stream);
        if (e != cudaSuccess) break;
        dim3 grid((unsigned)((nocc * nocc + 31) / 32), (unsigned)((qc + 31) / 32));
        k_transpose_ov<<<grid, dim3(32, 8), 0, stream>>>(W, opad, opad, qc, (int)nocc, (int)nocc, naux, q0, Gt);
        e = cudaGetLastError();
    }
    cudaFreeAsync(Cot, stream);
    cudaFreeAsync(Xt, stream);
    cudaFreeAsync(W, stream);
    return e;
}

// out[Q'][i][a] = W[(ql * bpad + i) * kpad + a] for Q = q0 + ql, Q' = ref[Q] (or Q).
__global__ void k_scatter_mo(const double* __restrict__ W, int bpad, int64_t kpad, int qc, int q0, int64_t nb,
                             int64_t nk, const int* __restrict__ ref, double* __restrict__ out) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t per_q = nb * nk;
    if (e >= per_q * qc) return;
    const int ql = (int)(e / per_q);
    const int64_t r = e % per_q;
    const int64_t i = r / nk, a = r % nk;
    const int64_t q = ref ? ref[q0 + ql] : q0 + ql;
    out[q * per_q + r] = W[((int64_t)ql * bpad + i) * kpad + a];
}

cudaError_t mo_fitted_tensor(const JkPlan& p, const double* Cb, int64_t nb, const double* Ck, int64_t nk,
                             const int* ref, double* out, cudaStream_t stream) {
    const int64_t n = p.n, npad = (int64_t)p.nt * 64, naux = p.naux;
    if (nb < 1 || nk < 1) return cudaSuccess;
    const int bpad = (int)std::max<int64_t>(64, round_up(nb, 64));
    const int64_t kpad = round_up(nk, 64);
    const int64_t per_q = (int64_t)bpad * (npad + kpad) * 8;
    const int qc_max = (int)std::max<int64_t>(1, std::min<int64_t>(naux, ((int64_t)1 << 30) / per_q));
    double *Cbt = nullptr, *Ckt = nullptr, *Xt = nullptr, *W = nullptr;
    cudaError_t e;
    if ((e = cudaMallocAsync((void**)&Cbt, sizeof(double) * (size_t)bpad * npad, stream)) != cudaSuccess) return e;
    if ((e = cudaMallocAsync((void**)&Ckt, sizeof(double) * (size_t)kpad * npad, stream)) != cudaSuccess ||
        (e = cudaMallocAsync((void**)&Xt, sizeof(double) * (size_t)qc_max * bpad * npad, stream)) != cudaSuccess ||
        (e = cudaMallocAsync((void**)&W, sizeof(double) * (size_t)qc_max * bpad * kpad, stream)) != cudaSuccess) {
        cudaFreeAsync(Cbt, stream);
        if (Ckt) cudaFreeAsync(Ckt, stream);
        if (Xt) cudaFreeAsync(Xt, stream);
        return e;
    }
    k_columns_t<<<(unsigned)((bpad * npad + 255) / 256), 256, 0, stream>>>(Cb, n, nb, 0, nb, Cbt, bpad, npad);
    k_columns_t<<<(unsigned)((kpad * npad + 255) / 256), 256, 0, stream>>>(Ck, n, nk, 0, nk, Ckt, kpad, npad);
    for (int q0 = 0; q0 < naux && e == cudaSuccess; q0 += qc_max) {
        const int qc = (int)std::min<int64_t>(qc_max, naux - q0);
        e = half_transform_t(p, Cbt, bpad, q0, qc, Xt, stream);
        if (e != cudaSuccess) break;
        GemmArgs g{};
        g.M = qc * bpad;
        g.N = (int)nk;
        g.K = (int)npad;
        g.A = Xt;
        g.lda = npad;
        g.B = Ckt;
        g.ldb = npad;
        g.C = W;
        g.ldc = kpad;
        g.alpha = 1.0;
        g.beta = 0.0;
        e = dgemm_nt(g, 1, stream);
        if (e != cudaSuccess) break;
        const int64_t cnt = nb * nk * qc;
        k_scatter_mo<<<(unsigned)((cnt + 255) / 256), 256, 0, stream>>>(W, bpad, kpad, qc, q0, nb, nk, ref, out);
        e = cudaGetLastError();
    }
    cudaFreeAsync(Cbt, stream);
    cudaFreeAsync(Ckt, stream);
    cudaFreeAsync(Xt, stream);
    cudaFreeAsync(W, stream);
    return e;
}

cudaError_t mp2_energy(const JkPlan& p, const double* C, int64_t nmo, const double* eps, int64_t nocc,
                       double* correlation, cudaStream_t stream) {
    const int64_t n = p.n, npad = (int64_t)p.nt * 64, naux = p.naux;
    const int64_t nv = nmo - nocc;
    if (nocc < 1 || nv < 1) {
        *correlation = 0.0;
        return cudaSuccess;
    }
    const int opad = (int)std::max<int64_t>(64, round_up(nocc, 64));
    const int64_t vpad = round_up(nv, 64);
    // Q chunk: Xt and W for qc auxiliary functions within ~1 GB
    const int64_t per_q = (int64_t)opad * (npad + vpad) * 8;
    const int qc_max = (int)std::max<int64_t>(1, std::min<int64_t>(naux, ((int64_t)1 << 30) / per_q));
    double *Cot = nullptr, *Cvt = nullptr, *Xt = nullptr, *W = nullptr, *Bt = nullptr, *V = nullptr, *pair = nullptr;
    double* eps_d = nullptr;
    auto grab = [&](double** ptr, int64_t doubles) {
        return cudaMallocAsync((void**)ptr, sizeof(double) * std::max<int64_t>(doubles, 1), stream);
    };
    cudaError_t e;
    if ((e = grab(&Cot, (int64_t)opad * npad)) != cudaSuccess || (e = grab(&Cvt, vpad * npad)) != cudaSuccess ||
        (e = grab(&Xt, (int64_t)qc_max * opad * npad)) != cudaSuccess ||
        (e = grab(&W, (int64_t)qc_max * opad * vpad)) != cudaSuccess ||
        (e = grab(&Bt, nocc * nv * naux)) != cudaSuccess || (e = grab(&V, nocc * nv * nv)) != cudaSuccess ||
        (e = grab(&pair, nocc * nocc)) != cudaSuccess || (e = grab(&eps_d, nmo)) != cudaSuccess) {
        cudaFreeAsync(Cot, stream), cudaFreeAsync(Cvt, stream), cudaFreeAsync(Xt, stream), cudaFreeAsync(W, stream);
        cudaFreeAsync(Bt, stream), cudaFreeAsync(V, stream), cudaFreeAsync(pair, stream), cudaFreeAsync(eps_d, stream);
        return e;
    }
    cudaMemcpyAsync(eps_d, eps, sizeof(double) * nmo, cudaMemcpyDeviceToDevice, stream);
    k_columns_t<<<(unsigned)((opad * npad + 255) / 256), 256, 0, stream>>>(C, n, nmo, 0, nocc, Cot, opad, npad);
    k_columns_t<<<(unsigned)((vpad * npad + 255) / 256), 256, 0, stream>>>(C, n, nmo, nocc, nv, Cvt, vpad, npad);
    for (int q0 = 0; q0 < naux && e == cudaSuccess; q0 += qc_max) {
        const int qc = (int)std::min<int64_t>(qc_max, naux - q0);
        e = half_transform_t(p, Cot, opad, q0, qc, Xt, stream);
        if (e != cudaSuccess) break;
        GemmArgs g{};
        g.M = qc * opad;
        g.N = (int)nv;
        g.K = (int)npad;
        g.A = Xt;
        g.lda = npad;
        g.B = Cvt;
        g.ldb = npad;
        g.C = W;
        g.ldc = vpad;
        g.alpha = 1.0;
        g.beta = 0.0;
        e = dgemm_nt(g, 1, stream);
        if (e != cudaSuccess) break;
        dim3 grid((unsigned)((nocc * nv + 31) / 32), (unsigned)((qc + 31) / 32));
        k_transpose_ov<<<grid, dim3(32, 8), 0, stream>>>(W, vpad, opad, qc, (int)nocc, (int)nv, naux, q0, Bt);
        e = cudaGetLastError();
    }
    for (int64_t i = 0; i < nocc && e == cudaSuccess; ++i) {
        const int cnt = (int)(nocc - i);
        GemmArgs g{};
        g.M = g.N = (int)nv;
        g.K = (int)naux;
        g.A = Bt + i * nv * naux;
        g.lda = naux;
        g.B = Bt + i * nv * naux;
        g.ldb = naux;
        g.C = V;
        g.ldc = nv;
        g.alpha = 1.0;
        g.beta = 0.0;
        g.strideA = 0;
        g.strideB = nv * naux;
        g.strideC = nv * nv;
        e = dgemm_nt(g, cnt, stream);
        if (e != cudaSuccess) break;
        k_mp2_pairs<<<cnt, 256, 0, stream>>>(V, (int)nv, (int)i, eps_d, eps_d + nocc, pair + i * nocc);
        e = cudaGetLastError();
    }
    std::vector<double> h((size_t)nocc * nocc, 0.0);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h.data(), pair, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, stream);
    cudaFreeAsync(Cot, stream), cudaFreeAsync(Cvt, stream), cudaFreeAsync(Xt, stream), cudaFreeAsync(W, stream);
    cudaFreeAsync(Bt, stream), cudaFreeAsync(V, stream), cudaFreeAsync(pair, stream), cudaFreeAsync(eps_d, stream);
    const cudaError_t s = cudaStreamSynchronize(stream);
    if (e == cudaSuccess) e = s;
    if (e != cudaSuccess) return e;
    double total = 0.0;
    for (int64_t i = 0; i < nocc; ++i)
        for (int64_t j = i; j < nocc; ++j) total += (j == i ? 1.0 : 2.0) * h[(size_t)i * nocc + j];
    *correlation = total;
    return cudaSuccess;
}

}  // namespace hf
