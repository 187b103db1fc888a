// Batched restricted SCF over many clusters of one shape, resident in one CUDA
// graph (include/hfbatch.h states the contract and the reference it follows).
//
// Layout: every per-cluster matrix is n x n row-major, clusters back to back
// (stride n^2): S, H, X = L^-T, XT = X^T, D, J, K, F, G, Fx (extrapolated F),
// two GEMM temporaries T1/T2, the purification state P, P2, Y, the pivoted
// Cholesky rows Lc, and the DIIS rings of F and of the orthonormal-basis
// gradient G (diis_size slots each). The fitted tensors stay in their own
// contexts; a device table lists them for the batched J/K kernels.
//
// One iteration (the body of the graph's WHILE node) for the clusters still
// iterating, every step a batched launch with per-cluster activity masks:
//   G = X^T (F D S - S D F) X           four DMMA GEMMs + an antisymmetrisation
//   status                               energy change, |G|, convergence, limits
//   DIIS                                 push (F, G), overlaps, bordered solve, Fx
//   F' = X^T Fx X                        two GEMMs
//   P = purify(F')                       Palser-Manolopoulos, two GEMMs per step
//   D = X P X^T                          two GEMMs + symmetrisation
//   Fock build on D                      pivoted Cholesky factor, K, J, F, energy
//   condition                            any cluster still iterating or finishing
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/hfbatch.h"
#include "context.cuh"
#include "dgemm.cuh"
#include "jk.cuh"
#include "linalg.cuh"

using namespace hf;

namespace {

// per-cluster doubles
constexpr int kScal = 8;
constexpr int S_ENUC = 0, S_ENERGY = 1, S_EPREV = 2, S_GNORM = 3, S_FINAL = 4, S_CHANGE = 5;
// per-cluster ints
constexpr int kInts = 8;
constexpr int I_STATE = 0, I_ITERS = 1, I_PUSHES = 2, I_CROSSED = 3, I_PMSTEPS = 4, I_HASPREV = 5;

constexpr int kThreads = 512;
constexpr double kNullSpaceTolerance = 1e-14;  // hafnium/scf/diis.py:17
constexpr double kOverlapThreshold = 1e-10;    // hafnium/scf/orthogonalization.py:12
constexpr double kRankTolerance = 1e-14;

__device__ double block_sum(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0) {
        for (int i = 0; i < nw; ++i) s += red[i];
        red[32] = s;
    }
    __syncthreads();
    return red[32];
}

__device__ double block_min(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = red[0];
        for (int i = 1; i < nw; ++i) s = fmin(s, red[i]);
        red[32] = s;
    }
    __syncthreads();
    return red[32];
}

__device__ double block_max(double v, double* red) { return -block_min(-v, red); }

// F = H + J - K and E = E_nuc + 2 <D,H> + <D,J> - <D,K> (hafnium/scf/hamiltonian.py:331-370,
// the restricted case: J built from 2 D, K from D).
__global__ void __launch_bounds__(kThreads) k_fock_energy(const double* __restrict__ H, const double* __restrict__ J,
                                                          const double* __restrict__ K, const double* __restrict__ D,
                                                          double* __restrict__ F, int64_t nn, double* __restrict__ scal,
                                                          const int* __restrict__ active) {
    __shared__ double red[33];
    const int c = blockIdx.x;
    if (active[c] == 0) return;
    const int64_t o = (int64_t)c * nn;
    double e1 = 0.0, ej = 0.0, ek = 0.0;
    for (int64_t i = threadIdx.x; i < nn; i += blockDim.x) {
        const double h = H[o + i], j = J[o + i], k = K[o + i], d = D[o + i];
        F[o + i] = h + j - k;
        e1 += d * h;
        ej += d * j;
        ek += d * k;
    }
    e1 = block_sum(e1, red);
    ej = block_sum(ej, red);
    ek = block_sum(ek, red);
    if (threadIdx.x == 0) scal[c * kScal + S_ENERGY] = scal[c * kScal + S_ENUC] + 2.0 * e1 + ej - ek;
}

// out = A - A^T
__global__ void k_antisymmetric(const double* __restrict__ A, double* __restrict__ out, int64_t n,
                                const int* __restrict__ active) {
    const int c = blockIdx.y;
    if (active[c] == 0) return;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * n) return;
    const int64_t o = (int64_t)c * n * n, i = e / n, j = e % n;
    out[o + e] = A[o + e] - A[o + j * n + i];
}

// out = (A + A^T) / 2
__global__ void k_symmetric(const double* __restrict__ A, double* __restrict__ out, int64_t n,
                            const int* __restrict__ active) {
    const int c = blockIdx.y;
    if (active[c] == 0) return;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * n) return;
    const int64_t o = (int64_t)c * n * n, i = e / n, j = e % n;
    out[o + e] = 0.5 * (A[o + e] + A[o + j * n + i]);
}

// Convergence bookkeeping after a Fock build (hafnium/scf/driver.py:198-213):
// ITERATING clusters get |G| = sqrt(2 sum G^2), the energy change and the test
// |dE| < etol and |G| < gtol; FINISHING clusters have just made their final
// build (driver.py:336) and are done.
__global__ void __launch_bounds__(kThreads) k_status(const double* __restrict__ G, int64_t nn, double* __restrict__ scal,
                                                     int* __restrict__ ints, int* __restrict__ act_diis,
                                                     int* __restrict__ act_next, double etol, double gtol,
                                                     int max_iterations) {
    __shared__ double red[33];
    const int c = blockIdx.x;
    int* st = ints + c * kInts;
    double* sc = scal + c * kScal;
    const int state = st[I_STATE];
    if (state == HF_SCF_ITERATING) {
        const int64_t o = (int64_t)c * nn;
        double s = 0.0;
        for (int64_t i = threadIdx.x; i < nn; i += blockDim.x) s += G[o + i] * G[o + i];
        s = block_sum(s, red);
        if (threadIdx.x == 0) {
            const double gnorm = sqrt(2.0 * s);
            const double e = sc[S_ENERGY];
            const double change = st[I_HASPREV] ? e - sc[S_EPREV] : INFINITY;
            sc[S_EPREV] = e;
            sc[S_GNORM] = gnorm;
            sc[S_CHANGE] = change;
            st[I_HASPREV] = 1;
            const int iters = ++st[I_ITERS];
            int next = HF_SCF_ITERATING;
            if (fabs(change) < etol && gnorm < gtol) next = HF_SCF_FINISHING;
            else if (iters >= max_iterations) {
                next = HF_SCF_NOT_CONVERGED;
                sc[S_FINAL] = e;
            }
            st[I_STATE] = next;
            act_diis[c] = next == HF_SCF_ITERATING;
            act_next[c] = next == HF_SCF_ITERATING || next == HF_SCF_FINISHING;
        }
    } else if (threadIdx.x == 0) {
        if (state == HF_SCF_FINISHING) {
            sc[S_FINAL] = sc[S_ENERGY];
            st[I_STATE] = HF_SCF_CONVERGED;
        }
        act_diis[c] = 0;
        act_next[c] = 0;
    }
}

// Cyclic Jacobi eigendecomposition of a symmetric m x m matrix (m <= 9) held by
// one thread: a becomes diagonal (eigenvalues), v holds the eigenvectors as columns.
__device__ void jacobi_eigh(double (&a)[HF_BATCH_MAX_DIIS + 1][HF_BATCH_MAX_DIIS + 1],
                            double (&v)[HF_BATCH_MAX_DIIS + 1][HF_BATCH_MAX_DIIS + 1], int m) {
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) v[i][j] = i == j ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 64; ++sweep) {
        double off = 0.0, diag = 0.0;
        for (int i = 0; i < m; ++i) {
            diag += a[i][i] * a[i][i];
            for (int j = i + 1; j < m; ++j) off += a[i][j] * a[i][j];
        }
        if (off <= 1e-32 * diag || off == 0.0) break;
        for (int p = 0; p < m - 1; ++p)
            for (int q = p + 1; q < m; ++q) {
                const double apq = a[p][q];
                if (apq == 0.0) continue;
                const double theta = (a[q][q] - a[p][p]) / (2.0 * apq);
                const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double cs = 1.0 / sqrt(t * t + 1.0), sn = t * cs;
                for (int k = 0; k < m; ++k) {
                    const double akp = a[k][p], akq = a[k][q];
                    a[k][p] = cs * akp - sn * akq;
                    a[k][q] = sn * akp + cs * akq;
                }
                for (int k = 0; k < m; ++k) {
                    const double apk = a[p][k], aqk = a[q][k];
                    a[p][k] = cs * apk - sn * aqk;
                    a[q][k] = sn * apk + cs * aqk;
                }
                for (int k = 0; k < m; ++k) {
                    const double vkp = v[k][p], vkq = v[k][q];
                    v[k][p] = cs * vkp - sn * vkq;
                    v[k][q] = sn * vkp + cs * vkq;
                }
            }
    }
}

// DIIS (hafnium/scf/diis.py:55-106): push (F, G) into the rings, update the
// overlaps 2 <G_i, G_j>, solve the bordered system of the scaled overlaps by
// eigendecomposition with the null space dropped, and extrapolate Fx. A cluster
// that has just converged takes Fx = F (driver.py:336 finishes from the last F).
__global__ void __launch_bounds__(kThreads) k_diis(const double* __restrict__ F, const double* __restrict__ G,
                                                   double* __restrict__ Fring, double* __restrict__ Gring,
                                                   double* __restrict__ ov, double* __restrict__ Fx, int64_t nn,
                                                   int* __restrict__ ints, const int* __restrict__ act_diis,
                                                   int diis) {
    __shared__ double red[33];
    __shared__ double coef[HF_BATCH_MAX_DIIS];
    const int c = blockIdx.x;
    int* st = ints + c * kInts;
    const int64_t o = (int64_t)c * nn;
    if (st[I_STATE] == HF_SCF_FINISHING) {
        for (int64_t i = threadIdx.x; i < nn; i += blockDim.x) Fx[o + i] = F[o + i];
        return;
    }
    if (act_diis[c] == 0) return;
    const int pushes = st[I_PUSHES];
    const int slot = pushes % diis;
    const int cnt = min(pushes + 1, diis);
    const int64_t ro = (int64_t)c * diis * nn;
    for (int64_t i = threadIdx.x; i < nn; i += blockDim.x) {
        Fring[ro + slot * nn + i] = F[o + i];
        Gring[ro + slot * nn + i] = G[o + i];
    }
    __syncthreads();
    double* O = ov + c * HF_BATCH_MAX_DIIS * HF_BATCH_MAX_DIIS;
    for (int j = 0; j < cnt; ++j) {
        double s = 0.0;
        const double* gj = Gring + ro + j * nn;
        for (int64_t i = threadIdx.x; i < nn; i += blockDim.x) s += G[o + i] * gj[i];
        s = block_sum(s, red);
        if (threadIdx.x == 0) {
            O[slot * HF_BATCH_MAX_DIIS + j] = 2.0 * s;
            O[j * HF_BATCH_MAX_DIIS + slot] = 2.0 * s;
        }
    }
    __syncthreads();
    if (cnt == 1) {
        for (int64_t i = threadIdx.x; i < nn; i += blockDim.x) Fx[o + i] = F[o + i];
        if (threadIdx.x == 0) st[I_PUSHES] = pushes + 1;
        return;
    }
    if (threadIdx.x == 0) {
        double a[HF_BATCH_MAX_DIIS + 1][HF_BATCH_MAX_DIIS + 1], v[HF_BATCH_MAX_DIIS + 1][HF_BATCH_MAX_DIIS + 1];
        double scale = 0.0;
        for (int i = 0; i < cnt; ++i) scale = fmax(scale, O[i * HF_BATCH_MAX_DIIS + i]);
        const double inv = scale > 0.0 ? 1.0 / scale : 1.0;
        for (int i = 0; i <= cnt; ++i)
            for (int j = 0; j <= cnt; ++j) {
                double x;
                if (i < cnt && j < cnt) x = O[i * HF_BATCH_MAX_DIIS + j] * inv;
                else if (i == cnt && j == cnt) x = 0.0;
                else x = -1.0;
                a[i][j] = x;
            }
        jacobi_eigh(a, v, cnt + 1);
        double wmax = 0.0;
        for (int i = 0; i <= cnt; ++i) wmax = fmax(wmax, fabs(a[i][i]));
        // x = V diag(1/w) V^T r with r = (0, ..., 0, -1)
        double sol[HF_BATCH_MAX_DIIS + 1];
        for (int k = 0; k <= cnt; ++k) sol[k] = 0.0;
        for (int i = 0; i <= cnt; ++i) {
            const double w = a[i][i];
            if (!(fabs(w) > kNullSpaceTolerance * wmax)) continue;
            const double proj = -v[cnt][i] / w;
            for (int k = 0; k <= cnt; ++k) sol[k] += v[k][i] * proj;
        }
        for (int k = 0; k < cnt; ++k) coef[k] = sol[k];
        st[I_PUSHES] = pushes + 1;
    }
    __syncthreads();
    for (int64_t i = threadIdx.x; i < nn; i += blockDim.x) {
        double s = 0.0;
        for (int j = 0; j < cnt; ++j) s += coef[j] * Fring[ro + j * nn + i];
        Fx[o + i] = s;
    }
}

// Start of canonical purification (Palser and Manolopoulos 1998, eq. 13-15):
// P0 = (lambda / m)(mu I - F') + (n_occ / m) I, mu = tr F' / m,
// lambda = min(n_occ / (f_max - mu), (m - n_occ) / (mu - f_min)) with the
// spectral bounds f_min, f_max from Gershgorin discs. In place on P.
__global__ void __launch_bounds__(kThreads) k_pm_init(double* __restrict__ P, int64_t m, double nocc,
                                                      const int* __restrict__ act_next, int* __restrict__ act_pm,
                                                      int* __restrict__ ints) {
    __shared__ double red[33];
    const int c = blockIdx.x;
    if (act_next[c] == 0) {
        if (threadIdx.x == 0) act_pm[c] = 0;
        return;
    }
    double* A = P + (int64_t)c * m * m;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double lo = INFINITY, hi = -INFINITY, tr = 0.0;
    for (int64_t i = warp; i < m; i += nw) {
        double r = 0.0;
        for (int64_t j = lane; j < m; j += 32) r += fabs(A[i * m + j]);
        for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
        const double d = A[i * m + i];
        r -= fabs(d);
        lo = fmin(lo, d - r);
        hi = fmax(hi, d + r);
        if (lane == 0) tr += d;
    }
    lo = block_min(lo, red);
    hi = block_max(hi, red);
    tr = block_sum(tr, red);
    const double mu = tr / (double)m;
    const double lambda = fmin(nocc / (hi - mu), ((double)m - nocc) / (mu - lo));
    const double a = lambda / (double)m, b = nocc / (double)m;
    for (int64_t e = threadIdx.x; e < m * m; e += blockDim.x) {
        const int64_t i = e / m, j = e % m;
        A[e] = -a * A[e] + (i == j ? a * mu + b : 0.0);
    }
    if (threadIdx.x == 0) {
        act_pm[c] = 1;
        ints[c * kInts + I_CROSSED] = 0;
        ints[c * kInts + I_PMSTEPS] = 0;
    }
}

// One purification step's coefficients from P and P2 = P P:
// t1 = tr(P - P^2), t2 = tr(P^2 - P^3), c = t2 / t1; then
//   c >= 1/2: P' = ((1 + c) P^2 - P^3) / c           = P^2 Y,          Y = ((1 + c) I - P) / c
//   c <  1/2: P' = ((1 - 2c) P + (1 + c) P^2 - P^3) / (1 - c)
//                                                    = P^2 Y + beta P, Y = ((1 + c) I - P) / (1 - c)
// The step after t1 first falls below tol is the last one.
__global__ void __launch_bounds__(kThreads) k_pm_step(const double* __restrict__ P, const double* __restrict__ P2,
                                                      double* __restrict__ Y, int64_t m, double* __restrict__ beta,
                                                      int* __restrict__ ints, int* __restrict__ act_pm, double tol) {
    __shared__ double red[33];
    __shared__ double s_c, s_den;
    __shared__ int s_go;
    const int c = blockIdx.x;
    if (act_pm[c] == 0) return;
    const int64_t o = (int64_t)c * m * m;
    double d1 = 0.0, d2 = 0.0, x3 = 0.0;
    for (int64_t e = threadIdx.x; e < m * m; e += blockDim.x) {
        const int64_t i = e / m, j = e % m;
        const double p2 = P2[o + e];
        x3 += p2 * P[o + e];
        if (i == j) {
            d1 += P[o + e] - p2;
            d2 += p2;
        }
    }
    const double t1 = block_sum(d1, red);
    const double tr2 = block_sum(d2, red);
    const double tr3 = block_sum(x3, red);
    if (threadIdx.x == 0) {
        int* st = ints + c * kInts;
        const double t2 = tr2 - tr3;
        int go = 1;
        if (st[I_CROSSED]) go = 0;
        else if (!(t1 < tol)) {
            // still iterating
        } else {
            st[I_CROSSED] = 1;
        }
        double cc = 0.5;  // the McWeeny step when t1 is within rounding of zero
        if (go) {
            if (t1 > 0.0) cc = fmin(1.0, fmax(0.0, t2 / t1));
            else if (!(fabs(t1) < tol)) {
                go = 0;  // eigenvalues left [0, 1]: no convergent purification
                st[I_STATE] = HF_SCF_PURIFICATION_FAILED;
            }
        }
        if (go) {
            st[I_PMSTEPS] += 1;
            if (cc >= 0.5) {
                s_den = cc;
                beta[c] = 0.0;
            } else {
                s_den = 1.0 - cc;
                beta[c] = (1.0 - 2.0 * cc) / (1.0 - cc);
            }
            s_c = cc;
        } else {
            act_pm[c] = 0;
        }
        s_go = go;
    }
    __syncthreads();
    if (!s_go) return;
    const double inv = 1.0 / s_den, diag = (1.0 + s_c) * inv;
    for (int64_t e = threadIdx.x; e < m * m; e += blockDim.x) {
        const int64_t i = e / m, j = e % m;
        Y[o + e] = (i == j ? diag : 0.0) - inv * P[o + e];
    }
}

// Clusters whose purification has not ended after the captured steps fail.
__global__ void k_pm_check(int count, const int* __restrict__ act_pm, int* __restrict__ ints,
                           int* __restrict__ act_next) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= count) return;
    int* st = ints + c * kInts;
    if (act_pm[c] || st[I_STATE] == HF_SCF_PURIFICATION_FAILED) {
        if (act_next[c]) st[I_STATE] = HF_SCF_PURIFICATION_FAILED;
        act_next[c] = 0;
    }
}

// After a Fock build: the masks of the next iteration and whether any cluster
// still iterates or finishes; the iteration guard ends the loop regardless
// after max_bodies passes.
__global__ void k_continue(int count, const int* __restrict__ ints, int* __restrict__ act_grad,
                           int* __restrict__ glob, int* __restrict__ group_any) {
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    for (int c = threadIdx.x; c < count; c += blockDim.x) {
        const int s = ints[c * kInts + I_STATE];
        act_grad[c] = s == HF_SCF_ITERATING;
        if (s == HF_SCF_ITERATING || s == HF_SCF_FINISHING) atomicOr(&any, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        glob[1] = any;
        if (any) atomicOr(group_any, 1);
    }
}

__global__ void k_group_reset(int* __restrict__ group_any) { *group_any = 0; }

// Sets the WHILE node's condition: continue while any cluster of any batch is
// active and fewer than max_bodies iterations have run.
__global__ void k_group_condition(cudaGraphConditionalHandle handle, const int* __restrict__ group_any,
                                  int* __restrict__ counter, int max_bodies) {
    const int n = ++counter[0];
    const unsigned go = (*group_any != 0 && n < max_bodies) ? 1u : 0u;
    cudaGraphSetConditional(handle, go);
}

// Clusters still iterating when the loop guard ended the graph.
__global__ void k_mark_unfinished(int count, int* __restrict__ ints, double* __restrict__ scal) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= count) return;
    int* st = ints + c * kInts;
    if (st[I_STATE] == HF_SCF_ITERATING || st[I_STATE] == HF_SCF_FINISHING) {
        st[I_STATE] = HF_SCF_NOT_CONVERGED;
        scal[c * kScal + S_FINAL] = scal[c * kScal + S_ENERGY];
    }
}

// |X|_F^2 per cluster into out[c] (one CTA each).
__global__ void __launch_bounds__(kThreads) k_frobenius2(const double* __restrict__ X, int64_t nn,
                                                         double* __restrict__ out) {
    __shared__ double red[33];
    const int c = blockIdx.x;
    double s = 0.0;
    for (int64_t i = threadIdx.x; i < nn; i += blockDim.x) s += X[(int64_t)c * nn + i] * X[(int64_t)c * nn + i];
    s = block_sum(s, red);
    if (threadIdx.x == 0) out[c] = s;
}

int64_t round_up(int64_t v, int64_t m) { return (v + m - 1) / m * m; }

}  // namespace

struct hf_batch {
    int device = 0;
    cudaStream_t own = nullptr;
    cudaStream_t stream = nullptr;
    std::string err;
    int count = 0;
    int64_t n = 0, nn = 0, nocc = 0, npad = 0, naux = 0;
    int nt = 0;
    int64_t ntiles = 0;
    std::vector<hf_ctx*> ctxs;
    const double** d_btab = nullptr;
    JkPlan plan{};
    // per-cluster matrices
    double *S = nullptr, *H = nullptr, *X = nullptr, *XT = nullptr, *D = nullptr, *J = nullptr, *K = nullptr,
           *F = nullptr, *G = nullptr, *Fx = nullptr, *T1 = nullptr, *T2 = nullptr, *P = nullptr, *P2 = nullptr,
           *Y = nullptr, *Lc = nullptr, *Fring = nullptr, *Gring = nullptr;
    // J/K scratch
    double *Ct = nullptr, *Kp = nullptr, *Xch = nullptr, *jwork = nullptr, *partial = nullptr;
    int opad_max = 0, qchunk = 0;
    // bookkeeping
    double *ov = nullptr, *scal = nullptr, *pm_beta = nullptr;
    int *ints = nullptr, *info = nullptr, *act_grad = nullptr, *act_diis = nullptr, *act_next = nullptr,
        *act_pm = nullptr, *act_all = nullptr, *glob = nullptr;
    std::vector<void*> allocations;
    bool loaded = false;
    int64_t guess_rank = 0;
    int diis_alloc = HF_BATCH_MAX_DIIS;
};

namespace {

int fail(hf_batch* b, int code, const std::string& msg) {
    if (b) b->err = msg;
    return code;
}

#define HB_CU(call)                                                                          \
    do {                                                                                     \
        cudaError_t _e = (call);                                                             \
        if (_e != cudaSuccess)                                                               \
            return fail(b, _e == cudaErrorMemoryAllocation ? HF_ERR_OOM : HF_ERR_CUDA,       \
                        std::string(#call) + ": " + cudaGetErrorString(_e));                 \
    } while (0)

int balloc(hf_batch* b, void** p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes ? bytes : 8);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(b, HF_ERR_OOM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed");
    }
    b->allocations.push_back(*p);
    return HF_OK;
}

template <typename T>
int take(hf_batch* b, T** p, size_t elems) {
    return balloc(b, (void**)p, sizeof(T) * elems);
}

GemmArgs square(const hf_batch* b, const double* A, const double* Bm, double* C, const int* active, int tile) {
    GemmArgs g{};
    g.M = g.N = g.K = (int)b->n;
    g.A = A;
    g.lda = b->n;
    g.B = Bm;
    g.ldb = b->n;
    g.C = C;
    g.ldc = b->n;
    g.alpha = 1.0;
    g.beta = 0.0;
    g.strideA = g.strideB = g.strideC = b->nn;
    g.active = active;
    g.tile = tile;
    return g;
}

cudaError_t gemm(const hf_batch* b, const GemmArgs& g, cudaStream_t s) { return dgemm_nt(g, b->count, s); }

// The Fock build of the clusters in `active`: K from a rank-<= maxr pivoted
// Cholesky factor of D, J from 2 D, then F and the energy.
cudaError_t fock_build(hf_batch* b, cudaStream_t s, const int* active, int maxr) {
    const int opad = (int)std::max<int64_t>(64, round_up(maxr, 64));
    cudaError_t e = pivoted_cholesky(b->D, b->nn, (int)b->n, kRankTolerance, maxr, b->Lc, b->nn, b->info, b->count,
                                     active, s);
    if (e != cudaSuccess) return e;
    e = factor_pad(b->Lc, b->nn, b->n, b->info, b->Ct, (int64_t)opad * b->npad, b->npad, opad, nullptr, b->count,
                   active, s);
    if (e != cudaSuccess) return e;
    JkPlan p = b->plan;
    p.active = active;
    const int qchunk = (int)std::max<int64_t>(1, (int64_t)b->qchunk * b->opad_max / opad);
    e = exchange_build_fp64(p, b->Ct, (int64_t)opad * b->npad, opad, nullptr, b->K, b->nn, b->Kp, b->Xch, nullptr,
                            b->partial,
                            std::min<int>(qchunk, (int)b->naux), s);
    if (e != cudaSuccess) return e;
    e = coulomb_build(p, b->D, b->nn, 2.0, b->J, b->nn, b->jwork, s);
    if (e != cudaSuccess) return e;
    k_fock_energy<<<b->count, kThreads, 0, s>>>(b->H, b->J, b->K, b->D, b->F, b->nn, b->scal, active);
    return cudaGetLastError();
}

cudaError_t prologue(hf_batch* b, cudaStream_t s) {
    return fock_build(b, s, b->act_all, (int)b->guess_rank);
}

// One SCF iteration (see the file comment).
cudaError_t body(hf_batch* b, cudaStream_t s, const hf_batch_options& o, int* group_any) {
    const unsigned cnt = (unsigned)b->count;
    const unsigned eb = (unsigned)((b->nn + 255) / 256);
    const int tile = o.gemm_tile;
    cudaError_t e;
    // G = X^T (F D S - S D F) X
    if ((e = gemm(b, square(b, b->F, b->D, b->T1, b->act_grad, tile), s)) != cudaSuccess) return e;
    if ((e = gemm(b, square(b, b->T1, b->S, b->T2, b->act_grad, tile), s)) != cudaSuccess) return e;
    k_antisymmetric<<<dim3(eb, cnt), 256, 0, s>>>(b->T2, b->T1, b->n, b->act_grad);
    GemmArgs gx = square(b, b->T1, b->XT, b->T2, b->act_grad, tile);
    gx.epi = 1;  // T2 = (T1 X)^T
    if ((e = gemm(b, gx, s)) != cudaSuccess) return e;
    if ((e = gemm(b, square(b, b->XT, b->T2, b->G, b->act_grad, tile), s)) != cudaSuccess) return e;
    k_status<<<cnt, kThreads, 0, s>>>(b->G, b->nn, b->scal, b->ints, b->act_diis, b->act_next, o.energy_tolerance,
                                      o.gradient_tolerance, o.max_iterations);
    k_diis<<<cnt, kThreads, 0, s>>>(b->F, b->G, b->Fring, b->Gring, b->ov, b->Fx, b->nn, b->ints, b->act_diis,
                                    o.diis_size);
    // F' = X^T Fx X into P, then purification
    GemmArgs fx = square(b, b->Fx, b->XT, b->T2, b->act_next, tile);
    fx.epi = 1;
    if ((e = gemm(b, fx, s)) != cudaSuccess) return e;
    if ((e = gemm(b, square(b, b->XT, b->T2, b->P, b->act_next, tile), s)) != cudaSuccess) return e;
    k_pm_init<<<cnt, kThreads, 0, s>>>(b->P, b->n, (double)b->nocc, b->act_next, b->act_pm, b->ints);
    for (int step = 0; step < o.purify_steps; ++step) {
        if ((e = gemm(b, square(b, b->P, b->P, b->P2, b->act_pm, tile), s)) != cudaSuccess) return e;
        k_pm_step<<<cnt, kThreads, 0, s>>>(b->P, b->P2, b->Y, b->n, b->pm_beta, b->ints, b->act_pm,
                                           o.purify_tolerance);
        GemmArgs up = square(b, b->P2, b->Y, b->P, b->act_pm, tile);
        up.beta_v = b->pm_beta;
        if ((e = gemm(b, up, s)) != cudaSuccess) return e;
    }
    k_pm_check<<<(cnt + 127) / 128, 128, 0, s>>>(b->count, b->act_pm, b->ints, b->act_next);
    // D = X P X^T
    if ((e = gemm(b, square(b, b->X, b->P, b->T1, b->act_next, tile), s)) != cudaSuccess) return e;
    if ((e = gemm(b, square(b, b->T1, b->X, b->T2, b->act_next, tile), s)) != cudaSuccess) return e;
    k_symmetric<<<dim3(eb, cnt), 256, 0, s>>>(b->T2, b->D, b->n, b->act_next);
    if ((e = fock_build(b, s, b->act_next, (int)b->nocc)) != cudaSuccess) return e;
    k_continue<<<1, 256, 0, s>>>(b->count, b->ints, b->act_grad, b->glob, group_any);
    return cudaGetLastError();
}

}  // namespace

extern "C" {

int hf_batch_default_options(hf_batch_options* out) {
    if (!out) return HF_ERR_ARG;
    out->max_iterations = 100;
    out->diis_size = 8;
    out->energy_tolerance = 1e-10;
    out->gradient_tolerance = 1e-6;
    out->purify_steps = 64;
    out->purify_tolerance = 1e-9;
    out->gemm_tile = 0;
    out->use_graph = 1;
    return HF_OK;
}

int hf_batch_create(hf_ctx* const* clusters, int count, int64_t n_occ, hf_batch** out) {
    if (!clusters || !out || count < 1 || count > HF_BATCH_MAX_CLUSTERS || n_occ < 1) return HF_ERR_ARG;
    *out = nullptr;
    hf_batch* b = new hf_batch();
    b->count = count;
    b->nocc = n_occ;
    TensorView v0{};
    for (int c = 0; c < count; ++c) {
        TensorView v{};
        if (context_view(clusters[c], &v) != HF_OK || !v.built) {
            delete b;
            return HF_ERR_STATE;
        }
        if (c == 0) v0 = v;
        else if (v.device != v0.device || v.n != v0.n || v.naux != v0.naux) {
            delete b;
            return HF_ERR_ARG;
        }
        b->ctxs.push_back(clusters[c]);
    }
    if (n_occ > v0.n || v0.n > 4096 || (int64_t)((v0.nt * 64 + 127) / 128) * count > 65535) {
        delete b;
        return HF_ERR_ARG;
    }
    b->device = v0.device;
    b->n = v0.n;
    b->nn = v0.n * v0.n;
    b->nt = v0.nt;
    b->ntiles = v0.ntiles;
    b->naux = v0.naux;
    b->npad = (int64_t)v0.nt * 64;
    cudaSetDevice(b->device);
    int s = HF_OK;
#define HB_TAKE(ptr, elems)                                   \
    if ((s = take(b, &(ptr), (size_t)(elems))) != HF_OK) {    \
        hf_batch_destroy(b);                                  \
        return s;                                             \
    }
    const size_t nn = (size_t)b->nn * count;
    HB_TAKE(b->S, nn);
    HB_TAKE(b->H, nn);
    HB_TAKE(b->X, nn);
    HB_TAKE(b->XT, nn);
    HB_TAKE(b->D, nn);
    HB_TAKE(b->J, nn);
    HB_TAKE(b->K, nn);
    HB_TAKE(b->F, nn);
    HB_TAKE(b->G, nn);
    HB_TAKE(b->Fx, nn);
    HB_TAKE(b->T1, nn);
    HB_TAKE(b->T2, nn);
    HB_TAKE(b->P, nn);
    HB_TAKE(b->P2, nn);
    HB_TAKE(b->Y, nn);
    HB_TAKE(b->Lc, nn);
    HB_TAKE(b->Fring, nn * HF_BATCH_MAX_DIIS);
    HB_TAKE(b->Gring, nn * HF_BATCH_MAX_DIIS);
    // K scratch sized for factors up to n columns; X chunks within ~2 GB
    b->opad_max = (int)std::max<int64_t>(64, round_up(b->n, 64));
    HB_TAKE(b->Ct, (size_t)count * b->opad_max * b->npad);
    HB_TAKE(b->Kp, (size_t)count * b->npad * b->npad);
    if (syrk_partial_doubles(b->npad, count) > 0) HB_TAKE(b->partial, (size_t)syrk_partial_doubles(b->npad, count));
    const size_t per_q = sizeof(double) * (size_t)count * b->npad * b->opad_max;
    b->qchunk = (int)std::max<size_t>(1, std::min<size_t>(((size_t)2 << 30) / per_q, (size_t)b->naux));
    b->qchunk = std::min(b->qchunk, 65535);
    HB_TAKE(b->Xch, (size_t)count * b->npad * b->qchunk * b->opad_max);
    JkPlan p{};
    p.B = nullptr;
    p.ldb = b->ntiles * 4096;
    p.n = b->n;
    p.nt = b->nt;
    p.ntiles = b->ntiles;
    p.naux = (int)b->naux;
    p.count = count;
    HB_TAKE(b->jwork, (size_t)count * coulomb_work_doubles(p));
    HB_TAKE(b->ov, (size_t)count * HF_BATCH_MAX_DIIS * HF_BATCH_MAX_DIIS);
    HB_TAKE(b->scal, (size_t)count * kScal);
    HB_TAKE(b->pm_beta, (size_t)count);
    HB_TAKE(b->ints, (size_t)count * kInts);
    HB_TAKE(b->info, (size_t)count * 2);
    HB_TAKE(b->act_grad, (size_t)count);
    HB_TAKE(b->act_diis, (size_t)count);
    HB_TAKE(b->act_next, (size_t)count);
    HB_TAKE(b->act_pm, (size_t)count);
    HB_TAKE(b->act_all, (size_t)count);
    HB_TAKE(b->glob, 8);
    HB_TAKE(b->d_btab, (size_t)count);
#undef HB_TAKE
    std::vector<const double*> tab(count);
    for (int c = 0; c < count; ++c) {
        TensorView v{};
        context_view(clusters[c], &v);
        tab[c] = v.B;
    }
    std::vector<int> ones(count, 1);
    // synchronous copies from pageable memory may return before their DMA lands; the
    // device synchronisation orders them before any kernel on the batch's stream
    if (cudaMemcpy(b->d_btab, tab.data(), sizeof(double*) * count, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->act_all, ones.data(), sizeof(int) * count, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaDeviceSynchronize() != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking) != cudaSuccess) {
        hf_batch_destroy(b);
        return HF_ERR_CUDA;
    }
    p.Btab = b->d_btab;
    b->plan = p;
    b->stream = b->own;
    if (jk_configure() != cudaSuccess) {
        hf_batch_destroy(b);
        return HF_ERR_CUDA;
    }
    *out = b;
    return HF_OK;
}

int hf_batch_destroy(hf_batch* b) {
    if (!b) return HF_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (void* p : b->allocations) cudaFree(p);
    if (b->own) cudaStreamDestroy(b->own);
    delete b;
    return HF_OK;
}

const char* hf_batch_last_error(const hf_batch* b) { return b ? b->err.c_str() : "null batch"; }

int hf_batch_set_stream(hf_batch* b, void* stream) {
    if (!b) return HF_ERR_ARG;
    b->stream = stream ? (cudaStream_t)stream : b->own;
    return HF_OK;
}

int hf_batch_dims(const hf_batch* b, int* count, int64_t* n_ao, int64_t* n_aux, int64_t* n_occ) {
    if (!b) return HF_ERR_ARG;
    if (count) *count = b->count;
    if (n_ao) *n_ao = b->n;
    if (n_aux) *n_aux = b->naux;
    if (n_occ) *n_occ = b->nocc;
    return HF_OK;
}

int hf_batch_load(hf_batch* b, const double* overlap, const double* core, const double* guess,
                  const double* nuclear_repulsion, int64_t guess_rank) {
    if (!b || !overlap || !core || !guess || !nuclear_repulsion || guess_rank < 1) return HF_ERR_ARG;
    cudaSetDevice(b->device);
    cudaStream_t s = b->stream;
    const size_t bytes = sizeof(double) * (size_t)b->nn * b->count;
    b->guess_rank = std::min<int64_t>(guess_rank, b->n);
    HB_CU(cudaMemcpyAsync(b->S, overlap, bytes, cudaMemcpyDeviceToDevice, s));
    HB_CU(cudaMemcpyAsync(b->H, core, bytes, cudaMemcpyDeviceToDevice, s));
    HB_CU(cudaMemcpyAsync(b->D, guess, bytes, cudaMemcpyDeviceToDevice, s));
    // X = L^-T per cluster (S = L L^T); T1 holds the factor
    HB_CU(cudaMemcpyAsync(b->T1, overlap, bytes, cudaMemcpyDeviceToDevice, s));
    int* d_info = b->info;
    double* d_piv = b->pm_beta;
    std::vector<double> big(b->count, 1e300);
    HB_CU(cudaMemcpyAsync(d_piv, big.data(), sizeof(double) * b->count, cudaMemcpyHostToDevice, s));
    HB_CU(cudaMemsetAsync(d_info, 0, sizeof(int) * 2 * b->count, s));
    for (int c = 0; c < b->count; ++c) {
        double* L = b->T1 + (int64_t)c * b->nn;
        HB_CU(cholesky_lower(L, (int)b->n, b->n, d_info + c, d_piv + c, s));
        // XT = L^-1 (row-major lower), X = its transpose; the K chunk buffer (>= n x 64) as work
        HB_CU(triangular_inverse(L, (int)b->n, b->n, b->XT + (int64_t)c * b->nn, b->X + (int64_t)c * b->nn, b->Xch,
                                 s));
    }
    k_frobenius2<<<b->count, kThreads, 0, s>>>(b->X, b->nn, b->T2);
    HB_CU(cudaGetLastError());
    std::vector<int> info(b->count);
    std::vector<double> fro(b->count);
    HB_CU(cudaMemcpyAsync(info.data(), d_info, sizeof(int) * b->count, cudaMemcpyDeviceToHost, s));
    HB_CU(cudaMemcpyAsync(fro.data(), b->T2, sizeof(double) * b->count, cudaMemcpyDeviceToHost, s));
    HB_CU(cudaStreamSynchronize(s));
    for (int c = 0; c < b->count; ++c) {
        if (info[c] != 0)
            return fail(b, HF_ERR_NUMERIC, "overlap of cluster " + std::to_string(c) + " is not positive definite");
        // lambda_min(S) = 1 / |L^-1|_2^2 >= 1 / |L^-1|_F^2
        if (!(1.0 / fro[c] > kOverlapThreshold))
            return fail(b, HF_ERR_NUMERIC, "overlap of cluster " + std::to_string(c) +
                                               " may have an eigenvalue below the 1e-10 drop threshold");
    }
    // bookkeeping
    std::vector<double> scal((size_t)b->count * kScal, 0.0);
    for (int c = 0; c < b->count; ++c) scal[(size_t)c * kScal + S_ENUC] = nuclear_repulsion[c];
    HB_CU(cudaMemcpyAsync(b->scal, scal.data(), sizeof(double) * scal.size(), cudaMemcpyHostToDevice, s));
    HB_CU(cudaMemsetAsync(b->ints, 0, sizeof(int) * kInts * b->count, s));
    HB_CU(cudaMemsetAsync(b->ov, 0, sizeof(double) * HF_BATCH_MAX_DIIS * HF_BATCH_MAX_DIIS * b->count, s));
    HB_CU(cudaMemsetAsync(b->glob, 0, sizeof(int) * 8, s));
    HB_CU(cudaStreamSynchronize(s));
    b->loaded = true;
    return HF_OK;
}

}  // extern "C"

namespace {

int check_options(hf_batch* b, const hf_batch_options& o) {
    if (o.max_iterations < 1 || o.diis_size < 1 || o.diis_size > HF_BATCH_MAX_DIIS || !(o.energy_tolerance > 0.0) ||
        !(o.gradient_tolerance > 0.0) || o.purify_steps < 1 || o.purify_steps > 128 || !(o.purify_tolerance > 0.0) ||
        o.gemm_tile < 0 || o.gemm_tile >= kTileCount)
        return fail(b, HF_ERR_ARG, "invalid batch options");
    return HF_OK;
}

// Resets the per-run state (a load leaves it reset; a second run starts again
// from the loaded guess only after another load).
int run_group(hf_batch* const* batches, int nb, const hf_batch_options& o) {
    hf_batch* b = batches[0];
    cudaStream_t s = b->stream;
    const int max_bodies = o.max_iterations + 2;
    for (int i = 0; i < nb; ++i) {
        if (!batches[i]->loaded) return fail(batches[i], HF_ERR_STATE, "load the batch first");
        if (batches[i]->device != b->device) return fail(b, HF_ERR_ARG, "batches on different devices");
        int st = check_options(batches[i], o);
        if (st != HF_OK) return st;
    }
    cudaSetDevice(b->device);
    int* group = b->glob + 4;  // [0] any, [1] counter
    HB_CU(cudaMemsetAsync(group, 0, 2 * sizeof(int), s));
    for (int i = 1; i < nb; ++i) {
        cudaEvent_t ev;
        HB_CU(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        HB_CU(cudaEventRecord(ev, batches[i]->stream));
        HB_CU(cudaStreamWaitEvent(s, ev, 0));
        cudaEventDestroy(ev);
    }
    if (!o.use_graph) {
        for (int i = 0; i < nb; ++i) HB_CU(prologue(batches[i], s));
        for (int i = 0; i < nb; ++i)
            k_continue<<<1, 256, 0, s>>>(batches[i]->count, batches[i]->ints, batches[i]->act_grad, batches[i]->glob,
                                         group);
        HB_CU(cudaGetLastError());
        for (int it = 0; it < max_bodies; ++it) {
            int any = 0;
            HB_CU(cudaMemcpyAsync(&any, group, sizeof(int), cudaMemcpyDeviceToHost, s));
            HB_CU(cudaStreamSynchronize(s));
            if (!any) break;
            k_group_reset<<<1, 1, 0, s>>>(group);
            for (int i = 0; i < nb; ++i) HB_CU(body(batches[i], s, o, group));
        }
    } else {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        // one side stream per batch for the prologue and another for the loop
        // body (a stream forked into the outer capture stays in it until it ends)
        std::vector<cudaStream_t> side(2 * nb, nullptr);
        for (int i = 0; i < 2 * nb; ++i) HB_CU(cudaStreamCreateWithFlags(&side[i], cudaStreamNonBlocking));
        std::vector<cudaEvent_t> evs;
        auto cleanup = [&]() {
            for (cudaEvent_t ev : evs) cudaEventDestroy(ev);
            evs.clear();
            if (exec) cudaGraphExecDestroy(exec);
            if (graph) cudaGraphDestroy(graph);
            for (cudaStream_t x : side)
                if (x) cudaStreamDestroy(x);
        };
        auto check = [&](cudaError_t e, const char* what) -> int {
            if (e == cudaSuccess) return HF_OK;
            cudaStreamCaptureStatus cs;
            if (cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
                cudaGraph_t g2 = nullptr;
                cudaStreamEndCapture(s, &g2);
                if (g2) cudaGraphDestroy(g2);
            }
            cudaGetLastError();
            cleanup();
            return fail(b, HF_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
        };
        int st;
        if ((st = check(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture")) != HF_OK)
            return st;
        // prologue: every batch's first Fock build from its guess, forked per batch
        auto fork_join = [&](auto&& work, cudaStream_t root, int first) -> cudaError_t {
            cudaEvent_t fork;
            cudaError_t e = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
            if (e != cudaSuccess) return e;
            evs.push_back(fork);
            if ((e = cudaEventRecord(fork, root)) != cudaSuccess) return e;
            for (int i = 0; i < nb; ++i) {
                cudaStream_t x = side[first + i];
                if ((e = cudaStreamWaitEvent(x, fork, 0)) != cudaSuccess) return e;
                if ((e = work(i, x)) != cudaSuccess) return e;
                cudaEvent_t join;
                if ((e = cudaEventCreateWithFlags(&join, cudaEventDisableTiming)) != cudaSuccess) return e;
                evs.push_back(join);
                if ((e = cudaEventRecord(join, x)) != cudaSuccess) return e;
                if ((e = cudaStreamWaitEvent(root, join, 0)) != cudaSuccess) return e;
            }
            return cudaSuccess;
        };
        cudaError_t e = fork_join(
            [&](int i, cudaStream_t x) -> cudaError_t {
                cudaError_t r = prologue(batches[i], x);
                if (r != cudaSuccess) return r;
                k_continue<<<1, 256, 0, x>>>(batches[i]->count, batches[i]->ints, batches[i]->act_grad,
                                             batches[i]->glob, group);
                return cudaGetLastError();
            },
            s, 0);
        if ((st = check(e, "prologue capture")) != HF_OK) return st;
        cudaStreamCaptureStatus cs;
        cudaGraph_t cap = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t ndeps = 0;
        if ((st = check(cudaStreamGetCaptureInfo(s, &cs, nullptr, &cap, &deps, &ndeps), "capture info")) != HF_OK)
            return st;
        cudaGraphConditionalHandle handle;
        if ((st = check(cudaGraphConditionalHandleCreate(&handle, cap, 1, cudaGraphCondAssignDefault),
                        "conditional handle")) != HF_OK)
            return st;
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = handle;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t loop;
        if ((st = check(cudaGraphAddNode(&loop, cap, deps, ndeps, &cp), "conditional node")) != HF_OK) return st;
        cudaGraph_t body_graph = cp.conditional.phGraph_out[0];
        if ((st = check(cudaStreamUpdateCaptureDependencies(s, &loop, 1, cudaStreamSetCaptureDependencies),
                        "capture dependencies")) != HF_OK)
            return st;
        // the loop body, captured from a second stream into the node's graph
        cudaStream_t bs = nullptr;
        if ((st = check(cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking), "body stream")) != HF_OK) return st;
        side.push_back(bs);
        if ((st = check(cudaStreamBeginCaptureToGraph(bs, body_graph, nullptr, nullptr, 0,
                                                      cudaStreamCaptureModeThreadLocal),
                        "body capture")) != HF_OK)
            return st;
        k_group_reset<<<1, 1, 0, bs>>>(group);
        e = fork_join([&](int i, cudaStream_t x) -> cudaError_t { return body(batches[i], x, o, group); }, bs, nb);
        if (e == cudaSuccess) {
            k_group_condition<<<1, 1, 0, bs>>>(handle, group, group + 1, max_bodies);
            e = cudaGetLastError();
        }
        cudaGraph_t body_out = nullptr;
        const cudaError_t e2 = cudaStreamEndCapture(bs, &body_out);
        if ((st = check(e != cudaSuccess ? e : e2, "body capture")) != HF_OK) return st;
        if ((st = check(cudaStreamEndCapture(s, &graph), "end capture")) != HF_OK) return st;
        if ((st = check(cudaGraphInstantiate(&exec, graph, 0), "instantiate")) != HF_OK) return st;
        if ((st = check(cudaGraphLaunch(exec, s), "graph launch")) != HF_OK) return st;
        if ((st = check(cudaStreamSynchronize(s), "graph run")) != HF_OK) return st;
        cleanup();
    }
    for (int i = 0; i < nb; ++i)
        k_mark_unfinished<<<(batches[i]->count + 127) / 128, 128, 0, s>>>(batches[i]->count, batches[i]->ints,
                                                                          batches[i]->scal);
    HB_CU(cudaGetLastError());
    HB_CU(cudaStreamSynchronize(s));
    for (int i = 0; i < nb; ++i) batches[i]->loaded = false;
    return HF_OK;
}

}  // namespace

extern "C" {

int hf_batch_run(hf_batch* b, const hf_batch_options* options) {
    if (!b) return HF_ERR_ARG;
    hf_batch_options o;
    hf_batch_default_options(&o);
    if (options) o = *options;
    hf_batch* one[1] = {b};
    return run_group(one, 1, o);
}

int hf_batch_run_group(hf_batch* const* batches, int count, const hf_batch_options* options) {
    if (!batches || count < 1) return HF_ERR_ARG;
    for (int i = 0; i < count; ++i)
        if (!batches[i]) return HF_ERR_ARG;
    hf_batch_options o;
    hf_batch_default_options(&o);
    if (options) o = *options;
    return run_group(batches, count, o);
}

int hf_batch_results(hf_batch* b, double* energies, int* iterations, int* states, double* densities) {
    if (!b) return HF_ERR_ARG;
    cudaSetDevice(b->device);
    std::vector<double> scal((size_t)b->count * kScal);
    std::vector<int> ints((size_t)b->count * kInts);
    HB_CU(cudaMemcpyAsync(scal.data(), b->scal, sizeof(double) * scal.size(), cudaMemcpyDeviceToHost, b->stream));
    HB_CU(cudaMemcpyAsync(ints.data(), b->ints, sizeof(int) * ints.size(), cudaMemcpyDeviceToHost, b->stream));
    if (densities)
        HB_CU(cudaMemcpyAsync(densities, b->D, sizeof(double) * b->nn * b->count, cudaMemcpyDeviceToDevice,
                              b->stream));
    HB_CU(cudaStreamSynchronize(b->stream));
    for (int c = 0; c < b->count; ++c) {
        if (energies) energies[c] = scal[(size_t)c * kScal + S_FINAL];
        if (iterations) iterations[c] = ints[(size_t)c * kInts + I_ITERS];
        if (states) states[c] = ints[(size_t)c * kInts + I_STATE];
    }
    return HF_OK;
}

int hf_batch_coulomb(hf_batch* b, const double* density, double scale, double* coulomb) {
    if (!b || !density || !coulomb) return HF_ERR_ARG;
    cudaSetDevice(b->device);
    JkPlan p = b->plan;
    p.active = b->act_all;
    HB_CU(coulomb_build(p, density, b->nn, scale, coulomb, b->nn, b->jwork, b->stream));
    HB_CU(cudaStreamSynchronize(b->stream));
    return HF_OK;
}

int hf_batch_exchange(hf_batch* b, const double* density, int64_t max_rank, double* exchange) {
    if (!b || !density || !exchange || max_rank < 1) return HF_ERR_ARG;
    cudaSetDevice(b->device);
    const int maxr = (int)std::min<int64_t>(max_rank, b->n);
    const int opad = (int)std::max<int64_t>(64, round_up(maxr, 64));
    // one pivot beyond max_rank tells a density of higher rank from one of exactly max_rank
    const int probe = (int)std::min<int64_t>(maxr + 1, b->n);
    HB_CU(pivoted_cholesky(density, b->nn, (int)b->n, kRankTolerance, probe, b->Lc, b->nn, b->info, b->count,
                           b->act_all, b->stream));
    HB_CU(factor_pad(b->Lc, b->nn, b->n, b->info, b->Ct, (int64_t)opad * b->npad, b->npad, opad, nullptr, b->count,
                     b->act_all, b->stream));
    JkPlan p = b->plan;
    p.active = b->act_all;
    const int qchunk = (int)std::max<int64_t>(1, (int64_t)b->qchunk * b->opad_max / opad);
    HB_CU(exchange_build_fp64(p, b->Ct, (int64_t)opad * b->npad, opad, nullptr, exchange, b->nn, b->Kp, b->Xch,
                              nullptr, b->partial, std::min<int>(qchunk, (int)b->naux), b->stream));
    std::vector<int> info(2 * b->count);
    HB_CU(cudaMemcpyAsync(info.data(), b->info, sizeof(int) * info.size(), cudaMemcpyDeviceToHost, b->stream));
    HB_CU(cudaStreamSynchronize(b->stream));
    for (int c = 0; c < b->count; ++c) {
        if (info[2 * c + 1])
            return fail(b, HF_ERR_NUMERIC, "density of cluster " + std::to_string(c) + " is not positive semidefinite");
        if (info[2 * c] > maxr)
            return fail(b, HF_ERR_NUMERIC, "density of cluster " + std::to_string(c) + " has rank above " +
                                               std::to_string(maxr));
    }
    return HF_OK;
}

int hf_dgemm_nt(int64_t m, int64_t n, int64_t k, const double* a, int64_t lda, int64_t stride_a, const double* b_,
                int64_t ldb, int64_t stride_b, double* c, int64_t ldc, int64_t stride_c, double alpha, double beta,
                int batch, int tile, void* stream) {
    if (m < 1 || n < 1 || k < 1 || m > INT32_MAX || n > INT32_MAX || k > INT32_MAX || !a || !b_ || !c || batch < 1 ||
        batch > 65535 || tile < 0 || tile >= kTileCount || lda < k || ldb < k || ldc < n)
        return HF_ERR_ARG;
    GemmArgs g{};
    g.M = (int)m;
    g.N = (int)n;
    g.K = (int)k;
    g.A = a;
    g.lda = lda;
    g.B = b_;
    g.ldb = ldb;
    g.C = c;
    g.ldc = ldc;
    g.alpha = alpha;
    g.beta = beta;
    g.strideA = stride_a;
    g.strideB = stride_b;
    g.strideC = stride_c;
    g.tile = tile;
    cudaError_t e = dgemm_nt(g, batch, (cudaStream_t)stream);
    return e == cudaSuccess ? HF_OK : HF_ERR_CUDA;
}

}  // extern "C"
