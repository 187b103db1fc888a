// Coulomb and exchange builds over the packed fitted tensor.
//
// Reference: hafnium/scf/coulomb_exchange.py:176-190. The reference holds B as
// [aux, ao, ao] and computes J = (B . vec D) . B and K = sum_P B_P D B_P. Here B
// is stored once per auxiliary index as the upper-triangle 64x64 tiles of
// B_P (layout: B[q][tile][64][64], tile (I, J >= I) at I*nt - I(I-1)/2 + J - I):
//
//   J:  c_q = sum_t w_t <B_q[t], D[t]>  (w = 1 on diagonal tiles, 2 above), then
//       J[t] = sum_q c_q B_q[t]; both passes stream B once from HBM.
//   K:  with D = C W C^T (W diagonal), X_q = B_q C and K = sum_q X_q W X_q^T.
//       The half-transform runs per q on DMMA tensor cores reading the tiles of
//       B_q (transposed for tiles below the diagonal); the second product is a
//       GEMM over the q-chunk, only upper 64x64 output tiles computed.
#include <algorithm>
#include <cmath>
#include <mutex>

#include "dgemm.cuh"
#include "jk.cuh"

namespace hf {

namespace {

__device__ __forceinline__ const double* cluster_tensor(const double* const* Btab, const double* B, int c) {
    return Btab ? Btab[c] : B;
}

// Dw[t][r][c] = scale w_t D[64I + r][64J + c], zero outside n; cluster blockIdx.y.
__global__ void k_pack_density(const double* __restrict__ D, int64_t strideD, double scale, int64_t n, int nt,
                               double* __restrict__ Dw, int64_t strideW, const int* __restrict__ active) {
    const int cl = blockIdx.y;
    if (active && active[cl] == 0) return;
    D += cl * strideD;
    Dw += cl * strideW;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t ntiles = (int64_t)nt * (nt + 1) / 2;
    if (e >= ntiles * 4096) return;
    const int64_t t = e >> 12;
    const int r = (int)((e >> 6) & 63), c = (int)(e & 63);
    // tile index -> (I, J): rows of the upper triangle, row I holds nt - I tiles
    int I = 0;
    int64_t base = 0;
    while (base + (nt - I) <= t) {
        base += nt - I;
        ++I;
    }
    const int J = I + (int)(t - base);
    const int64_t mu = 64 * (int64_t)I + r, nu = 64 * (int64_t)J + c;
    double v = 0.0;
    if (mu < n && nu < n) v = (I == J ? scale : 2.0 * scale) * D[mu * n + nu];
    Dw[e] = v;
}

// c[q] = sum_e B[q][e] Dw[e]; one CTA per (q, cluster), 128-bit loads.
__global__ void __launch_bounds__(512) k_coulomb_charges(const double* const* __restrict__ Btab,
                                                         const double* __restrict__ B, int64_t ldb, int64_t nelem,
                                                         const double* __restrict__ Dw, double* __restrict__ c,
                                                         int64_t strideW, const int* __restrict__ active) {
    const int q = blockIdx.x, cl = blockIdx.y;
    if (active && active[cl] == 0) return;
    B = cluster_tensor(Btab, B, cl);
    Dw += cl * strideW;
    c += cl * strideW;
    const double2* row = reinterpret_cast<const double2*>(B + (int64_t)q * ldb);
    const double2* d = reinterpret_cast<const double2*>(Dw);
    const int64_t n2 = nelem / 2;
    double s0 = 0.0, s1 = 0.0;
    int64_t i = threadIdx.x;
    for (; i + 3 * blockDim.x < n2; i += 4 * blockDim.x) {
        double2 b0 = __ldcs(row + i), b1 = __ldcs(row + i + blockDim.x), b2 = __ldcs(row + i + 2 * blockDim.x),
                b3 = __ldcs(row + i + 3 * blockDim.x);
        double2 d0 = __ldg(d + i), d1 = __ldg(d + i + blockDim.x), d2 = __ldg(d + i + 2 * blockDim.x),
                d3 = __ldg(d + i + 3 * blockDim.x);
        s0 += b0.x * d0.x + b1.x * d1.x + b2.x * d2.x + b3.x * d3.x;
        s1 += b0.y * d0.y + b1.y * d1.y + b2.y * d2.y + b3.y * d3.y;
    }
    for (; i < n2; i += blockDim.x) {
        double2 b0 = __ldcs(row + i), d0 = __ldg(d + i);
        s0 += b0.x * d0.x;
        s1 += b0.y * d0.y;
    }
    double s = s0 + s1;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ double part[32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = (threadIdx.x < blockDim.x / 32) ? part[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) c[q] = v;
    }
}

// Jt[e] += sum_{q in slab} c[q] B[q][e]; each thread owns two adjacent elements.
constexpr int kJSlab = 256;
__global__ void __launch_bounds__(256) k_coulomb_assemble(const double* const* __restrict__ Btab,
                                                          const double* __restrict__ B, int64_t ldb, int64_t nelem,
                                                          int naux, const double* __restrict__ c,
                                                          double* __restrict__ Jt, int64_t strideW,
                                                          const int* __restrict__ active) {
    const int cl = blockIdx.z;
    if (active && active[cl] == 0) return;
    B = cluster_tensor(Btab, B, cl);
    c += cl * strideW;
    Jt += cl * strideW;
    const int64_t e2 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (2 * e2 >= nelem) return;
    const int q0 = blockIdx.y * kJSlab;
    const int q1 = min(naux, q0 + kJSlab);
    double a0 = 0.0, a1 = 0.0, b0 = 0.0, b1 = 0.0;
    int q = q0;
    for (; q + 1 < q1; q += 2) {
        const double2 x = __ldcs(reinterpret_cast<const double2*>(B + (int64_t)q * ldb) + e2);
        const double2 y = __ldcs(reinterpret_cast<const double2*>(B + (int64_t)(q + 1) * ldb) + e2);
        const double cq = __ldg(c + q), cr = __ldg(c + q + 1);
        a0 += cq * x.x;
        a1 += cq * x.y;
        b0 += cr * y.x;
        b1 += cr * y.y;
    }
    if (q < q1) {
        const double2 x = __ldcs(reinterpret_cast<const double2*>(B + (int64_t)q * ldb) + e2);
        const double cq = __ldg(c + q);
        a0 += cq * x.x;
        a1 += cq * x.y;
    }
    atomicAdd(Jt + 2 * e2, a0 + b0);
    atomicAdd(Jt + 2 * e2 + 1, a1 + b1);
}

// Full symmetric matrix from upper 64x64 tiles: J[mu][nu] = tiles(min, max).
__global__ void k_unpack_tiles(const double* __restrict__ Jt, int64_t strideW, int64_t n, int nt,
                               double* __restrict__ J, int64_t strideJ, const int* __restrict__ active) {
    const int cl = blockIdx.y;
    if (active && active[cl] == 0) return;
    Jt += cl * strideW;
    J += cl * strideJ;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * n) return;
    int64_t mu = e / n, nu = e % n;
    int I = (int)(mu >> 6), Jc = (int)(nu >> 6);
    if (I > Jc) {
        const int64_t t = mu;
        mu = nu;
        nu = t;
        const int ti = I;
        I = Jc;
        Jc = ti;
    }
    const int64_t tile = (int64_t)I * nt - (int64_t)I * (I - 1) / 2 + (Jc - I);
    J[e] = Jt[tile * 4096 + (mu & 63) * 64 + (nu & 63)];
}

// K[mu][nu] from the upper-tile-valid padded matrix Kp (row stride ldk).
__global__ void k_symmetrize_upper(const double* __restrict__ Kp, int64_t ldk, int64_t n, double* __restrict__ K,
                                   int64_t strideK, const int* __restrict__ active) {
    const int cl = blockIdx.y;
    if (active && active[cl] == 0) return;
    Kp += cl * ldk * ldk;
    K += cl * strideK;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * n) return;
    const int64_t mu = e / n, nu = e % n;
    K[e] = mu <= nu ? Kp[mu * ldk + nu] : Kp[nu * ldk + mu];
}

// X[p][ql][i] = sum_r B_q[p][r] Ct[i][r] for q = q0 + ql: 64 x 64 tiles, 4 warps,
// mma.sync.m16n8k8 (FP64), a 2-stage pipeline of 32-wide k slices moved by
// 16-byte cp.async copies (three CTAs per SM; 128 x 64 tiles with 3 stages of 16
// were 4 % slower). The A operand comes from the packed tiles: tile (Ip, J) when
// Ip <= J, else tile (J, Ip) read in its own orientation and transposed by the
// fragment loads.
constexpr int XBM = 64, XBN = 64, XBK = 32, XLD = XBK + 4, XST = 2, XTHREADS = 128;
constexpr int XLDT = 64 + 4;  // pitch of a k-major half: conflict-free fragment loads
static_assert(XBK * XLDT <= 64 * XLD, "a k-major half fits in the p-major half's space");
static_assert(XBM % 64 == 0 && 64 % XBK == 0, "a k slice stays inside one packed tile");

__device__ __forceinline__ uint32_t xsmem(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// 16-byte asynchronous copy (both addresses 16-byte aligned); an invalid piece
// copies nothing and zero-fills.
__device__ __forceinline__ void xcp16(double* dst, const double* src, const double* base, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(xsmem(dst)), "l"(valid ? src : base),
                 "r"(valid ? 16 : 0));
}

__device__ __forceinline__ void xmma(double (&c)[4], const double (&a)[4], const double (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

__global__ void __launch_bounds__(XTHREADS, 3) k_exchange_half(const double* const* __restrict__ Btab,
                                                             const double* __restrict__ B, int64_t ldb, int q0, int nt,
                                                             const double* __restrict__ Ct, int64_t ldc_t,
                                                             int64_t strideCt, int npad, double* __restrict__ X,
                                                             int64_t ldx, int64_t strideX, int opad,
                                                             const int* __restrict__ active, int transposed) {
    const int row_tiles = (npad + XBM - 1) / XBM;
    const int cl = blockIdx.y / row_tiles;
    if (active && active[cl] == 0) return;
    const int m0 = (blockIdx.y % row_tiles) * XBM, n0 = blockIdx.x * XBN;
    const int ql = blockIdx.z;
    B = cluster_tensor(Btab, B, cl);
    Ct += cl * strideCt;
    X += cl * strideX;
    const double* Bq = B + (int64_t)(q0 + ql) * ldb;
    extern __shared__ double xs[];
    double* As = xs;
    double* Bs = xs + XST * XBM * XLD;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int gq = lane >> 2, tq = lane & 3;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int nk = npad / XBK;

    // Each stage holds the A rows as two 64-row halves. A half whose tile lies on
    // or above the diagonal (Ip <= J) is stored p-major ([p][k], pitch XLD) from
    // tile (Ip, J); a half below it reads tile (J, Ip), where k is the slow index,
    // and is stored k-major ([k][p], pitch XLDT) so that both the global reads and
    // the shared writes are contiguous; the fragment loads read it transposed.
    auto tile_at = [&](int I, int Jt) -> const double* {
        return Bq + ((int64_t)I * nt - (int64_t)I * (I - 1) / 2 + (Jt - I)) * 4096;
    };
    auto load = [&](int stage, int k0) {
        double* as = As + stage * XBM * XLD;
        double* bs = Bs + stage * XBN * XLD;
        const int J = k0 >> 6, kin = k0 & 63;
        constexpr int PIECES = 64 * XBK / 2;  // 16-byte pieces of a 64 x XBK half
#pragma unroll
        for (int h = 0; h < XBM / 64; ++h) {
            const int p0 = m0 + 64 * h;
            const int Ip = p0 >> 6;
            double* ah = as + h * 64 * XLD;
            const bool valid = p0 < npad;
            const bool below = Ip > J;
            const double* tile = valid ? (below ? tile_at(J, Ip) : tile_at(Ip, J)) : Bq;
#pragma unroll
            for (int c = 0; c < PIECES / XTHREADS; ++c) {
                const int e = tid + c * XTHREADS;
                if (!below) {
                    const int r = e / (XBK / 2), kp = (e % (XBK / 2)) * 2;
                    xcp16(ah + r * XLD + kp, tile + r * 64 + kin + kp, Bq, valid);
                } else {
                    const int k = e >> 5, pp = (e & 31) * 2;
                    xcp16(ah + k * XLDT + pp, tile + (kin + k) * 64 + pp, Bq, valid);
                }
            }
        }
#pragma unroll
        for (int c = 0; c < XBN * XBK / 2 / XTHREADS; ++c) {
            const int e = tid + c * XTHREADS;  // the 16-byte pieces of the XBN x XBK tile of Ct
            const int r = e / (XBK / 2), kp = (e % (XBK / 2)) * 2;
            xcp16(bs + r * XLD + kp, Ct + (int64_t)(n0 + r) * ldc_t + k0 + kp, Ct, true);
        }
    };

    double acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[i][j][v] = 0.0;
#pragma unroll
    for (int s = 0; s < XST - 1; ++s) {
        if (s < nk) load(s, s * XBK);
        asm volatile("cp.async.commit_group;\n" ::);
    }
    for (int it = 0; it < nk; ++it) {
        asm volatile("cp.async.wait_group %0;\n" ::"n"(XST - 2));
        __syncthreads();
        const int nxt = it + XST - 1;
        if (nxt < nk) load(nxt % XST, nxt * XBK);
        asm volatile("cp.async.commit_group;\n" ::);
        const double* as = As + (it % XST) * XBM * XLD;
        const double* bs = Bs + (it % XST) * XBN * XLD;
        // this warp's 32 rows lie in one half; that half's layout for this k tile
        const int hh = wm >> 6, lr = wm & 63;
        const bool below = ((m0 >> 6) + hh) > ((it * XBK) >> 6);
        const double* ah = as + hh * 64 * XLD;
#pragma unroll
        for (int kk = 0; kk < XBK; kk += 8) {
            double af[2][4], bf[4][2];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int row = lr + i * 16 + gq;
                if (!below) {
                    const double* r0 = ah + row * XLD + kk + tq;
                    af[i][0] = r0[0];
                    af[i][1] = r0[8 * XLD];
                    af[i][2] = r0[4];
                    af[i][3] = r0[8 * XLD + 4];
                } else {
                    const double* c0 = ah + (kk + tq) * XLDT + row;
                    af[i][0] = c0[0];
                    af[i][1] = c0[8];
                    af[i][2] = c0[4 * XLDT];
                    af[i][3] = c0[4 * XLDT + 8];
                }
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const double* c0 = bs + (wn + j * 8 + gq) * XLD + kk + tq;
                bf[j][0] = c0[0];
                bf[j][1] = c0[4];
            }
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) xmma(acc[i][j], af[i], bf[j]);
        }
    }
    asm volatile("cp.async.wait_group 0;\n" ::);
    if (transposed) {
        // Xt[(ql, i)][p]: row (ql opad + i), row stride npad
        double* xt = X + (int64_t)ql * opad * npad;
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int m = m0 + wm + i * 16 + gq + h * 8;
                    const int nn = n0 + wn + j * 8 + 2 * tq;
                    if (m < npad) {
                        xt[(int64_t)nn * npad + m] = acc[i][j][2 * h];
                        xt[(int64_t)(nn + 1) * npad + m] = acc[i][j][2 * h + 1];
                    }
                }
        return;
    }
    double* xo = X + (int64_t)ql * opad;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int m = m0 + wm + i * 16 + gq + h * 8;
                const int nn = n0 + wn + j * 8 + 2 * tq;
                if (m < npad)
                    *reinterpret_cast<double2*>(xo + (int64_t)m * ldx + nn) = make_double2(acc[i][j][2 * h], acc[i][j][2 * h + 1]);
            }
}

// Pivoted Cholesky of a symmetric PSD n x n matrix D in one CTA per cluster:
// rows of Lc ([rank][n]) with D ~= Lc^T Lc, stopping after maxr rows or when the
// largest remaining diagonal entry falls to tol times the largest initial one.
// out = {rank, indefinite}.
__global__ void __launch_bounds__(1024) k_pivoted_cholesky(const double* __restrict__ D, int64_t strideD, int n,
                                                           double tol, int maxr, double* __restrict__ Lc,
                                                           int64_t strideL, int* __restrict__ out,
                                                           const int* __restrict__ active) {
    const int cl = blockIdx.x;
    if (active && active[cl] == 0) return;
    D += cl * strideD;
    Lc += cl * strideL;
    out += 2 * cl;
    extern __shared__ double sm[];
    double* d = sm;                                  // n
    unsigned char* used = (unsigned char*)(sm + n);  // n
    __shared__ double rv[32];
    __shared__ int ri[32];
    __shared__ double s_dmax0, s_piv;
    __shared__ int s_p, s_stop;
    const int tid = threadIdx.x;
    for (int i = tid; i < n; i += blockDim.x) {
        d[i] = D[(int64_t)i * n + i];
        used[i] = 0;
    }
    __syncthreads();
    // largest |diagonal|
    double m = 0.0;
    for (int i = tid; i < n; i += blockDim.x) m = fmax(m, fabs(d[i]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((tid & 31) == 0) rv[tid >> 5] = m;
    __syncthreads();
    if (tid == 0) {
        double v = 0.0;
        for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) v = fmax(v, rv[w]);
        s_dmax0 = v;
    }
    __syncthreads();
    int k = 0;
    for (; k < maxr; ++k) {
        double best = -1.0;
        int bi = -1;
        for (int i = tid; i < n; i += blockDim.x)
            if (!used[i] && d[i] > best) {
                best = d[i];
                bi = i;
            }
        for (int o = 16; o > 0; o >>= 1) {
            const double ob = __shfl_xor_sync(0xffffffffu, best, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ob > best || (ob == best && oi >= 0 && (bi < 0 || oi < bi))) {
                best = ob;
                bi = oi;
            }
        }
        if ((tid & 31) == 0) {
            rv[tid >> 5] = best;
            ri[tid >> 5] = bi;
        }
        __syncthreads();
        if (tid == 0) {
            double b = -1.0;
            int p = -1;
            for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w)
                if (rv[w] > b || (rv[w] == b && ri[w] >= 0 && (p < 0 || ri[w] < p))) {
                    b = rv[w];
                    p = ri[w];
                }
            s_stop = (p < 0 || !(b > tol * s_dmax0)) ? 1 : 0;
            s_p = p;
            s_piv = s_stop ? 0.0 : sqrt(b);
        }
        __syncthreads();
        if (s_stop) break;
        const int p = s_p;
        const double piv = s_piv;
        for (int i = tid; i < n; i += blockDim.x) {
            double l = 0.0;
            if (i == p) l = piv;
            else if (!used[i]) {
                double s = D[(int64_t)p * n + i];
                for (int j = 0; j < k; ++j) s -= Lc[(int64_t)j * n + i] * Lc[(int64_t)j * n + p];
                l = s / piv;
            }
            Lc[(int64_t)k * n + i] = l;
        }
        __syncthreads();
        for (int i = tid; i < n; i += blockDim.x) {
            if (i == p) used[i] = 1;
            else if (!used[i]) {
                const double l = Lc[(int64_t)k * n + i];
                d[i] -= l * l;
            }
        }
        __syncthreads();
    }
    // indefinite if a remaining diagonal entry is clearly negative
    int bad = 0;
    for (int i = tid; i < n; i += blockDim.x)
        if (!used[i] && d[i] < -1e3 * tol * s_dmax0) bad = 1;
    bad = __syncthreads_or(bad);
    if (tid == 0) {
        out[0] = k;
        out[1] = bad;
    }
}

// Blocked pivoted Cholesky of one matrix: the pivots and the factor of
// k_pivoted_cholesky, with the rows that pivots already taken subtract kept in
// a working copy W = D - sum L L^T that a DMMA product updates once per panel
// of kPivotPanel pivots. Within a panel each pivot's column needs W's row and
// at most kPivotPanel - 1 corrections instead of one per earlier pivot, so the
// sequential part no longer rereads the whole factor from L2 at every pivot.
constexpr int kPivotPanel = 32;
struct PivotState {
    double dmax0;  // the largest initial diagonal entry
    int k;         // pivots taken
    int stop;      // 1 once the remaining diagonal falls below tol dmax0 or k reaches maxr
    int active;    // the trailing update of this panel has work (DMMA batch flag)
    int pad;
};

__device__ __forceinline__ void block_argmax(double best, int bi, double* rv, int* ri, double& out_best,
                                             int& out_i) {
    for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi >= 0 && (bi < 0 || oi < bi))) {
            best = ob;
            bi = oi;
        }
    }
    if ((threadIdx.x & 31) == 0) {
        rv[threadIdx.x >> 5] = best;
        ri[threadIdx.x >> 5] = bi;
    }
    __syncthreads();
    double b = -1.0;
    int p = -1;
    for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w)
        if (rv[w] > b || (rv[w] == b && ri[w] >= 0 && (p < 0 || ri[w] < p))) {
            b = rv[w];
            p = ri[w];
        }
    out_best = b;
    out_i = p;
}

__global__ void __launch_bounds__(1024) k_pc_init(const double* __restrict__ D, int n, double* __restrict__ d,
                                                  unsigned char* __restrict__ used, PivotState* st) {
    __shared__ double rv[32];
    __shared__ int ri[32];
    double m = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        d[i] = D[(int64_t)i * n + i];
        used[i] = 0;
        m = fmax(m, fabs(d[i]));
    }
    double b;
    int unused_i;
    block_argmax(m, (int)threadIdx.x, rv, ri, b, unused_i);
    if (threadIdx.x == 0) {
        st->dmax0 = b;
        st->k = 0;
        st->stop = n > 0 ? 0 : 1;
        st->active = 0;
    }
}

__global__ void __launch_bounds__(512) k_pc_panel(const double* __restrict__ W, int n, double tol, int maxr,
                                                   double* __restrict__ Lc, double* __restrict__ Lp,
                                                   double* __restrict__ d, unsigned char* __restrict__ used,
                                                   PivotState* st) {
    __shared__ double rv[32];
    __shared__ int ri[32];
    __shared__ double s_piv;
    __shared__ int s_p, s_stop;
    const int tid = threadIdx.x;
    const int k0 = st->k;
    const double dmax0 = st->dmax0;
    if (st->stop) {
        if (tid == 0) st->active = 0;
        return;
    }
    const int b = min(kPivotPanel, maxr - k0);
    int done = 0;
    for (int j = 0; j < b; ++j) {
        double best = -1.0;
        int bi = -1;
        for (int i = tid; i < n; i += blockDim.x)
            if (!used[i] && d[i] > best) {
                best = d[i];
                bi = i;
            }
        double bb;
        int p;
        block_argmax(best, bi, rv, ri, bb, p);
        if (tid == 0) {
            s_stop = (p < 0 || !(bb > tol * dmax0)) ? 1 : 0;
            s_p = p;
            s_piv = s_stop ? 0.0 : sqrt(bb);
        }
        __syncthreads();
        if (s_stop) break;
        const int pv = s_p;
        const double piv = s_piv;
        // each thread owns rows i = tid + m blockDim.x: it alone writes their column
        // entries, diagonal and used flag, and alone reads d and used for them in
        // the next pivot's search, so the two barriers of the search suffice
        for (int i = tid; i < n; i += blockDim.x) {
            double l = 0.0;
            if (i == pv) {
                l = piv;
                used[i] = 1;
            } else if (!used[i]) {
                double sum = W[(int64_t)pv * n + i];
                for (int jj = 0; jj < j; ++jj) sum -= Lp[i * kPivotPanel + jj] * Lp[pv * kPivotPanel + jj];
                l = sum / piv;
                d[i] -= l * l;
            }
            Lc[(int64_t)(k0 + j) * n + i] = l;
            Lp[i * kPivotPanel + j] = l;
        }
        ++done;
    }
    __syncthreads();
    // columns of the panel past its last pivot add nothing to the trailing update
    for (int e = tid; e < n * kPivotPanel; e += blockDim.x)
        if (e % kPivotPanel >= done) Lp[e] = 0.0;
    if (tid == 0) {
        st->k = k0 + done;
        st->stop = (done < b || k0 + done >= maxr) ? 1 : 0;
        st->active = done > 0 ? 1 : 0;
    }
}

__global__ void __launch_bounds__(1024) k_pc_finish(int n, double tol, const double* __restrict__ d,
                                                    const unsigned char* __restrict__ used,
                                                    const PivotState* st, int* __restrict__ out) {
    // indefinite if a remaining diagonal entry is clearly negative
    int bad = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        if (!used[i] && d[i] < -1e3 * tol * st->dmax0) bad = 1;
    bad = __syncthreads_or(bad);
    if (threadIdx.x == 0) {
        out[0] = st->k;
        out[1] = bad;
    }
}

// Ct[i][mu] = Lc[i][mu] for i < rank and mu < n (rank = info[2 c]), else 0;
// sign[i] = 1 when sign is given (single cluster).
__global__ void k_factor_pad(const double* __restrict__ Lc, int64_t strideL, int64_t n, const int* __restrict__ info,
                             double* __restrict__ Ct, int64_t strideCt, int64_t npad, int64_t opad,
                             double* __restrict__ sign, const int* __restrict__ active) {
    const int cl = blockIdx.y;
    if (active && active[cl] == 0) return;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= opad * npad) return;
    const int64_t rank = info[2 * cl];
    const int64_t i = e / npad, mu = e % npad;
    Ct[cl * strideCt + e] = (i < rank && mu < n) ? Lc[cl * strideL + i * n + mu] : 0.0;
    if (sign && mu == 0) sign[i] = 1.0;
}

// Kp[c][e] += sum_s P[c][s][e] in split order (deterministic split-K reduction).
__global__ void k_sum_splits(const double* __restrict__ P, int splits, int64_t nn, double* __restrict__ Kp,
                             const int* __restrict__ active) {
    const int c = blockIdx.y;
    if (active && active[c] == 0) return;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nn) return;
    const double* src = P + (int64_t)c * splits * nn + e;
    double s = 0.0;
    for (int k = 0; k < splits; ++k) s += src[(int64_t)k * nn];
    Kp[(int64_t)c * nn + e] += s;
}

constexpr int kMaxDevices = 64;
constexpr int kPivotSmem = 200 * 1024;
std::mutex g_jk_mutex;
bool g_jk_configured[kMaxDevices] = {};

__global__ void k_scale_columns(const double* __restrict__ X, double* __restrict__ Xs, int64_t rows, int64_t ld,
                                int opad, const double* __restrict__ sign) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= rows * ld) return;
    Xs[e] = X[e] * sign[(e % ld) % opad];
}

}  // namespace

cudaError_t coulomb_build(const JkPlan& p, const double* D, int64_t strideD, double scale, double* J, int64_t strideJ,
                          double* work, cudaStream_t stream) {
    // work per cluster: Dw (ntiles*4096) | c (naux) | Jt (ntiles*4096)
    const int64_t nelem = p.ntiles * 4096;
    const int64_t sw = coulomb_work_doubles(p);
    double* Dw = work;
    double* c = work + nelem;
    double* Jt = c + ((p.naux + 1) / 2) * 2;
    const unsigned cnt = (unsigned)p.count;
    k_pack_density<<<dim3((unsigned)((nelem + 255) / 256), cnt), 256, 0, stream>>>(D, strideD, scale, p.n, p.nt, Dw, sw,
                                                                                   p.active);
    k_coulomb_charges<<<dim3(p.naux, cnt), 512, 0, stream>>>(p.Btab, p.B, p.ldb, nelem, Dw, c, sw, p.active);
    if (p.count == 1) {
        cudaMemsetAsync(Jt, 0, sizeof(double) * nelem, stream);
    } else {
        cudaMemset2DAsync(Jt, sizeof(double) * sw, 0, sizeof(double) * nelem, p.count, stream);
    }
    dim3 grid((unsigned)((nelem / 2 + 255) / 256), (p.naux + kJSlab - 1) / kJSlab, cnt);
    k_coulomb_assemble<<<grid, 256, 0, stream>>>(p.Btab, p.B, p.ldb, nelem, p.naux, c, Jt, sw, p.active);
    const int64_t nn = p.n * p.n;
    k_unpack_tiles<<<dim3((unsigned)((nn + 255) / 256), cnt), 256, 0, stream>>>(Jt, sw, p.n, p.nt, J, strideJ, p.active);
    return cudaGetLastError();
}

int64_t coulomb_work_doubles(const JkPlan& p) { return 2 * p.ntiles * 4096 + ((p.naux + 1) / 2) * 2; }

cudaError_t fitted_charges(const JkPlan& p, const double* D, double* d, double* work, cudaStream_t stream) {
    const int64_t nelem = p.ntiles * 4096;
    k_pack_density<<<dim3((unsigned)((nelem + 255) / 256), 1), 256, 0, stream>>>(D, 0, 1.0, p.n, p.nt, work, 0,
                                                                                 nullptr);
    k_coulomb_charges<<<dim3(p.naux, 1), 512, 0, stream>>>(nullptr, p.B, p.ldb, nelem, work, d, 0, nullptr);
    return cudaGetLastError();
}

// The SYRK's CTA tile: 64 x 64 with 2 stages of 32-wide k slices (tile 5).
constexpr int kSyrkTile = 5;

int syrk_splits(int64_t npad, int count) {
    const int bm = kTileShapes[kSyrkTile][0], bn = kTileShapes[kSyrkTile][1];
    const int64_t mt = (npad + bm - 1) / bm, nt = (npad + bn - 1) / bn;
    int64_t upper = 0;
    for (int64_t i = 0; i < mt; ++i)
        for (int64_t j = 0; j < nt; ++j)
            if (i * bm <= j * bn + bn - 1) ++upper;
    const int64_t ctas = upper * std::max(1, count);
    // enough CTAs for many waves: the tail of a last partial wave cost up to 13 %
    // of an FP64 K build at (H2O)64 with two splits
    const int64_t want = 12 * 148;
    int s = (int)std::min<int64_t>(32, (want + ctas - 1) / ctas);
    while (s > 1 && (int64_t)s * std::max(1, count) > 65535) --s;
    return std::max(1, s);
}

int64_t syrk_partial_doubles(int64_t npad, int count) {
    const int s = syrk_splits(npad, count);
    return s > 1 ? (int64_t)s * std::max(1, count) * npad * npad : 0;
}

cudaError_t exchange_build_fp64(const JkPlan& p, const double* Ct, int64_t strideCt, int opad, const double* sign,
                                double* K, int64_t strideK, double* Kp, double* X, double* Xs, double* partial,
                                int qchunk, cudaStream_t stream) {
    const int64_t npad = (int64_t)p.nt * 64;
    if (sign != nullptr && p.count != 1) return cudaErrorInvalidValue;
    cudaError_t e = jk_configure();
    if (e != cudaSuccess) return e;
    cudaMemsetAsync(Kp, 0, sizeof(double) * npad * npad * p.count, stream);
    const int smem = XST * (XBM + XBN) * XLD * (int)sizeof(double);
    const int row_tiles = (int)((npad + XBM - 1) / XBM);
    const int64_t strideX = npad * (int64_t)qchunk * opad;
    for (int q0 = 0; q0 < p.naux; q0 += qchunk) {
        const int qc = (p.naux - q0 < qchunk) ? p.naux - q0 : qchunk;
        const int64_t ldx = (int64_t)qc * opad;
        dim3 grid(opad / 64, (unsigned)(row_tiles * p.count), qc);
        k_exchange_half<<<grid, XTHREADS, smem, stream>>>(p.Btab, p.B, p.ldb, q0, p.nt, Ct, npad, strideCt, (int)npad, X,
                                                          ldx, strideX, opad, p.active, 0);
        const double* Xb = X;
        if (sign != nullptr) {
            const int64_t tot = npad * ldx;
            k_scale_columns<<<(unsigned)((tot + 255) / 256), 256, 0, stream>>>(X, Xs, npad, ldx, opad, sign);
            Xb = Xs;
        }
        GemmArgs g{};
        g.M = g.N = (int)npad;
        g.K = (int)ldx;
        g.A = X;
        g.lda = ldx;
        g.B = Xb;
        g.ldb = ldx;
        g.C = Kp;
        g.ldc = npad;
        g.alpha = 1.0;
        g.beta = 1.0;
        g.kmode = 0;
        g.epi = 3;
        g.tile = kSyrkTile;
        g.strideA = g.strideB = strideX;
        g.strideC = npad * npad;
        g.active = p.active;
        const int splits = partial ? syrk_splits(npad, p.count) : 1;
        if (splits > 1) {
            // partial products per split, then a fixed-order sum into Kp
            g.C = partial;
            g.beta = 0.0;
            g.splits = splits;
            e = dgemm_nt(g, p.count, stream);
            if (e != cudaSuccess) return e;
            const int64_t nn2 = npad * npad;
            k_sum_splits<<<dim3((unsigned)((nn2 + 255) / 256), (unsigned)p.count), 256, 0, stream>>>(
                partial, splits, nn2, Kp, p.active);
        } else {
            e = dgemm_nt(g, p.count, stream);
        }
        if (e != cudaSuccess) return e;
    }
    const int64_t nn = p.n * p.n;
    k_symmetrize_upper<<<dim3((unsigned)((nn + 255) / 256), (unsigned)p.count), 256, 0, stream>>>(Kp, npad, p.n, K,
                                                                                                 strideK, p.active);
    return cudaGetLastError();
}

cudaError_t pivoted_cholesky(const double* D, int64_t strideD, int n, double tol, int maxr, double* Lc,
                             int64_t strideL, int* info, int count, const int* active, cudaStream_t stream) {
    const size_t smem = sizeof(double) * n + n + 16;
    if (smem > kPivotSmem) return cudaErrorInvalidValue;
    cudaError_t e = jk_configure();
    if (e != cudaSuccess) return e;
    k_pivoted_cholesky<<<count, 1024, smem, stream>>>(D, strideD, n, tol, maxr, Lc, strideL, info, active);
    return cudaGetLastError();
}

size_t pivoted_cholesky_work_doubles(int n) {
    return (size_t)n * n + (size_t)n * kPivotPanel + n + (n + 7) / 8 + 4;
}

cudaError_t pivoted_cholesky_blocked(const double* D, int n, double tol, int maxr, double* Lc, int* info,
                                     double* work, cudaStream_t stream) {
    if (n < 1 || maxr < 1) return cudaErrorInvalidValue;
    cudaError_t e = jk_configure();
    if (e != cudaSuccess) return e;
    double* W = work;
    double* Lp = W + (size_t)n * n;
    double* d = Lp + (size_t)n * kPivotPanel;
    unsigned char* used = reinterpret_cast<unsigned char*>(d + n);
    PivotState* st = reinterpret_cast<PivotState*>(d + n + (n + 7) / 8);
    e = cudaMemcpyAsync(W, D, sizeof(double) * (size_t)n * n, cudaMemcpyDeviceToDevice, stream);
    if (e != cudaSuccess) return e;
    k_pc_init<<<1, 1024, 0, stream>>>(D, n, d, used, st);
    const int panels = (maxr + kPivotPanel - 1) / kPivotPanel;
    for (int pnl = 0; pnl < panels; ++pnl) {
        k_pc_panel<<<1, 512, 0, stream>>>(W, n, tol, maxr, Lc, Lp, d, used, st);
        if (pnl + 1 == panels) break;  // no pivot follows the last panel
        // W -= Lp Lp^T (skipped, CTA by CTA, once the factorisation has stopped)
        GemmArgs g{};
        g.M = g.N = n;
        g.K = kPivotPanel;
        g.A = g.B = Lp;
        g.lda = g.ldb = kPivotPanel;
        g.C = W;
        g.ldc = n;
        g.alpha = -1.0;
        g.beta = 1.0;
        g.kmode = 0;
        g.epi = 0;
        g.tile = 5;
        g.active = &st->active;
        e = dgemm_nt(g, 1, stream);
        if (e != cudaSuccess) return e;
    }
    k_pc_finish<<<1, 1024, 0, stream>>>(n, tol, d, used, st, info);
    return cudaGetLastError();
}

cudaError_t factor_pad(const double* Lc, int64_t strideL, int64_t n, const int* info, double* Ct, int64_t strideCt,
                       int64_t npad, int64_t opad, double* sign, int count, const int* active, cudaStream_t stream) {
    k_factor_pad<<<dim3((unsigned)((opad * npad + 255) / 256), (unsigned)count), 256, 0, stream>>>(
        Lc, strideL, n, info, Ct, strideCt, npad, opad, sign, active);
    return cudaGetLastError();
}

cudaError_t half_transform_t(const JkPlan& p, const double* Ct, int opad, int q0, int qc, double* Xt,
                             cudaStream_t stream) {
    if (p.count != 1) return cudaErrorInvalidValue;
    cudaError_t e = jk_configure();
    if (e != cudaSuccess) return e;
    const int64_t npad = (int64_t)p.nt * 64;
    const int smem = XST * (XBM + XBN) * XLD * (int)sizeof(double);
    dim3 grid(opad / 64, (unsigned)((npad + XBM - 1) / XBM), qc);
    k_exchange_half<<<grid, XTHREADS, smem, stream>>>(p.Btab, p.B, p.ldb, q0, p.nt, Ct, npad, 0, (int)npad, Xt, 0, 0,
                                                      opad, nullptr, 1);
    return cudaGetLastError();
}

cudaError_t jk_configure() {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_jk_mutex);
    if (g_jk_configured[dev]) return cudaSuccess;
    const int smem = XST * (XBM + XBN) * XLD * (int)sizeof(double);
    e = cudaFuncSetAttribute(k_exchange_half, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_pivoted_cholesky, cudaFuncAttributeMaxDynamicSharedMemorySize, kPivotSmem);
    if (e != cudaSuccess) return e;
    g_jk_configured[dev] = true;
    return dgemm_configure();
}

}  // namespace hf
