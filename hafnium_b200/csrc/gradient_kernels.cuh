// Derivative integrals for the DF-RHF nuclear gradient, contracted on the fly.
//
// Included by gradient.cu, which holds the __constant__ tables. The reference
// (hafnium/properties/gradient.py:72-235) forms dense derivative tensors
// [3, aux, ao, ao] and contracts them with effective
// densities; at cluster sizes those tensors are 3x the fitted tensor, so here
// every derivative integral is contracted with its density weight as soon as
// it is formed and only per-shell force sums leave the kernels:
//
//   k_three_center_grad  (d_P P|uv) and (P|d_A uv) against the Coulomb weight
//                        c_P D_uv and the exchange weight GK_P,uv of one block
//                        of auxiliary functions; the derivative for the second
//                        orbital centre follows from translational invariance,
//                        d_A + d_B + d_P = 0 (two_electron.rs:300-394).
//   k_metric_grad        (d_P P|Q) against the metric weights W^J, W^K (of W^K only
//                        the upper triangle is read).
//   k_one_electron_grad  <d_A u|O|v> for S, T and V against W and D.
//   k_attraction_nucleus_grad
//                        <u|d_C V_C|v> against D, one nucleus per grid row.
//
// Derivatives follow two rules (the reference's Differentiate,
// two_electron.rs:1138-1150): a lone function's centre (an auxiliary function,
// a nucleus) by the shift of the Hermite integrals, d/dX R_tuv(X - Y) =
// R_{t+1,u,v}; the centre of an orbital function by raising and lowering its
// angular momentum, d/dA_x x_A^i e^{-a x_A^2} = 2a x_A^{i+1} e^{..} - i x_A^{i-1} e^{..}.
// Force sums are accumulated with FP64 atomics (their order varies from run to
// run at the level of rounding).
#pragma once

namespace hf {

template <int LA, int LB>
struct GradPairLayout {
    static constexpr int NSA = nsph(LA), NSB = nsph(LB), NSAB = NSA * NSB;
    static constexpr int KA = kMaxOrbContr[LA], KB = kMaxOrbContr[LB], KK = KA * KB;
    static constexpr int NH = ntet(LA + LB), NH1 = ntet(LA + LB + 1);
    // per primitive pair: p, Px, Py, Pz | cc[KK] | E[NSAB][NH] | EA[3][NSAB][NH1] | EJ[NH] | EJA[3][NH1]
    static constexpr int OFF_E = 4 + KK;
    static constexpr int OFF_EA = OFF_E + NSAB * NH;
    static constexpr int OFF_EJ = OFF_EA + 3 * NSAB * NH1;
    static constexpr int OFF_EJA = OFF_EJ + NH;
    static constexpr int STRIDE = OFF_EJA + 3 * NH1;
};

// Spherical Hermite coefficients of a primitive pair and of its derivative by the
// centre of its first function, and both contracted with the pair's block of the
// total density D (the Coulomb weight's orbital part).
template <int LA, int LB>
__device__ int grad_pair_prologue(const DevShell& A, const DevShell& B, const double* __restrict__ exps,
                                  const double* __restrict__ coefs, const double* __restrict__ D, int64_t n,
                                  double* smem, int* s_pos) {
    using PL = GradPairLayout<LA, LB>;
    constexpr int NCA = ncart(LA), NCB = ncart(LB);
    const int npp = A.nprim * B.nprim;
    const double abx = A.x - B.x, aby = A.y - B.y, abz = A.z - B.z;
    const double rab2 = abx * abx + aby * aby + abz * abz;
    for (int pp0 = threadIdx.x; pp0 < npp; pp0 += blockDim.x) {
        const int i = pp0 / B.nprim, j = pp0 % B.nprim;
        const double a = exps[A.prim + i], b = exps[B.prim + j];
        double cmax = 0.0;
        for (int ka = 0; ka < A.ncontr; ++ka)
            for (int kb = 0; kb < B.ncontr; ++kb)
                cmax = fmax(cmax, fabs(coefs[A.coef + ka * A.nprim + i] * coefs[B.coef + kb * B.nprim + j]));
        s_pos[pp0] = (cmax * exp(-(a * b / (a + b)) * rab2) >= kPairScreen) ? 1 : 0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int k = 0;
        for (int pp0 = 0; pp0 < npp; ++pp0) {
            const int keep = s_pos[pp0];
            s_pos[pp0] = keep ? k : -1;
            k += keep;
        }
        s_pos[kMaxPrimPairs] = k;
    }
    __syncthreads();
    for (int pp0 = threadIdx.x; pp0 < npp; pp0 += blockDim.x) {
        const int pp = s_pos[pp0];
        if (pp < 0) continue;
        const int i = pp0 / B.nprim, j = pp0 % B.nprim;
        const double a = exps[A.prim + i], b = exps[B.prim + j];
        const double p = a + b;
        const double mu = a * b / p;
        const double px = (a * A.x + b * B.x) / p, py = (a * A.y + b * B.y) / p, pz = (a * A.z + b * B.z) / p;
        double* s = smem + pp * PL::STRIDE;
        s[0] = p;
        s[1] = px;
        s[2] = py;
        s[3] = pz;
#pragma unroll
        for (int ka = 0; ka < PL::KA; ++ka)
#pragma unroll
            for (int kb = 0; kb < PL::KB; ++kb)
                s[4 + ka * PL::KB + kb] = (ka < A.ncontr && kb < B.ncontr)
                                              ? coefs[A.coef + ka * A.nprim + i] * coefs[B.coef + kb * B.nprim + j]
                                              : 0.0;
        Hermite1D<LA + 1, LB> ex, ey, ez;
        ex.build(p, exp(-mu * rab2), px - A.x, px - B.x);
        ey.build(p, 1.0, py - A.y, py - B.y);
        ez.build(p, 1.0, pz - A.z, pz - B.z);
        double* et = s + PL::OFF_E;
        double* ea = s + PL::OFF_EA;
        for (int k = 0; k < PL::NSAB * PL::NH; ++k) et[k] = 0.0;
        for (int k = 0; k < 3 * PL::NSAB * PL::NH1; ++k) ea[k] = 0.0;
#pragma unroll 1
        for (int ca = 0; ca < NCA; ++ca)
#pragma unroll 1
            for (int cb = 0; cb < NCB; ++cb) {
                const int ix = c_cart[LA][ca][0], iy = c_cart[LA][ca][1], iz = c_cart[LA][ca][2];
                const int jx = c_cart[LB][cb][0], jy = c_cart[LB][cb][1], jz = c_cart[LB][cb][2];
                // value: E^{ij}_t per axis
#pragma unroll 1
                for (int t = 0; t <= ix + jx; ++t)
#pragma unroll 1
                    for (int u = 0; u <= iy + jy; ++u)
#pragma unroll 1
                        for (int v = 0; v <= iz + jz; ++v) {
                            const double w = ex.e[ix][jx][t] * ey.e[iy][jy][u] * ez.e[iz][jz][v];
#pragma unroll 1
                            for (int ma = 0; ma < PL::NSA; ++ma) {
                                const double wa = c_c2s[c2s_offset(LA) + ma * NCA + ca] * w;
                                if (wa == 0.0) continue;
#pragma unroll 1
                                for (int mb = 0; mb < PL::NSB; ++mb)
                                    et[(ma * PL::NSB + mb) * PL::NH + tet(t, u, v)] +=
                                        c_c2s[c2s_offset(LB) + mb * NCB + cb] * wa;
                            }
                        }
                // derivative by the first centre along each axis: 2a E^{i+1,j} - i E^{i-1,j}
#pragma unroll 1
                for (int d = 0; d < 3; ++d) {
                    const int ext = 1;
#pragma unroll 1
                    for (int t = 0; t <= ix + jx + (d == 0 ? ext : 0); ++t) {
                        const double fx = d == 0 ? 2.0 * a * ex.e[ix + 1][jx][t] - (ix > 0 ? ix * ex.e[ix - 1][jx][t] : 0.0)
                                                 : (t <= ix + jx ? ex.e[ix][jx][t] : 0.0);
                        if (fx == 0.0) continue;
#pragma unroll 1
                        for (int u = 0; u <= iy + jy + (d == 1 ? ext : 0); ++u) {
                            const double fy = d == 1 ? 2.0 * a * ey.e[iy + 1][jy][u] - (iy > 0 ? iy * ey.e[iy - 1][jy][u] : 0.0)
                                                     : (u <= iy + jy ? ey.e[iy][jy][u] : 0.0);
                            if (fy == 0.0) continue;
#pragma unroll 1
                            for (int v = 0; v <= iz + jz + (d == 2 ? ext : 0); ++v) {
                                const double fz = d == 2 ? 2.0 * a * ez.e[iz + 1][jz][v] - (iz > 0 ? iz * ez.e[iz - 1][jz][v] : 0.0)
                                                         : (v <= iz + jz ? ez.e[iz][jz][v] : 0.0);
                                const double w = fx * fy * fz;
                                if (w == 0.0) continue;
#pragma unroll 1
                                for (int ma = 0; ma < PL::NSA; ++ma) {
                                    const double wa = c_c2s[c2s_offset(LA) + ma * NCA + ca] * w;
                                    if (wa == 0.0) continue;
#pragma unroll 1
                                    for (int mb = 0; mb < PL::NSB; ++mb)
                                        ea[(d * PL::NSAB + ma * PL::NSB + mb) * PL::NH1 + tet(t, u, v)] +=
                                            c_c2s[c2s_offset(LB) + mb * NCB + cb] * wa;
                                }
                            }
                        }
                    }
                }
            }
        // the Coulomb weight's orbital part: DJ[m] = sum_k cc[k] D[mu_k,m][nu_k,m]
        double dj[PL::NSAB];
#pragma unroll
        for (int m = 0; m < PL::NSAB; ++m) dj[m] = 0.0;
        for (int ka = 0; ka < A.ncontr; ++ka)
            for (int kb = 0; kb < B.ncontr; ++kb) {
                const double c = s[4 + ka * PL::KB + kb];
#pragma unroll
                for (int ma = 0; ma < PL::NSA; ++ma)
#pragma unroll
                    for (int mb = 0; mb < PL::NSB; ++mb)
                        dj[ma * PL::NSB + mb] +=
                            c * D[(int64_t)(A.fn + ka * PL::NSA + ma) * n + B.fn + kb * PL::NSB + mb];
            }
        double* ej = s + PL::OFF_EJ;
        double* eja = s + PL::OFF_EJA;
        for (int h = 0; h < PL::NH; ++h) {
            double acc = 0.0;
#pragma unroll
            for (int m = 0; m < PL::NSAB; ++m) acc += dj[m] * et[m * PL::NH + h];
            ej[h] = acc;
        }
        for (int k = 0; k < 3 * PL::NH1; ++k) {
            const int d = k / PL::NH1, h = k % PL::NH1;
            double acc = 0.0;
#pragma unroll
            for (int m = 0; m < PL::NSAB; ++m) acc += dj[m] * ea[(d * PL::NSAB + m) * PL::NH1 + h];
            eja[k] = acc;
        }
    }
    __syncthreads();
    return s_pos[kMaxPrimPairs];
}

// Sum of 12 per-thread values over the CTA into red[0..11] (thread 0 reads them).
__device__ __forceinline__ void cta_sum12(double* v, double* red) {
#pragma unroll
    for (int k = 0; k < 12; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < 12; ++k) red[warp * 12 + k] = v[k];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
            for (int k = 0; k < 12; ++k) red[k] += red[w * 12 + k];
    }
}

// Threads per CTA of the pair-data kernel (one CTA per shell pair).
constexpr int kGradThreads = 256;

// The pair data of grad_pair_prologue, built once per shell pair into global
// memory (data + offsets[task], npp * STRIDE doubles; npps[task] = the primitive
// pairs kept) for every auxiliary class and block to copy.
template <int LA, int LB>
__global__ void __launch_bounds__(kGradThreads) k_grad_pair_data(const PairTask* __restrict__ tasks,
                                                                 const DevShell* __restrict__ orb,
                                                                 const double* __restrict__ exps,
                                                                 const double* __restrict__ coefs,
                                                                 const double* __restrict__ D, int64_t n,
                                                                 const int64_t* __restrict__ offsets,
                                                                 double* __restrict__ data, int* __restrict__ npps) {
    using PL = GradPairLayout<LA, LB>;
    extern __shared__ double smem[];
    __shared__ int s_pos[kMaxPrimPairs + 1];
    const PairTask task = tasks[blockIdx.x];
    const DevShell A = orb[task.swap ? task.second : task.first];
    const DevShell B = orb[task.swap ? task.first : task.second];
    const int npp = grad_pair_prologue<LA, LB>(A, B, exps, coefs, D, n, smem, s_pos);
    double* dst = data + offsets[blockIdx.x];
    const int total = npp * PL::STRIDE;
    for (int k = threadIdx.x; k < total; k += blockDim.x) dst[k] = smem[k];
    if (threadIdx.x == 0) npps[blockIdx.x] = npp;
}

// Shapes of one class of the three-centre derivative kernel. As in the (P|mu nu)
// kernel, the threads of an auxiliary shell (one per m_P, all in one warp) share
// each primitive triple's R table (order l_a + l_b + l_P + 1): per round TPR of
// them evaluate one triple's table each into a row of shared memory, and after
// a warp barrier every thread contracts all TPR rows with the nonzero entries of
// its own Cartesian-to-spherical row. The pair data stays in global memory
// (read-only, the same address across the CTA), which leaves shared memory to
// the tables.
constexpr int kGradCenterThreads = 128;
constexpr int kGradRTableBytes = 40 * 1024;
template <int LA, int LB, int LP>
struct GradCenterShape {
    static constexpr int L = LA + LB + LP + 1;
    static constexpr int NCP = ncart(LP), NSP = nsph(LP);
    static constexpr int SPW = 32 / NSP;                           // auxiliary shells per warp
    static constexpr int SPB = (kGradCenterThreads / 32) * SPW;    // ... per CTA
    static constexpr int NH = ntet(LA + LB), NH1 = ntet(LA + LB + 1);
    static constexpr int NR = ntet(L);
    static constexpr int RS = (NR + 1) | 1;  // the table and its prefactor, odd: rows in different banks
    static constexpr int FIT = kGradRTableBytes / (SPB * RS * 8);
    static constexpr int TPR = FIT < 1 ? 1 : (FIT > NSP ? NSP : FIT);
    static constexpr int R_DOUBLES = SPB * TPR * RS;
};

// One CTA per orbital shell pair of class (LA <= LB) and slab of SPB auxiliary
// shells of class LP from this block's list; thread (slot, m_P) accumulates,
// for the Coulomb (slot 0..2) and exchange (slot 3..5) weights, the
// auxiliary-centre derivative into gaux[aux shell][6] and the two orbital
// centres' derivatives into gorb[orbital shell][6].
template <int LA, int LB, int LP>
__global__ void __launch_bounds__(kGradCenterThreads) k_three_center_grad(const PairTask* __restrict__ tasks,
                                                           const DevShell* __restrict__ orb,
                                                           const DevShell* __restrict__ aux,
                                                           const double* __restrict__ exps,
                                                           const double* __restrict__ coefs,
                                                           const int* __restrict__ alist, int nalist,
                                                           const double* __restrict__ btable, GradWeights g,
                                                           const int64_t* __restrict__ offsets,
                                                           const double* __restrict__ pdata,
                                                           const int* __restrict__ npps,
                                                           double* __restrict__ gorb, double* __restrict__ gaux) {
    using PL = GradPairLayout<LA, LB>;
    using SH = GradCenterShape<LA, LB, LP>;
    constexpr int L = SH::L, NCP = SH::NCP, NSP = SH::NSP, SPW = SH::SPW, NH = SH::NH, NH1 = SH::NH1;
    constexpr int TPR = SH::TPR, RS = SH::RS, NR = SH::NR;
    extern __shared__ double sR[];           // the round's R tables
    __shared__ int s_idx1[NCP * NH1];        // tet(h + c), h of order <= l_a + l_b + 1
    __shared__ int s_idx3[NCP * NH * 3];     // tet(h + c + e_d), h of order <= l_a + l_b
    __shared__ int s_nzc[NSP * NCP];         // per m_P: the Cartesian components with a nonzero weight
    __shared__ double s_nzw[NSP * NCP];      // ... and the weights
    __shared__ int s_nnz[NSP];
    __shared__ int s_tp[SH::SPB * TPR];      // primitive pair of each table of the round, -1 past the end
    __shared__ double red[kGradCenterThreads / 32 * 12];
    const PairTask task = tasks[blockIdx.x];
    const int ia_shell = task.swap ? task.second : task.first;
    const int ib_shell = task.swap ? task.first : task.second;
    const int npp = npps[blockIdx.x];
    if (npp == 0) return;  // the same for the whole CTA: nothing survives screening
    const double* __restrict__ pd = pdata + offsets[blockIdx.x];

    for (int e = threadIdx.x; e < NCP * NH1; e += blockDim.x) {
        const int c = e / NH1, h = e - c * NH1;
        s_idx1[e] = tet(c_tet_t[h] + c_cart[LP][c][0], c_tet_u[h] + c_cart[LP][c][1], c_tet_v[h] + c_cart[LP][c][2]);
    }
    for (int e = threadIdx.x; e < NCP * NH * 3; e += blockDim.x) {
        const int c = e / (NH * 3), r = e - c * NH * 3, h = r / 3, d = r - h * 3;
        s_idx3[e] = tet(c_tet_t[h] + c_cart[LP][c][0] + (d == 0), c_tet_u[h] + c_cart[LP][c][1] + (d == 1),
                        c_tet_v[h] + c_cart[LP][c][2] + (d == 2));
    }
    if (threadIdx.x < NSP) {
        int k = 0;
        for (int c = 0; c < NCP; ++c) {
            const double w = c_c2s[c2s_offset(LP) + threadIdx.x * NCP + c];
            if (w != 0.0) {
                s_nzc[threadIdx.x * NCP + k] = c;
                s_nzw[threadIdx.x * NCP + k] = w;
                ++k;
            }
        }
        s_nnz[threadIdx.x] = k;
    }
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wslot = lane / NSP, mp = lane - wslot * NSP;
    const int slot = warp * SPW + wslot;
    const int ia = blockIdx.y * SH::SPB + slot;
    const bool active = wslot < SPW && ia < nalist;
    const double fac = task.first == task.second ? 1.0 : 2.0;
    // per-thread sums for the two orbital centres: A_J[3] A_K[3] B_J[3] B_K[3]
    // (J parts with the factor c_P applied)
    double v[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) v[k] = 0.0;
    // acc: Q_J[3] Q_K[3] A_J[3] A_K[3] (J parts without the factor c_P)
    double acc[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) acc[k] = 0.0;
    DevShell P{};
    int pshell = 0, ntrip = 0;
    double cP = 0.0;
    double gk[PL::KK][PL::NSAB];
    if (active) {
        pshell = alist[ia];
        P = aux[pshell];
        ntrip = P.nprim * npp;
        const int pf = P.fn + mp;
        cP = g.cfit[pf];
        const DevShell A = orb[ia_shell];
        const DevShell B = orb[ib_shell];
#pragma unroll
        for (int ka = 0; ka < PL::KA; ++ka)
#pragma unroll
            for (int kb = 0; kb < PL::KB; ++kb)
#pragma unroll
                for (int ma = 0; ma < PL::NSA; ++ma)
#pragma unroll
                    for (int mb = 0; mb < PL::NSB; ++mb) {
                        double val = 0.0;
                        if (ka < A.ncontr && kb < B.ncontr) {
                            const int64_t mu = A.fn + ka * PL::NSA + ma, nu = B.fn + kb * PL::NSB + mb;
                            val = g.GK[(mu * g.n + nu) * g.Pb + (pf - g.P0)];
                        }
                        gk[ka * PL::KB + kb][ma * PL::NSB + mb] = val;
                    }
    } else {
#pragma unroll
        for (int k = 0; k < PL::KK; ++k)
#pragma unroll
            for (int m = 0; m < PL::NSAB; ++m) gk[k][m] = 0.0;
    }
    // rounds of this warp: its slowest shell's triples over TPR
    const int rounds = __reduce_max_sync(0xffffffffu, (ntrip + TPR - 1) / TPR);
    const int nnz = s_nnz[active ? mp : 0];
    const int* __restrict__ nzc = s_nzc + (active ? mp : 0) * NCP;
    const double* __restrict__ nzw = s_nzw + (active ? mp : 0) * NCP;

    // this thread's triple t = r TPR + mp as (auxiliary primitive i, primitive pair pp),
    // advanced by TPR per round; the auxiliary primitive's factors are kept while i stays
    int ti = mp / npp, tpp = mp - (mp / npp) * npp;
    int ci = -1;
    double q = 0.0, cq = 0.0;
    for (int r = 0; r < rounds; ++r) {
        if (active && mp < TPR) {
            int pp = -1;
            if (ti < P.nprim) {
                pp = tpp;
                if (ti != ci) {
                    ci = ti;
                    q = exps[P.prim + ti];
                    // c_P (2q)^-l_P (-1)^l_P
                    const double h2q = 0.5 / q;
                    cq = coefs[P.coef + ti];
#pragma unroll
                    for (int k = 0; k < LP; ++k) cq *= h2q;
                    if (LP & 1) cq = -cq;
                }
                const double* s = pd + (int64_t)pp * PL::STRIDE;
                const double p = s[0];
                const double inv_pq = 1.0 / (p + q);
                const double alpha = p * q * inv_pq;
                double* row = sR + (slot * TPR + mp) * RS;
                if constexpr (L <= 4) {
                    double Rr[NR];
                    hermite_r<L>(alpha, s[1] - P.x, s[2] - P.y, s[3] - P.z, btable, Rr);
#pragma unroll
                    for (int e = 0; e < NR; ++e) row[e] = Rr[e];
                } else {
                    hermite_r<L>(alpha, s[1] - P.x, s[2] - P.y, s[3] - P.z, btable, row);
                }
                // 2 pi^(5/2) / (p q sqrt(p + q)) c_P (2q)^-l_P (-1)^l_P
                row[NR] = kTwoPi52 * sqrt(inv_pq) / (p * q) * cq;
                tpp += TPR;
                while (tpp >= npp) {
                    tpp -= npp;
                    ++ti;
                }
            }
            s_tp[slot * TPR + mp] = pp;
        }
        __syncwarp();
        if (active) {
#pragma unroll 1
            for (int j = 0; j < TPR; ++j) {
                const int pj = s_tp[slot * TPR + j];
                if (pj < 0) break;
                const double* row = sR + (slot * TPR + j) * RS;
                const double pref = row[NR];
                const double* s = pd + (int64_t)pj * PL::STRIDE;
                // exchange weight of this primitive pair: w[m] = sum_k cc[k] gk[k][m]
                double w[PL::NSAB];
#pragma unroll
                for (int m = 0; m < PL::NSAB; ++m) {
                    double x = 0.0;
#pragma unroll
                    for (int k = 0; k < PL::KK; ++k) x += s[4 + k] * gk[k][m];
                    w[m] = x;
                }
                const double* et = s + PL::OFF_E;
                const double* ea = s + PL::OFF_EA;
                const double* ej = s + PL::OFF_EJ;
                const double* eja = s + PL::OFF_EJA;
                // auxiliary centre: -sum_c w_c R[h + c + e_d], formed as it is used
#pragma unroll 1
                for (int h = 0; h < NH; ++h) {
                    double gx = 0.0, gy = 0.0, gz = 0.0;
#pragma unroll 1
                    for (int k = 0; k < nnz; ++k) {
                        const int* ix = s_idx3 + (nzc[k] * NH + h) * 3;
                        const double wc = nzw[k];
                        gx += wc * row[ix[0]];
                        gy += wc * row[ix[1]];
                        gz += wc * row[ix[2]];
                    }
                    double wk = 0.0;
#pragma unroll
                    for (int m = 0; m < PL::NSAB; ++m) wk += w[m] * et[m * NH + h];
                    const double wj = pref * ej[h];
                    wk *= pref;
                    acc[0] -= wj * gx;
                    acc[1] -= wj * gy;
                    acc[2] -= wj * gz;
                    acc[3] -= wk * gx;
                    acc[4] -= wk * gy;
                    acc[5] -= wk * gz;
                }
                // centre of the first orbital function: sum_c w_c R[h + c], h up to LAB + 1
#pragma unroll 1
                for (int h = 0; h < NH1; ++h) {
                    double g1 = 0.0;
#pragma unroll 1
                    for (int k = 0; k < nnz; ++k) g1 += nzw[k] * row[s_idx1[nzc[k] * NH1 + h]];
                    g1 *= pref;
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        double wk = 0.0;
#pragma unroll
                        for (int m = 0; m < PL::NSAB; ++m) wk += w[m] * ea[(d * PL::NSAB + m) * NH1 + h];
                        acc[6 + d] += eja[d * NH1 + h] * g1;
                        acc[9 + d] += wk * g1;
                    }
                }
            }
        }
        __syncwarp();
    }
    if (active) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            atomicAdd(gaux + (int64_t)pshell * 6 + d, fac * cP * acc[d]);
            atomicAdd(gaux + (int64_t)pshell * 6 + 3 + d, fac * acc[3 + d]);
            // first centre: A; second: B = -(Q + A)
            v[d] += cP * acc[6 + d];
            v[3 + d] += acc[9 + d];
            v[6 + d] -= cP * (acc[d] + acc[6 + d]);
            v[9 + d] -= acc[3 + d] + acc[9 + d];
        }
    }
    cta_sum12(v, red);
    if (threadIdx.x == 0) {
        for (int k = 0; k < 6; ++k) {
            atomicAdd(gorb + (int64_t)ia_shell * 6 + k, fac * red[k]);
            atomicAdd(gorb + (int64_t)ib_shell * 6 + k, fac * red[6 + k]);
        }
    }
}

template <int LA, int LB, int LP>
static cudaError_t three_center_grad_one(const PairTask* tasks, int ntasks, int max_npp, const DevShell* orb,
                                         const DevShell* aux, const double* exps, const double* coefs,
                                         const int* alist, int nalist, const double* btable, GradWeights g,
                                         GradPairData pd, double* gorb, double* gaux, cudaStream_t stream) {
    if (ntasks == 0 || nalist == 0) return cudaSuccess;
    using SH = GradCenterShape<LA, LB, LP>;
    (void)max_npp;  // the pair data is read from global memory
    const size_t smem = sizeof(double) * (size_t)SH::R_DOUBLES;
    // the attribute covers the dynamic part; the static tables count against
    // the 48 KB default too
    if (smem > 32 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_three_center_grad<LA, LB, LP>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    dim3 grid(ntasks, (nalist + SH::SPB - 1) / SH::SPB);
    k_three_center_grad<LA, LB, LP><<<grid, kGradCenterThreads, smem, stream>>>(
        tasks, orb, aux, exps, coefs, alist, nalist, btable, g, pd.offsets, pd.data, pd.npps, gorb, gaux);
    return cudaGetLastError();
}

cudaError_t launch_three_center_grad(int la, int lb, const PairTask* tasks, int ntasks, int max_npp,
                                     const DevShell* orb, const DevShell* aux, const double* exps,
                                     const double* coefs, const int* const* alist_by_l, const int* count_by_l,
                                     const double* btable, GradWeights g, GradPairData pd, double* gorb,
                                     double* gaux, cudaStream_t stream) {
    cudaError_t e = cudaSuccess;
#define HF_3CG(LA, LB, LP)                                                                                        \
    if (e == cudaSuccess && la == LA && lb == LB)                                                                 \
        e = three_center_grad_one<LA, LB, LP>(tasks, ntasks, max_npp, orb, aux, exps, coefs, alist_by_l[LP],       \
                                              count_by_l[LP], btable, g, pd, gorb, gaux, stream);
#define HF_3CG_P(LA, LB) HF_3CG(LA, LB, 0) HF_3CG(LA, LB, 1) HF_3CG(LA, LB, 2) HF_3CG(LA, LB, 3) HF_3CG(LA, LB, 4)
    HF_3CG_P(0, 0)
    HF_3CG_P(0, 1)
    HF_3CG_P(0, 2)
    HF_3CG_P(1, 1)
    HF_3CG_P(1, 2)
    HF_3CG_P(2, 2)
#undef HF_3CG_P
#undef HF_3CG
    return e;
}

template <int LA, int LB>
static cudaError_t grad_pair_data_one(const PairTask* tasks, int ntasks, int max_npp, const DevShell* orb,
                                      const double* exps, const double* coefs, const double* D, int64_t n,
                                      GradPairData pd, cudaStream_t stream) {
    if (ntasks == 0) return cudaSuccess;
    const size_t smem = sizeof(double) * (size_t)max_npp * GradPairLayout<LA, LB>::STRIDE;
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    if (smem > 40 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_grad_pair_data<LA, LB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
    }
    k_grad_pair_data<LA, LB><<<ntasks, kGradThreads, smem, stream>>>(tasks, orb, exps, coefs, D, n, pd.offsets,
                                                                     pd.data, pd.npps);
    return cudaGetLastError();
}

cudaError_t launch_grad_pair_data(int la, int lb, const PairTask* tasks, int ntasks, int max_npp,
                                  const DevShell* orb, const double* exps, const double* coefs, const double* D,
                                  int64_t n, GradPairData pd, cudaStream_t stream) {
    cudaError_t e = cudaSuccess;
#define HF_GPD(LA, LB) \
    if (la == LA && lb == LB) e = grad_pair_data_one<LA, LB>(tasks, ntasks, max_npp, orb, exps, coefs, D, n, pd, stream);
    HF_GPD(0, 0) HF_GPD(0, 1) HF_GPD(0, 2) HF_GPD(1, 1) HF_GPD(1, 2) HF_GPD(2, 2)
#undef HF_GPD
    return e;
}

size_t three_center_grad_smem(int la, int lb, int max_npp) {
    int stride = 0;
#define HF_STRIDE(LA, LB) \
    if (la == LA && lb == LB) stride = GradPairLayout<LA, LB>::STRIDE;
    HF_STRIDE(0, 0) HF_STRIDE(0, 1) HF_STRIDE(0, 2) HF_STRIDE(1, 1) HF_STRIDE(1, 2) HF_STRIDE(2, 2)
#undef HF_STRIDE
    return sizeof(double) * (size_t)max_npp * stride;
}

// ------------------------------------------------------------ metric
// One warp per (auxiliary shell P of class LP, m_P); its lanes run over the
// shells Q of class LQ. 2 sum_Q (d_P P|Q) W_PQ into gaux[P shell] (Coulomb weight
// in slots 0..2, exchange in 3..5), the factor 2 adding the ket derivative of
// the symmetric metric (gradient.py:196-199).
template <int LP, int LQ>
__global__ void __launch_bounds__(128) k_metric_grad(const DevShell* __restrict__ aux, const double* __restrict__ exps,
                                                     const double* __restrict__ coefs, const int* __restrict__ plist,
                                                     int np, const int* __restrict__ qlist, int nq,
                                                     const double* __restrict__ btable, const double* __restrict__ WJ,
                                                     const double* __restrict__ WK, int64_t ldw,
                                                     double* __restrict__ gaux) {
    constexpr int L = LP + LQ + 1;
    constexpr int NCP = ncart(LP), NCQ = ncart(LQ), NSP = nsph(LP), NSQ = nsph(LQ);
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= (int64_t)np * NSP) return;
    const int ip = (int)(warp / NSP), mp = (int)(warp % NSP);
    const int pshell = plist[ip];
    const DevShell P = aux[pshell];
    double crow[NCP];
#pragma unroll
    for (int c = 0; c < NCP; ++c) crow[c] = c_c2s[c2s_offset(LP) + mp * NCP + c];
    double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int iq = lane; iq < nq; iq += 32) {
        const DevShell Q = aux[qlist[iq]];
        const double X = P.x - Q.x, Y = P.y - Q.y, Z = P.z - Q.z;
        double val[3][NSQ];
#pragma unroll
        for (int d = 0; d < 3; ++d)
#pragma unroll
            for (int m = 0; m < NSQ; ++m) val[d][m] = 0.0;
        for (int i = 0; i < P.nprim; ++i) {
            const double p = exps[P.prim + i];
            const double cp = coefs[P.coef + i] * pow(2.0 * p, -(double)LP);
            for (int j = 0; j < Q.nprim; ++j) {
                const double q = exps[Q.prim + j];
                double cq = coefs[Q.coef + j] * pow(2.0 * q, -(double)LQ);
                if (LQ & 1) cq = -cq;
                const double alpha = p * q / (p + q);
                double R[ntet(L)];
                hermite_r<L>(alpha, X, Y, Z, btable, R);
                const double pref = kTwoPi52 / (p * q * sqrt(p + q)) * cp * cq;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    double h[NCQ];
#pragma unroll
                    for (int b = 0; b < NCQ; ++b) {
                        double s = 0.0;
#pragma unroll
                        for (int a = 0; a < NCP; ++a)
                            s += crow[a] * R[tet(cart_x(LP, a) + cart_x(LQ, b) + (d == 0),
                                                 cart_y(LP, a) + cart_y(LQ, b) + (d == 1),
                                                 cart_z(LP, a) + cart_z(LQ, b) + (d == 2))];
                        h[b] = s;
                    }
#pragma unroll
                    for (int m = 0; m < NSQ; ++m) {
                        double s = 0.0;
#pragma unroll
                        for (int b = 0; b < NCQ; ++b) s += c_c2s[c2s_offset(LQ) + m * NCQ + b] * h[b];
                        val[d][m] += pref * s;
                    }
                }
            }
        }
        const int64_t pr = P.fn + mp;
        const int64_t row = pr * ldw + Q.fn;
#pragma unroll
        for (int m = 0; m < NSQ; ++m) {
            // W^K is symmetric and only its upper triangle (row <= column) is formed
            const int64_t qc = Q.fn + m;
            const double wj = WJ[row + m], wk = pr <= qc ? WK[row + m] : WK[qc * ldw + pr];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                acc[d] += val[d][m] * wj;
                acc[3 + d] += val[d][m] * wk;
            }
        }
    }
#pragma unroll
    for (int k = 0; k < 6; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < 6; ++k) atomicAdd(gaux + (int64_t)pshell * 6 + k, 2.0 * acc[k]);
}

template <int LP, int LQ>
static cudaError_t metric_grad_one(const DevShell* aux, const double* exps, const double* coefs, const int* plist,
                                   int np, const int* qlist, int nq, const double* btable, const double* WJ,
                                   const double* WK, int64_t ldw, double* gaux, cudaStream_t stream) {
    if (np == 0 || nq == 0) return cudaSuccess;
    const int64_t threads = (int64_t)np * nsph(LP) * 32;
    k_metric_grad<LP, LQ><<<(unsigned)((threads + 127) / 128), 128, 0, stream>>>(aux, exps, coefs, plist, np, qlist,
                                                                                 nq, btable, WJ, WK, ldw, gaux);
    return cudaGetLastError();
}

cudaError_t launch_metric_grad(const DevShell* aux, const double* exps, const double* coefs,
                               const int* const* aux_by_l, const int* count, const double* btable, const double* WJ,
                               const double* WK, int64_t ldw, double* gaux, cudaStream_t stream) {
    cudaError_t e = cudaSuccess;
#define HF_MG(LP, LQ)                                                                                            \
    if (e == cudaSuccess)                                                                                        \
        e = metric_grad_one<LP, LQ>(aux, exps, coefs, aux_by_l[LP], count[LP], aux_by_l[LQ], count[LQ], btable, WJ, \
                                    WK, ldw, gaux, stream);
#define HF_MG_ROW(LP) HF_MG(LP, 0) HF_MG(LP, 1) HF_MG(LP, 2) HF_MG(LP, 3) HF_MG(LP, 4)
    HF_MG_ROW(0)
    HF_MG_ROW(1)
    HF_MG_ROW(2)
    HF_MG_ROW(3)
    HF_MG_ROW(4)
#undef HF_MG_ROW
#undef HF_MG
    return e;
}

// ------------------------------------------------------- one-electron terms
// Cartesian weights of the spherical density block of (A, B):
// out[k][ca][cb] = sum_{ma,mb} c2s_A[ma][ca] c2s_B[mb][cb] M[mu_k,ma][nu_k,mb].
template <int LA, int LB>
__device__ __forceinline__ void cartesian_weights(const DevShell& A, const DevShell& B, const double* __restrict__ M,
                                                  int64_t n, double (&out)[kMaxOrbContr[LA] * kMaxOrbContr[LB]]
                                                                          [ncart(LA)][ncart(LB)]) {
    constexpr int NCA = ncart(LA), NCB = ncart(LB), NSA = nsph(LA), NSB = nsph(LB);
    constexpr int KA = kMaxOrbContr[LA], KB = kMaxOrbContr[LB];
#pragma unroll
    for (int ka = 0; ka < KA; ++ka)
#pragma unroll
        for (int kb = 0; kb < KB; ++kb) {
            double sph[NSA][NSB];
#pragma unroll
            for (int ma = 0; ma < NSA; ++ma)
#pragma unroll
                for (int mb = 0; mb < NSB; ++mb)
                    sph[ma][mb] = (ka < A.ncontr && kb < B.ncontr)
                                      ? M[(int64_t)(A.fn + ka * NSA + ma) * n + B.fn + kb * NSB + mb]
                                      : 0.0;
#pragma unroll
            for (int ca = 0; ca < NCA; ++ca)
#pragma unroll
                for (int cb = 0; cb < NCB; ++cb) {
                    double v = 0.0;
#pragma unroll
                    for (int ma = 0; ma < NSA; ++ma) {
                        const double ta = c_c2s[c2s_offset(LA) + ma * NCA + ca];
                        if (ta == 0.0) continue;
#pragma unroll
                        for (int mb = 0; mb < NSB; ++mb) v += ta * c_c2s[c2s_offset(LB) + mb * NCB + cb] * sph[ma][mb];
                    }
                    out[ka * KB + kb][ca][cb] = v;
                }
        }
}

// One thread per ordered shell pair (A, B) of class (LA, LB): <d_A u|T + V|v>
// against D (slots 0..2, times 2 for the ket by symmetry) and -<d_A u|v> against
// W (slots 3..5, times -2) into gorb[A] (gradient.py:171-178, 119-124).
template <int LA, int LB>
__global__ void __launch_bounds__(128) k_one_electron_grad(const int2* __restrict__ tasks, int ntasks,
                                                           const DevShell* __restrict__ orb,
                                                           const double* __restrict__ exps,
                                                           const double* __restrict__ coefs,
                                                           const double* __restrict__ charges,
                                                           const double* __restrict__ positions, int natoms,
                                                           const double* __restrict__ btable,
                                                           const double* __restrict__ D, const double* __restrict__ W,
                                                           int64_t n, double* __restrict__ gorb) {
    constexpr int NCA = ncart(LA), NCB = ncart(LB);
    constexpr int KA = kMaxOrbContr[LA], KB = kMaxOrbContr[LB];
    constexpr int LAB = LA + LB;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntasks) return;
    const int2 task = tasks[t];
    const DevShell A = orb[task.x];
    const DevShell B = orb[task.y];
    double dc[KA * KB][NCA][NCB], wc[KA * KB][NCA][NCB];
    cartesian_weights<LA, LB>(A, B, D, n, dc);
    cartesian_weights<LA, LB>(A, B, W, n, wc);
    double g1[3] = {0.0, 0.0, 0.0}, gs[3] = {0.0, 0.0, 0.0};
    const double abx = A.x - B.x, aby = A.y - B.y, abz = A.z - B.z;
    const double rab2 = abx * abx + aby * aby + abz * abz;
    for (int i = 0; i < A.nprim; ++i)
        for (int j = 0; j < B.nprim; ++j) {
            const double a = exps[A.prim + i], b = exps[B.prim + j];
            const double p = a + b, mu = a * b / p;
            const double px = (a * A.x + b * B.x) / p, py = (a * A.y + b * B.y) / p, pz = (a * A.z + b * B.z) / p;
            Hermite1D<LA + 1, LB + 2> e[3];
            e[0].build(p, exp(-mu * rab2), px - A.x, px - B.x);
            e[1].build(p, 1.0, py - A.y, py - B.y);
            e[2].build(p, 1.0, pz - A.z, pz - B.z);
            double Rs[ntet(LAB + 1)];
#pragma unroll
            for (int h = 0; h < ntet(LAB + 1); ++h) Rs[h] = 0.0;
            for (int c = 0; c < natoms; ++c) {
                double R[ntet(LAB + 1)];
                hermite_r<LAB + 1>(p, px - positions[3 * c], py - positions[3 * c + 1], pz - positions[3 * c + 2],
                                   btable, R);
                const double z = charges[c];
#pragma unroll
                for (int h = 0; h < ntet(LAB + 1); ++h) Rs[h] -= z * R[h];
            }
            const double ov = pow(kPi / p, 1.5);
            const double vpref = 2.0 * kPi / p;
            // per-primitive density weights
            double cf[KA * KB];
#pragma unroll
            for (int ka = 0; ka < KA; ++ka)
#pragma unroll
                for (int kb = 0; kb < KB; ++kb)
                    cf[ka * KB + kb] = (ka < A.ncontr && kb < B.ncontr)
                                           ? coefs[A.coef + ka * A.nprim + i] * coefs[B.coef + kb * B.nprim + j]
                                           : 0.0;
#pragma unroll
            for (int ca = 0; ca < NCA; ++ca)
#pragma unroll
                for (int cb = 0; cb < NCB; ++cb) {
                    double wd = 0.0, ww = 0.0;
#pragma unroll
                    for (int k = 0; k < KA * KB; ++k) {
                        wd += cf[k] * dc[k][ca][cb];
                        ww += cf[k] * wc[k][ca][cb];
                    }
                    const int ii[3] = {cart_x(LA, ca), cart_y(LA, ca), cart_z(LA, ca)};
                    const int jj[3] = {cart_x(LB, cb), cart_y(LB, cb), cart_z(LB, cb)};
                    double s[3], ds[3], t2[3], dt2[3];
#pragma unroll
                    for (int x = 0; x < 3; ++x) {
                        const int i0 = ii[x], j0 = jj[x];
                        auto d2 = [&](int iq) {
                            double v = 4.0 * b * b * e[x].e[iq][j0 + 2][0] - 2.0 * b * (2 * j0 + 1) * e[x].e[iq][j0][0];
                            if (j0 >= 2) v += j0 * (j0 - 1) * e[x].e[iq][j0 - 2][0];
                            return v;
                        };
                        s[x] = e[x].e[i0][j0][0];
                        ds[x] = 2.0 * a * e[x].e[i0 + 1][j0][0] - (i0 > 0 ? i0 * e[x].e[i0 > 0 ? i0 - 1 : 0][j0][0] : 0.0);
                        t2[x] = d2(i0);
                        dt2[x] = 2.0 * a * d2(i0 + 1) - (i0 > 0 ? i0 * d2(i0 > 0 ? i0 - 1 : 0) : 0.0);
                    }
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        double f[3], tf[3];
#pragma unroll
                        for (int x = 0; x < 3; ++x) {
                            f[x] = x == d ? ds[x] : s[x];
                            tf[x] = x == d ? dt2[x] : t2[x];
                        }
                        const double dS = ov * f[0] * f[1] * f[2];
                        const double dT = -0.5 * ov * (tf[0] * f[1] * f[2] + f[0] * tf[1] * f[2] + f[0] * f[1] * tf[2]);
                        // attraction: the raised Hermite coefficients along d
                        double dV = 0.0;
#pragma unroll
                        for (int tt = 0; tt <= ii[0] + jj[0] + (d == 0); ++tt) {
                            const double fx = d == 0 ? 2.0 * a * e[0].e[ii[0] + 1][jj[0]][tt] -
                                                           (ii[0] > 0 ? ii[0] * e[0].e[ii[0] > 0 ? ii[0] - 1 : 0][jj[0]][tt] : 0.0)
                                                     : e[0].e[ii[0]][jj[0]][tt];
#pragma unroll
                            for (int u = 0; u <= ii[1] + jj[1] + (d == 1); ++u) {
                                const double fy = d == 1 ? 2.0 * a * e[1].e[ii[1] + 1][jj[1]][u] -
                                                               (ii[1] > 0 ? ii[1] * e[1].e[ii[1] > 0 ? ii[1] - 1 : 0][jj[1]][u] : 0.0)
                                                         : e[1].e[ii[1]][jj[1]][u];
#pragma unroll
                                for (int v = 0; v <= ii[2] + jj[2] + (d == 2); ++v) {
                                    const double fz = d == 2 ? 2.0 * a * e[2].e[ii[2] + 1][jj[2]][v] -
                                                                   (ii[2] > 0 ? ii[2] * e[2].e[ii[2] > 0 ? ii[2] - 1 : 0][jj[2]][v] : 0.0)
                                                             : e[2].e[ii[2]][jj[2]][v];
                                    dV += fx * fy * fz * Rs[tet(tt, u, v)];
                                }
                            }
                        }
                        dV *= vpref;
                        g1[d] += (dT + dV) * wd;
                        gs[d] += dS * ww;
                    }
                }
        }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        atomicAdd(gorb + (int64_t)task.x * 6 + d, 2.0 * g1[d]);
        atomicAdd(gorb + (int64_t)task.x * 6 + 3 + d, -2.0 * gs[d]);
    }
}

// Grid row C = blockIdx.y is one nucleus; one thread per ordered shell pair:
// sum_uv <u|d_C V_C|v> D_uv into gatom[C] (gradient.py:122-124), with
// d/dC R_tuv(P - C) = -R_{t+1,u,v}.
template <int LA, int LB>
__global__ void __launch_bounds__(128) k_attraction_nucleus_grad(const int2* __restrict__ tasks, int ntasks,
                                                                 const DevShell* __restrict__ orb,
                                                                 const double* __restrict__ exps,
                                                                 const double* __restrict__ coefs,
                                                                 const double* __restrict__ charges,
                                                                 const double* __restrict__ positions,
                                                                 const double* __restrict__ btable,
                                                                 const double* __restrict__ D, int64_t n,
                                                                 double* __restrict__ gatom) {
    constexpr int NCA = ncart(LA), NCB = ncart(LB);
    constexpr int KA = kMaxOrbContr[LA], KB = kMaxOrbContr[LB];
    constexpr int LAB = LA + LB;
    __shared__ double red[4 * 12];
    const int c = blockIdx.y;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) acc[k] = 0.0;
    if (t < ntasks) {
        const int2 task = tasks[t];
        const DevShell A = orb[task.x];
        const DevShell B = orb[task.y];
        double dc[KA * KB][NCA][NCB];
        cartesian_weights<LA, LB>(A, B, D, n, dc);
        const double abx = A.x - B.x, aby = A.y - B.y, abz = A.z - B.z;
        const double rab2 = abx * abx + aby * aby + abz * abz;
        const double cx = positions[3 * c], cy = positions[3 * c + 1], cz = positions[3 * c + 2];
        const double z = charges[c];
        for (int i = 0; i < A.nprim; ++i)
            for (int j = 0; j < B.nprim; ++j) {
                const double a = exps[A.prim + i], b = exps[B.prim + j];
                const double p = a + b, mu = a * b / p;
                const double px = (a * A.x + b * B.x) / p, py = (a * A.y + b * B.y) / p, pz = (a * A.z + b * B.z) / p;
                Hermite1D<LA, LB> ex, ey, ez;
                ex.build(p, exp(-mu * rab2), px - A.x, px - B.x);
                ey.build(p, 1.0, py - A.y, py - B.y);
                ez.build(p, 1.0, pz - A.z, pz - B.z);
                double R[ntet(LAB + 1)];
                hermite_r<LAB + 1>(p, px - cx, py - cy, pz - cz, btable, R);
                const double pref = z * 2.0 * kPi / p;
#pragma unroll
                for (int ca = 0; ca < NCA; ++ca)
#pragma unroll
                    for (int cb = 0; cb < NCB; ++cb) {
                        double wd = 0.0;
#pragma unroll
                        for (int ka = 0; ka < KA; ++ka)
#pragma unroll
                            for (int kb = 0; kb < KB; ++kb)
                                if (ka < A.ncontr && kb < B.ncontr)
                                    wd += coefs[A.coef + ka * A.nprim + i] * coefs[B.coef + kb * B.nprim + j] *
                                          dc[ka * KB + kb][ca][cb];
                        if (wd == 0.0) continue;
                        const int ix = cart_x(LA, ca), iy = cart_y(LA, ca), iz = cart_z(LA, ca);
                        const int jx = cart_x(LB, cb), jy = cart_y(LB, cb), jz = cart_z(LB, cb);
                        double sx = 0.0, sy = 0.0, sz = 0.0;
#pragma unroll
                        for (int tt = 0; tt <= ix + jx; ++tt)
#pragma unroll
                            for (int u = 0; u <= iy + jy; ++u)
#pragma unroll
                                for (int v = 0; v <= iz + jz; ++v) {
                                    const double w = ex.e[ix][jx][tt] * ey.e[iy][jy][u] * ez.e[iz][jz][v];
                                    sx += w * R[tet(tt + 1, u, v)];
                                    sy += w * R[tet(tt, u + 1, v)];
                                    sz += w * R[tet(tt, u, v + 1)];
                                }
                        acc[0] += pref * wd * sx;
                        acc[1] += pref * wd * sy;
                        acc[2] += pref * wd * sz;
                    }
            }
    }
    cta_sum12(acc, red);
    if (threadIdx.x == 0)
        for (int d = 0; d < 3; ++d) atomicAdd(gatom + 3 * c + d, red[d]);
}

template <int LA, int LB>
static cudaError_t one_electron_grad_one(const int2* tasks, int ntasks, const DevShell* orb, const double* exps,
                                         const double* coefs, const double* charges, const double* positions,
                                         int natoms, const double* btable, const double* D, const double* W, int64_t n,
                                         double* gorb, double* gatom, cudaStream_t stream) {
    if (ntasks == 0) return cudaSuccess;
    const unsigned blocks = (unsigned)((ntasks + 127) / 128);
    k_one_electron_grad<LA, LB><<<blocks, 128, 0, stream>>>(tasks, ntasks, orb, exps, coefs, charges, positions, natoms,
                                                            btable, D, W, n, gorb);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || natoms == 0) return e;
    k_attraction_nucleus_grad<LA, LB><<<dim3(blocks, natoms), 128, 0, stream>>>(tasks, ntasks, orb, exps, coefs, charges,
                                                                               positions, btable, D, n, gatom);
    return cudaGetLastError();
}

cudaError_t launch_one_electron_grad(int la, int lb, const int2* tasks, int ntasks, const DevShell* orb,
                                     const double* exps, const double* coefs, const double* charges,
                                     const double* positions, int natoms, const double* btable, const double* D,
                                     const double* W, int64_t n, double* gorb, double* gatom, cudaStream_t stream) {
    cudaError_t e = cudaSuccess;
#define HF_1EG(LA, LB)                                                                                        \
    if (la == LA && lb == LB)                                                                                 \
        e = one_electron_grad_one<LA, LB>(tasks, ntasks, orb, exps, coefs, charges, positions, natoms, btable, D, W, \
                                          n, gorb, gatom, stream);
    HF_1EG(0, 0) HF_1EG(0, 1) HF_1EG(0, 2) HF_1EG(1, 0) HF_1EG(1, 1) HF_1EG(1, 2) HF_1EG(2, 0) HF_1EG(2, 1)
    HF_1EG(2, 2)
#undef HF_1EG
    return e;
}

}  // namespace hf
