// Exact four-centre integrals (ab|cd) for small systems: the spherical atoms of
// the superposition-of-atomic-densities guess (hafnium/scf/atoms.py:55-73, which
// builds an ExactCoulombExchange from the Rust coulomb_four_center,
// two_electron.rs:429-935). One thread per shell quartet, generic in l with
// runtime loops: these problems have a handful of shells, so simplicity wins
// over speed. The quartet contraction is Helgaker 9.9.33 with the prefactor
// 2 pi^(5/2) / (p q sqrt(p+q)) (two_electron.rs:1398-1531).
//
// Included by integrals.cu, whose __constant__ tables it shares.
#pragma once

namespace hf {

namespace {

constexpr int kL = kMaxOrbL;  // per shell
constexpr int kNT = 2 * kL + 1;

// 1D Hermite expansion E[i][j][t], i, j <= 2, runtime l.
struct E1 {
    double e[kL + 1][kL + 1][kNT];
    __device__ void build(int la, int lb, double p, double e00, double xpa, double xpb) {
        const double h = 0.5 / p;
        for (int i = 0; i <= kL; ++i)
            for (int j = 0; j <= kL; ++j)
                for (int t = 0; t < kNT; ++t) e[i][j][t] = 0.0;
        e[0][0][0] = e00;
        for (int i = 0; i < la; ++i)
            for (int t = 0; t <= i + 1; ++t)
                e[i + 1][0][t] = (t > 0 ? h * e[i][0][t - 1] : 0.0) + xpa * (t <= i ? e[i][0][t] : 0.0) +
                                 (t + 1 <= i ? (t + 1) * e[i][0][t + 1] : 0.0);
        for (int i = 0; i <= la; ++i)
            for (int j = 0; j < lb; ++j)
                for (int t = 0; t <= i + j + 1; ++t)
                    e[i][j + 1][t] = (t > 0 ? h * e[i][j][t - 1] : 0.0) + xpb * (t <= i + j ? e[i][j][t] : 0.0) +
                                     (t + 1 <= i + j ? (t + 1) * e[i][j][t + 1] : 0.0);
    }
};

// R^0_tuv for t+u+v <= L (runtime L <= 8), same in-place recursion as md.cuh.
__device__ void hermite_r_rt(int L, double alpha, double X, double Y, double Z, const double* btable, double* R) {
    double F[9];
    boys<8>(alpha * (X * X + Y * Y + Z * Z), btable, F);
    const double m2a = -2.0 * alpha;
    double pw = 1.0;
    for (int k = 0; k < L; ++k) pw *= m2a;
    R[0] = pw * F[L];
    for (int n = L - 1; n >= 0; --n) {
        pw /= m2a;
        for (int s = L - n; s >= 1; --s)
            for (int t = s; t >= 0; --t) {
                const int r = s - t;
                for (int v = 0; v <= r; ++v) {
                    const int u = r - v;
                    double val;
                    if (t > 0) {
                        val = X * R[tet(t - 1, u, v)];
                        if (t > 1) val += (t - 1) * R[tet(t - 2, u, v)];
                    } else if (u > 0) {
                        val = Y * R[tet(t, u - 1, v)];
                        if (u > 1) val += (u - 1) * R[tet(t, u - 2, v)];
                    } else {
                        val = Z * R[tet(t, u, v - 1)];
                        if (v > 1) val += (v - 1) * R[tet(t, u, v - 2)];
                    }
                    R[tet(t, u, v)] = val;
                }
            }
        R[0] = pw * F[n];
    }
}

__global__ void __launch_bounds__(64) k_four_center(const DevShell* __restrict__ sh, int ns,
                                                    const double* __restrict__ exps, const double* __restrict__ coefs,
                                                    const double* __restrict__ btable, double* __restrict__ out, int n) {
    const int64_t qid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (qid >= (int64_t)ns * ns * ns * ns) return;
    const int a = (int)(qid / ((int64_t)ns * ns * ns)), b = (int)((qid / (ns * ns)) % ns), c = (int)((qid / ns) % ns),
              d = (int)(qid % ns);
    const DevShell S[4] = {sh[a], sh[b], sh[c], sh[d]};
    int nc[4], ns4[4];
    for (int k = 0; k < 4; ++k) {
        nc[k] = ncart(S[k].l);
        ns4[k] = nsph(S[k].l);
    }
    // Cartesian block [ka][ca][kb][cb][kc][cc][kd][cd], at most 6^4 * (contractions) values.
    double block[1296];
    const int dims[4] = {S[0].ncontr * nc[0], S[1].ncontr * nc[1], S[2].ncontr * nc[2], S[3].ncontr * nc[3]};
    const int total = dims[0] * dims[1] * dims[2] * dims[3];
    for (int i = 0; i < total; ++i) block[i] = 0.0;
    const int Lab = S[0].l + S[1].l, Lcd = S[2].l + S[3].l, L = Lab + Lcd;
    double R[ntet(8)];
    double X[36 * 35];  // [cc*cd][tuv <= Lab]
    for (int i = 0; i < S[0].nprim; ++i)
        for (int j = 0; j < S[1].nprim; ++j) {
            const double ea = exps[S[0].prim + i], eb = exps[S[1].prim + j];
            const double p = ea + eb, mu = ea * eb / p;
            const double P[3] = {(ea * S[0].x + eb * S[1].x) / p, (ea * S[0].y + eb * S[1].y) / p,
                                 (ea * S[0].z + eb * S[1].z) / p};
            const double ab[3] = {S[0].x - S[1].x, S[0].y - S[1].y, S[0].z - S[1].z};
            E1 Eab[3];
            Eab[0].build(S[0].l, S[1].l, p, exp(-mu * ab[0] * ab[0]), P[0] - S[0].x, P[0] - S[1].x);
            Eab[1].build(S[0].l, S[1].l, p, exp(-mu * ab[1] * ab[1]), P[1] - S[0].y, P[1] - S[1].y);
            Eab[2].build(S[0].l, S[1].l, p, exp(-mu * ab[2] * ab[2]), P[2] - S[0].z, P[2] - S[1].z);
            for (int k = 0; k < S[2].nprim; ++k)
                for (int l = 0; l < S[3].nprim; ++l) {
                    const double ec = exps[S[2].prim + k], ed = exps[S[3].prim + l];
                    const double q = ec + ed, nu = ec * ed / q;
                    const double Q[3] = {(ec * S[2].x + ed * S[3].x) / q, (ec * S[2].y + ed * S[3].y) / q,
                                         (ec * S[2].z + ed * S[3].z) / q};
                    const double cd[3] = {S[2].x - S[3].x, S[2].y - S[3].y, S[2].z - S[3].z};
                    E1 Ecd[3];
                    Ecd[0].build(S[2].l, S[3].l, q, exp(-nu * cd[0] * cd[0]), Q[0] - S[2].x, Q[0] - S[3].x);
                    Ecd[1].build(S[2].l, S[3].l, q, exp(-nu * cd[1] * cd[1]), Q[1] - S[2].y, Q[1] - S[3].y);
                    Ecd[2].build(S[2].l, S[3].l, q, exp(-nu * cd[2] * cd[2]), Q[2] - S[2].z, Q[2] - S[3].z);
                    const double alpha = p * q / (p + q);
                    hermite_r_rt(L, alpha, P[0] - Q[0], P[1] - Q[1], P[2] - Q[2], btable, R);
                    const double pref = 34.98683665524972 / (p * q * sqrt(p + q));
                    // X[cd][tuv] = sum (-1)^(tau+nu+phi) E^cd R_{t+tau,...}
                    for (int ic = 0; ic < nc[2]; ++ic)
                        for (int id = 0; id < nc[3]; ++id) {
                            const int* c1 = c_cart[S[2].l][ic];
                            const int* d1 = c_cart[S[3].l][id];
                            for (int h = 0; h < ntet(Lab); ++h) {
                                const int t = c_tet_t[h], u = c_tet_u[h], v = c_tet_v[h];
                                double s = 0.0;
                                for (int tau = 0; tau <= c1[0] + d1[0]; ++tau)
                                    for (int nn = 0; nn <= c1[1] + d1[1]; ++nn)
                                        for (int ph = 0; ph <= c1[2] + d1[2]; ++ph) {
                                            const double sg = ((tau + nn + ph) & 1) ? -1.0 : 1.0;
                                            s += sg * Ecd[0].e[c1[0]][d1[0]][tau] * Ecd[1].e[c1[1]][d1[1]][nn] *
                                                 Ecd[2].e[c1[2]][d1[2]][ph] * R[tet(t + tau, u + nn, v + ph)];
                                        }
                                X[(ic * nc[3] + id) * 35 + h] = s;
                            }
                        }
                    for (int ia = 0; ia < nc[0]; ++ia)
                        for (int jb = 0; jb < nc[1]; ++jb) {
                            const int* a1 = c_cart[S[0].l][ia];
                            const int* b1 = c_cart[S[1].l][jb];
                            for (int icd = 0; icd < nc[2] * nc[3]; ++icd) {
                                double v = 0.0;
                                for (int t = 0; t <= a1[0] + b1[0]; ++t)
                                    for (int u = 0; u <= a1[1] + b1[1]; ++u)
                                        for (int w = 0; w <= a1[2] + b1[2]; ++w)
                                            v += Eab[0].e[a1[0]][b1[0]][t] * Eab[1].e[a1[1]][b1[1]][u] *
                                                 Eab[2].e[a1[2]][b1[2]][w] * X[icd * 35 + tet(t, u, w)];
                                v *= pref;
                                const int ic = icd / nc[3], id = icd % nc[3];
                                for (int ka = 0; ka < S[0].ncontr; ++ka)
                                    for (int kb = 0; kb < S[1].ncontr; ++kb)
                                        for (int kc = 0; kc < S[2].ncontr; ++kc)
                                            for (int kd = 0; kd < S[3].ncontr; ++kd) {
                                                const double cf = coefs[S[0].coef + ka * S[0].nprim + i] *
                                                                  coefs[S[1].coef + kb * S[1].nprim + j] *
                                                                  coefs[S[2].coef + kc * S[2].nprim + k] *
                                                                  coefs[S[3].coef + kd * S[3].nprim + l];
                                                const int r0 = ka * nc[0] + ia, r1 = kb * nc[1] + jb,
                                                          r2 = kc * nc[2] + ic, r3 = kd * nc[3] + id;
                                                block[((r0 * dims[1] + r1) * dims[2] + r2) * dims[3] + r3] += cf * v;
                                            }
                            }
                        }
                }
        }
    // spherical transform of each index, then write (ab|cd) in AO order
    for (int k0 = 0; k0 < S[0].ncontr; ++k0)
        for (int m0 = 0; m0 < ns4[0]; ++m0)
            for (int k1 = 0; k1 < S[1].ncontr; ++k1)
                for (int m1 = 0; m1 < ns4[1]; ++m1)
                    for (int k2 = 0; k2 < S[2].ncontr; ++k2)
                        for (int m2 = 0; m2 < ns4[2]; ++m2)
                            for (int k3 = 0; k3 < S[3].ncontr; ++k3)
                                for (int m3 = 0; m3 < ns4[3]; ++m3) {
                                    double v = 0.0;
                                    for (int c0 = 0; c0 < nc[0]; ++c0) {
                                        const double t0 = c_c2s[c2s_offset(S[0].l) + m0 * nc[0] + c0];
                                        if (t0 == 0.0) continue;
                                        for (int c1 = 0; c1 < nc[1]; ++c1) {
                                            const double t1 = t0 * c_c2s[c2s_offset(S[1].l) + m1 * nc[1] + c1];
                                            if (t1 == 0.0) continue;
                                            for (int c2 = 0; c2 < nc[2]; ++c2) {
                                                const double t2 = t1 * c_c2s[c2s_offset(S[2].l) + m2 * nc[2] + c2];
                                                if (t2 == 0.0) continue;
                                                for (int c3 = 0; c3 < nc[3]; ++c3) {
                                                    const double t3 = c_c2s[c2s_offset(S[3].l) + m3 * nc[3] + c3];
                                                    const int r0 = k0 * nc[0] + c0, r1 = k1 * nc[1] + c1,
                                                              r2 = k2 * nc[2] + c2, r3 = k3 * nc[3] + c3;
                                                    v += t2 * t3 * block[((r0 * dims[1] + r1) * dims[2] + r2) * dims[3] + r3];
                                                }
                                            }
                                        }
                                    }
                                    const int64_t i0 = S[0].fn + k0 * ns4[0] + m0, i1 = S[1].fn + k1 * ns4[1] + m1,
                                                  i2 = S[2].fn + k2 * ns4[2] + m2, i3 = S[3].fn + k3 * ns4[3] + m3;
                                    out[((i0 * n + i1) * n + i2) * n + i3] = v;
                                }
}

}  // namespace

cudaError_t launch_four_center(const DevShell* shells, int ns, const double* exps, const double* coefs,
                               const double* btable, double* out, int n, cudaStream_t stream) {
    const int64_t total = (int64_t)ns * ns * ns * ns;
    if (total == 0) return cudaSuccess;
    k_four_center<<<(unsigned)((total + 63) / 64), 64, 0, stream>>>(shells, ns, exps, coefs, btable, out, n);
    return cudaGetLastError();
}

}  // namespace hf
