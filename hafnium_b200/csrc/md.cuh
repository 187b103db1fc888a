// Device McMurchie–Davidson building blocks, FP64 throughout.
//
// Boys function: Taylor expansion about the nearest point of a 0.05-spaced grid
// on [0, 36) (8 terms, |dT| <= 0.025, truncation below 4e-18 relative), then the
// downward recursion F_{n-1} = (2T F_n + e^{-T}) / (2n - 1); above the grid,
// F_0 = sqrt(pi/T)/2 and the upward recursion, as the reference's special.rs:34-51
// does above max(35, 2n). The grid values come from the reference's series
// (special.rs:67-81) evaluated on the host.
//
// Hermite Coulomb integrals R_tuv (coulomb.rs:162-215): the downward recursion
// in n is done in place in one tetrahedral array, updating total orders from
// the highest down, so R^{n+1} values are still present when R^n needs them.
//
// Spherical functions use the sphere-normalised real solid harmonics of
// cartesian.rs:93-110 (p ordered x, y, z). An auxiliary primitive
// S_lm(r) exp(-q r^2) expands into Hermite Gaussians of degree exactly l with
// coefficients (2q)^-l times the Cartesian coefficients of S_lm (Hobson's
// theorem), so its side of the contraction needs no E-coefficients.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace hf {

constexpr int kMaxOrbL = 2;   // cc-pVDZ / def2-SVP / STO-3G for H-Ne
constexpr int kMaxAuxL = 4;   // def2-universal-jkfit for H-Ne
constexpr int kMaxOrbContr[3] = {3, 2, 1};  // general contractions per l (cc-pVDZ O)
constexpr int kBoysTerms = 8;
// one order more than the integrals need, for their first derivatives
constexpr int kBoysOrders = 2 * kMaxOrbL + kMaxAuxL + 1 + kBoysTerms;  // 17
constexpr double kBoysStep = 0.05;
constexpr double kBoysTmax = 36.0;
constexpr int kBoysGrid = 721;  // T = 0 .. 36 inclusive

__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }
__host__ __device__ constexpr int nsph(int l) { return 2 * l + 1; }
// Number of (t,u,v) with t+u+v <= L.
__host__ __device__ constexpr int ntet(int L) { return (L + 1) * (L + 2) * (L + 3) / 6; }
// Tetrahedral index of (t,u,v): shells of total order s, then u+v, then v.
__host__ __device__ constexpr int tet(int t, int u, int v) {
    return (t + u + v) * (t + u + v + 1) * (t + u + v + 2) / 6 + (u + v) * (u + v + 1) / 2 + v;
}
// Cartesian component c of angular momentum l (x^l first, z^l last): exponents.
__host__ __device__ constexpr int cart_x(int l, int c) {
    int i = l, k = 0;
    for (; i >= 0; --i) {
        if (c < k + (l - i + 1)) return i;
        k += l - i + 1;
    }
    return 0;
}
__host__ __device__ constexpr int cart_y(int l, int c) {
    int i = l, k = 0;
    for (; i >= 0; --i) {
        if (c < k + (l - i + 1)) return (l - i) - (c - k);
        k += l - i + 1;
    }
    return 0;
}
__host__ __device__ constexpr int cart_z(int l, int c) { return l - cart_x(l, c) - cart_y(l, c); }

// Cartesian-to-spherical matrices for l = 0..4, row-major [2l+1][ncart(l)],
// concatenated; offsets c2s_offset(l).
__host__ __device__ constexpr int c2s_offset(int l) {
    int o = 0;
    for (int k = 0; k < l; ++k) o += nsph(k) * ncart(k);
    return o;
}
constexpr int kC2sSize = 1 + 9 + 30 + 70 + 135;

// Primitive pairs whose |c_a c_b| exp(-mu R_AB^2) falls below this contribute
// less than ~1e-15 to any (P|ab) and are skipped (the reference evaluates every
// primitive triple; the difference is far below its 1e-12 integral tolerance).
constexpr double kPairScreen = 1e-22;
constexpr int kMaxPrimPairs = 256;
constexpr double kPi = 3.14159265358979323846;
constexpr double kTwoPi52 = 34.98683665524972;  // 2 pi^(5/2)
// The matrices live in __constant__ memory of the translation unit that uses them.

// F_0..F_L at T. `table` is [kBoysGrid][kBoysOrders].
template <int L>
__device__ __forceinline__ void boys(double T, const double* __restrict__ table, double* F) {
    const double et = exp(-T);
    if (T < kBoysTmax) {
        const int j = __double2int_rn(T * (1.0 / kBoysStep));
        const double d = j * kBoysStep - T;  // T0 - T
        const double* row = table + j * kBoysOrders + L;
        // F_L(T) = sum_k F_{L+k}(T0) (T0 - T)^k / k!
        double v = __ldg(row + kBoysTerms - 1);
#pragma unroll
        for (int k = kBoysTerms - 1; k >= 1; --k) v = __ldg(row + k - 1) + v * d / k;
        F[L] = v;
#pragma unroll
        for (int n = L; n >= 1; --n) F[n - 1] = (2.0 * T * F[n] + et) / (2 * n - 1);
    } else {
        F[0] = 0.5 * sqrt(3.14159265358979323846 / T);
        const double inv2T = 0.5 / T;
#pragma unroll
        for (int n = 0; n < L; ++n) F[n + 1] = ((2 * n + 1) * F[n] - et) * inv2T;
    }
}

// R^0_tuv(alpha, X, Y, Z) for t+u+v <= L into R[tet(t,u,v)]. Up to L = 4 the
// recursion is unrolled so the table stays in registers; above, the loops are
// left rolled (the table lives in L1-resident local memory), which keeps the
// kernels compact and their compile time short.
template <int L>
__device__ __forceinline__ void hermite_r(double alpha, double X, double Y, double Z,
                                          const double* __restrict__ btable, double* R) {
    double F[L + 1];
    boys<L>(alpha * (X * X + Y * Y + Z * Z), btable, F);
    const double m2a = -2.0 * alpha;
    double pw[L + 1];
    pw[0] = 1.0;
#pragma unroll
    for (int k = 1; k <= L; ++k) pw[k] = pw[k - 1] * m2a;
    R[0] = pw[L] * F[L];
    if constexpr (L <= 4) {
#pragma unroll
        for (int n = L - 1; n >= 0; --n) {
#pragma unroll
            for (int s = L - n; s >= 1; --s)
#pragma unroll
                for (int t = s; t >= 0; --t)
#pragma unroll
                    for (int v = 0; v <= s - t; ++v) {
                        const int u = s - t - v;
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
            R[0] = pw[n] * F[n];
        }
    } else {
#pragma unroll 1
        for (int n = L - 1; n >= 0; --n) {
#pragma unroll 1
            for (int s = L - n; s >= 1; --s) {
                const int idx = s * (s + 1) * (s + 2) / 6;  // tet(s, 0, 0)
#pragma unroll 1
                for (int t = s; t >= 0; --t) {
                    const int r = s - t;  // u + v
#pragma unroll 1
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
                        R[idx + r * (r + 1) / 2 + v] = val;
                    }
                }
            }
            R[0] = pw[n] * F[n];
        }
    }
}

// One axis of the Hermite expansion of a primitive pair: E[i][j][t] for i<=LA,
// j<=LB+X, t<=i+j (hermite.rs:23-61, Helgaker 9.5.6/9.5.7).
template <int LA, int LB>
struct Hermite1D {
    double e[LA + 1][LB + 1][LA + LB + 1];
    __device__ __forceinline__ void build(double p, double e00, double xpa, double xpb) {
        const double h = 0.5 / p;
#pragma unroll
        for (int i = 0; i <= LA; ++i)
#pragma unroll
            for (int j = 0; j <= LB; ++j)
#pragma unroll
                for (int t = 0; t <= LA + LB; ++t) e[i][j][t] = 0.0;
        e[0][0][0] = e00;
#pragma unroll
        for (int i = 0; i < LA; ++i)
#pragma unroll
            for (int t = 0; t <= i + 1; ++t)
                e[i + 1][0][t] = (t > 0 ? h * e[i][0][t - 1] : 0.0) + xpa * (t <= i ? e[i][0][t] : 0.0) +
                                 (t + 1 <= i ? (t + 1) * e[i][0][t + 1] : 0.0);
#pragma unroll
        for (int i = 0; i <= LA; ++i)
#pragma unroll
            for (int j = 0; j < LB; ++j)
#pragma unroll
                for (int t = 0; t <= i + j + 1; ++t)
                    e[i][j + 1][t] = (t > 0 ? h * e[i][j][t - 1] : 0.0) +
                                     xpb * (t <= i + j ? e[i][j][t] : 0.0) +
                                     (t + 1 <= i + j ? (t + 1) * e[i][j][t + 1] : 0.0);
    }
};

}  // namespace hf
