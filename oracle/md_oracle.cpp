// Oracle: a CPU restatement of the reference's McMurchie–Davidson integrals.
//
// TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and the CPU
// baseline leg of bench.py may load this library, and only as the checker.
//
// The reference implements these kernels in Rust (crates/hafnium-core), which
// cannot be compiled here. This file restates the same mathematics in C++17 with
// OpenMP, function by function:
//   Boys function          special.rs:34-81 (series below max(35, 2n), else erf and
//                          upward recursion; series stops at relative 1e-17)
//   Hermite E coefficients hermite.rs:23-61 (Helgaker 9.5.6/9.5.7 from exp(-mu X_AB^2))
//   primitive pairs        pairs.rs:206-269 (a lone auxiliary is a pair with a unit
//                          s partner of exponent zero)
//   Hermite Coulomb R_tuv  coulomb.rs:162-261 (downward recursion in n; erf/erfc
//                          range separation by the attenuated exponent)
//   cart -> spherical      cartesian.rs:23-31, 93-110, 165-228 (Helgaker 6.4.47,
//                          sphere-normalised; p ordered x, y, z)
//   (ab|cd) contraction    two_electron.rs:1398-1580 (prefactor 2 pi^(5/2)/(pq sqrt(p+q)))
//   2c / 3c / 4c drivers   two_electron.rs:74-130, 212-297, 429-935
//   S, T, V                one_electron.rs:40-190
// Output layouts follow the reference's PyO3 binding (crates/hafnium-py/src/lib.rs):
// [image, bra, ket], [image, aux, bra, ket], [image, a, b, c, d], and
// [image, bra_shell, ket_shell] for the Schwarz bounds.
//
// Screening thresholds of the 2c/3c/attraction kernels are accepted but every
// term is evaluated (the density-fitting path of the reference passes 0); the
// four-centre kernel applies the reference's shell-quartet Schwarz screening.

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr int kMaxL = 8;  // per shell; cc-pVDZ and def2-universal-jkfit need 4

enum Kernel : int { kFull = 0, kLongRange = 1, kShortRange = 2 };

struct ShellView {
    int l;
    double center[3];
    int nprim;
    const double* exps;
    int ncontr;
    const double* coefs;  // [ncontr][nprim]
    int first_function;
};

struct Table {
    std::vector<ShellView> shells;
    int nfunc = 0;
    int maxl = 0;
};

int n_cart(int l) { return (l + 1) * (l + 2) / 2; }

// ---------------------------------------------------------------- Boys function
void boys(int nmax, double t, double* out) {
    const double et = std::exp(-t);
    if (t < std::max(35.0, 2.0 * nmax)) {
        double term = 1.0 / (2 * nmax + 1);
        double sum = term;
        for (int i = 1;; ++i) {
            term *= 2.0 * t / (2 * nmax + 2 * i + 1);
            sum += term;
            if (term < sum * 1e-17) break;
        }
        out[nmax] = et * sum;
        for (int n = nmax; n >= 1; --n) out[n - 1] = (2.0 * t * out[n] + et) / (2 * n - 1);
    } else {
        out[0] = 0.5 * std::sqrt(kPi / t) * std::erf(std::sqrt(t));
        for (int n = 0; n < nmax; ++n) out[n + 1] = ((2 * n + 1) * out[n] - et) / (2.0 * t);
    }
}

// -------------------------------------------------------- cartesian components
// Components (i, j, k) of angular momentum l with x^l first and z^l last.
std::vector<std::array<int, 3>> cart_components(int l) {
    std::vector<std::array<int, 3>> c;
    for (int i = l; i >= 0; --i)
        for (int j = l - i; j >= 0; --j) c.push_back({i, j, l - i - j});
    return c;
}

double factorial(int n) {
    double v = 1.0;
    for (int k = 2; k <= n; ++k) v *= k;
    return v;
}
double binomial(int n, int k) {
    if (k < 0 || k > n) return 0.0;
    double v = 1.0;
    for (int i = 0; i < k; ++i) v = v * (n - i) / (i + 1);
    return std::round(v);
}

// Row-major [2l+1][n_cart(l)] matrix from Cartesian monomials to real solid
// harmonics normalised on the unit sphere (Helgaker 6.4.47 times sqrt((2l+1)/4pi)).
std::vector<double> sph_transform(int l) {
    auto comps = cart_components(l);
    const int nc = (int)comps.size();
    std::vector<double> m((2 * l + 1) * nc, 0.0);
    const double sphere = std::sqrt((2.0 * l + 1.0) / (4.0 * kPi));
    std::vector<int> ms;
    if (l == 1) ms = {1, -1, 0};
    else for (int mm = -l; mm <= l; ++mm) ms.push_back(mm);
    for (int row = 0; row < (int)ms.size(); ++row) {
        const int mval = ms[row];
        const int am = std::abs(mval);
        const bool neg = mval < 0;
        const double delta = (mval == 0) ? 2.0 : 1.0;
        const double norm = std::sqrt(2.0 * factorial(l + am) * factorial(l - am) / delta) /
                            (std::pow(2.0, am) * factorial(l));
        for (int t = 0; t <= (l - am) / 2; ++t)
            for (int u = 0; u <= t; ++u) {
                const int vmax = neg ? (am - 1) / 2 : am / 2;
                for (int vh = 0; vh <= vmax; ++vh) {
                    const int two_v = neg ? 2 * vh + 1 : 2 * vh;
                    if (two_v > am) continue;
                    const double sign = ((t + vh) % 2 == 0) ? 1.0 : -1.0;
                    const double coef = sign * std::pow(0.25, t) * binomial(l, t) *
                                        binomial(l - t, am + t) * binomial(t, u) *
                                        binomial(am, two_v);
                    const int py = 2 * u + two_v;
                    const int px = 2 * t + am - py;
                    const int pz = l - 2 * t - am;
                    for (int c = 0; c < nc; ++c)
                        if (comps[c][0] == px && comps[c][1] == py && comps[c][2] == pz)
                            m[row * nc + c] += sphere * norm * coef;
                }
            }
    }
    return m;
}

struct Transforms {
    std::vector<std::vector<double>> t;
    std::vector<std::vector<std::array<int, 3>>> comps;
    explicit Transforms(int maxl) {
        for (int l = 0; l <= maxl; ++l) {
            t.push_back(sph_transform(l));
            comps.push_back(cart_components(l));
        }
    }
};

// --------------------------------------------------------- Hermite expansions
// One axis of a primitive pair: E[i][j][t] for i <= imax, j <= jmax, t <= i + j.
struct Hermite1D {
    int imax, jmax, nt;
    std::vector<double> d;
    double get(int i, int j, int t) const {
        if (t < 0 || t > i + j) return 0.0;
        return d[(i * (jmax + 1) + j) * nt + t];
    }
    void build(int im, int jm, double p, double mu, double xab, double xpa, double xpb) {
        imax = im; jmax = jm; nt = im + jm + 1;
        d.assign((im + 1) * (jm + 1) * nt, 0.0);
        auto at = [&](int i, int j, int t) -> double& { return d[(i * (jmax + 1) + j) * nt + t]; };
        const double h = 0.5 / p;
        at(0, 0, 0) = std::exp(-mu * xab * xab);
        for (int i = 0; i < im; ++i)
            for (int t = 0; t <= i + 1; ++t)
                at(i + 1, 0, t) = h * get(i, 0, t - 1) + xpa * get(i, 0, t) + (t + 1) * get(i, 0, t + 1);
        for (int i = 0; i <= im; ++i)
            for (int j = 0; j < jm; ++j)
                for (int t = 0; t <= i + j + 1; ++t)
                    at(i, j + 1, t) = h * get(i, j, t - 1) + xpb * get(i, j, t) + (t + 1) * get(i, j, t + 1);
    }
};

struct PrimPair {
    double p, ea, eb;
    double P[3];
    Hermite1D e[3];
};

struct Pair {
    int la, lb, ka, kb;
    std::vector<PrimPair> prims;
    std::vector<double> coef;  // [pp][ka][kb]
};

// All primitive pairs of shells a (at ca) and b (at cb); extra raises the order
// of the expansion on the bra / ket side.
Pair make_pair(const ShellView& a, const double* ca, const ShellView& b, const double* cb,
               int extra_a = 0, int extra_b = 0) {
    Pair pr;
    pr.la = a.l; pr.lb = b.l; pr.ka = a.ncontr; pr.kb = b.ncontr;
    pr.prims.reserve(a.nprim * b.nprim);
    for (int i = 0; i < a.nprim; ++i)
        for (int j = 0; j < b.nprim; ++j) {
            PrimPair pp;
            pp.ea = a.exps[i]; pp.eb = b.exps[j];
            pp.p = pp.ea + pp.eb;
            const double mu = pp.ea * pp.eb / pp.p;
            for (int x = 0; x < 3; ++x) {
                pp.P[x] = (pp.ea * ca[x] + pp.eb * cb[x]) / pp.p;
                pp.e[x].build(a.l + extra_a, b.l + extra_b, pp.p, mu, ca[x] - cb[x], pp.P[x] - ca[x],
                              pp.P[x] - cb[x]);
            }
            pr.prims.push_back(std::move(pp));
            for (int ka = 0; ka < a.ncontr; ++ka)
                for (int kb = 0; kb < b.ncontr; ++kb)
                    pr.coef.push_back(a.coefs[ka * a.nprim + i] * b.coefs[kb * b.nprim + j]);
        }
    return pr;
}

const double kZeroExp = 0.0;
const double kUnitCoef = 1.0;
// A lone shell as a pair with a unit s partner of exponent zero at its centre.
Pair single_pair(const ShellView& a, const double* ca) {
    ShellView unit{0, {ca[0], ca[1], ca[2]}, 1, &kZeroExp, 1, &kUnitCoef, 0};
    return make_pair(a, ca, unit, ca);
}

// ------------------------------------------------------ Hermite Coulomb R_tuv
struct RWork {
    std::vector<double> boys, prev, cur, diff;
};

// R^0_tuv(alpha, pc) for t+u+v <= L, into out[(t*(L+1)+u)*(L+1)+v].
void hermite_r(int L, double alpha, const double* pc, RWork& w, double* out) {
    const int s1 = L + 1;
    const int size = s1 * s1 * s1;
    w.boys.resize(L + 1);
    w.prev.assign(size, 0.0);
    w.cur.assign(size, 0.0);
    const double r2 = pc[0] * pc[0] + pc[1] * pc[1] + pc[2] * pc[2];
    boys(L, alpha * r2, w.boys.data());
    auto idx = [&](int t, int u, int v) { return (t * s1 + u) * s1 + v; };
    double power = std::pow(-2.0 * alpha, L);
    for (int n = L; n >= 0; --n) {
        w.cur[0] = power * w.boys[n];
        for (int s = 1; s <= L - n; ++s)
            for (int t = 0; t <= s; ++t)
                for (int u = 0; u <= s - t; ++u) {
                    const int v = s - t - u;
                    double val;
                    if (t > 0)
                        val = pc[0] * w.prev[idx(t - 1, u, v)] + (t > 1 ? (t - 1) * w.prev[idx(t - 2, u, v)] : 0.0);
                    else if (u > 0)
                        val = pc[1] * w.prev[idx(t, u - 1, v)] + (u > 1 ? (u - 1) * w.prev[idx(t, u - 2, v)] : 0.0);
                    else
                        val = pc[2] * w.prev[idx(t, u, v - 1)] + (v > 1 ? (v - 1) * w.prev[idx(t, u, v - 2)] : 0.0);
                    w.cur[idx(t, u, v)] = val;
                }
        power /= -2.0 * alpha;
        std::swap(w.prev, w.cur);
    }
    std::memcpy(out, w.prev.data(), sizeof(double) * size);
}

void hermite_r_kernel(int L, double alpha, int kernel, double omega, const double* pc, RWork& w,
                      double* out) {
    const int s1 = L + 1;
    const int size = s1 * s1 * s1;
    if (kernel == kFull) {
        hermite_r(L, alpha, pc, w, out);
        return;
    }
    const double weak = alpha * omega * omega / (alpha + omega * omega);
    const double scale = std::sqrt(weak / alpha);
    if (kernel == kLongRange) {
        hermite_r(L, weak, pc, w, out);
        for (int i = 0; i < size; ++i) out[i] *= scale;
        return;
    }
    std::vector<double> full(size);
    hermite_r(L, alpha, pc, w, full.data());
    hermite_r(L, weak, pc, w, out);
    for (int i = 0; i < size; ++i) out[i] = full[i] - scale * out[i];
}

// ------------------------------------------------------ generic Coulomb block
// out[ka][ca][kb][cb][kc][cc][kd][cd] += (ab|cd) summed over primitive quartets.
void coulomb_block(const Pair& bra, const Pair& ket, const Transforms& tr, int kernel, double omega,
                   RWork& w, std::vector<double>& out) {
    const auto& ca = tr.comps[bra.la];
    const auto& cb = tr.comps[bra.lb];
    const auto& cc = tr.comps[ket.la];
    const auto& cd = tr.comps[ket.lb];
    const int na = (int)ca.size(), nb = (int)cb.size(), nc = (int)cc.size(), nd = (int)cd.size();
    const int Lb = bra.la + bra.lb, Lk = ket.la + ket.lb, L = Lb + Lk;
    const int s1 = L + 1;
    const int nt = Lb + 1;
    std::vector<double> R(s1 * s1 * s1);
    std::vector<double> X(nc * nd * nt * nt * nt);
    std::vector<double> val(na * nb * nc * nd);
    const int sc = ket.kb * nd, sb = ket.ka * nc * sc, sa = bra.kb * nb * sb;
    for (size_t ib = 0; ib < bra.prims.size(); ++ib) {
        const PrimPair& P = bra.prims[ib];
        for (size_t ik = 0; ik < ket.prims.size(); ++ik) {
            const PrimPair& Q = ket.prims[ik];
            const double p = P.p, q = Q.p;
            const double alpha = p * q / (p + q);
            const double pq[3] = {P.P[0] - Q.P[0], P.P[1] - Q.P[1], P.P[2] - Q.P[2]};
            hermite_r_kernel(L, alpha, kernel, omega, pq, w, R.data());
            auto r = [&](int t, int u, int v) { return R[(t * s1 + u) * s1 + v]; };
            // X[cd][tuv] = sum_{tau nu phi} (-1)^(tau+nu+phi) E^{cd}_{tau nu phi} R_{t+tau, u+nu, v+phi}
            for (int ic = 0; ic < nc; ++ic)
                for (int id = 0; id < nd; ++id) {
                    double* slot = &X[(ic * nd + id) * nt * nt * nt];
                    const auto& c1 = cc[ic];
                    const auto& d1 = cd[id];
                    for (int t = 0; t < nt; ++t)
                        for (int u = 0; u < nt - t; ++u)
                            for (int v = 0; v < nt - t - u; ++v) {
                                double sum = 0.0;
                                for (int tau = 0; tau <= c1[0] + d1[0]; ++tau) {
                                    const double ex = Q.e[0].get(c1[0], d1[0], tau);
                                    if (ex == 0.0) continue;
                                    for (int nu = 0; nu <= c1[1] + d1[1]; ++nu) {
                                        const double ey = ex * Q.e[1].get(c1[1], d1[1], nu);
                                        if (ey == 0.0) continue;
                                        for (int phi = 0; phi <= c1[2] + d1[2]; ++phi) {
                                            const double sign = ((tau + nu + phi) & 1) ? -1.0 : 1.0;
                                            sum += sign * ey * Q.e[2].get(c1[2], d1[2], phi) *
                                                   r(t + tau, u + nu, v + phi);
                                        }
                                    }
                                }
                                slot[(t * nt + u) * nt + v] = sum;
                            }
                }
            for (int ia = 0; ia < na; ++ia)
                for (int jb = 0; jb < nb; ++jb) {
                    const auto& a1 = ca[ia];
                    const auto& b1 = cb[jb];
                    for (int icd = 0; icd < nc * nd; ++icd) {
                        const double* slot = &X[icd * nt * nt * nt];
                        double v = 0.0;
                        for (int t = 0; t <= a1[0] + b1[0]; ++t) {
                            const double ex = P.e[0].get(a1[0], b1[0], t);
                            for (int u = 0; u <= a1[1] + b1[1]; ++u) {
                                const double ey = ex * P.e[1].get(a1[1], b1[1], u);
                                for (int vv = 0; vv <= a1[2] + b1[2]; ++vv)
                                    v += ey * P.e[2].get(a1[2], b1[2], vv) * slot[(t * nt + u) * nt + vv];
                            }
                        }
                        val[(ia * nb + jb) * nc * nd + icd] = v;
                    }
                }
            const double pref = 2.0 * std::pow(kPi, 2.5) / (p * q * std::sqrt(p + q));
            for (int ka = 0; ka < bra.ka; ++ka)
                for (int kb = 0; kb < bra.kb; ++kb) {
                    const double cbra = pref * bra.coef[(ib * bra.ka + ka) * bra.kb + kb];
                    for (int kc = 0; kc < ket.ka; ++kc)
                        for (int kd = 0; kd < ket.kb; ++kd) {
                            const double cf = cbra * ket.coef[(ik * ket.ka + kc) * ket.kb + kd];
                            if (cf == 0.0) continue;
                            const int base = ka * na * sa + kb * nb * sb + kc * nc * sc + kd * nd;
                            for (int ia = 0; ia < na; ++ia)
                                for (int jb = 0; jb < nb; ++jb)
                                    for (int ic = 0; ic < nc; ++ic) {
                                        double* o = &out[base + ia * sa + jb * sb + ic * sc];
                                        const double* s = &val[((ia * nb + jb) * nc + ic) * nd];
                                        for (int id = 0; id < nd; ++id) o[id] += cf * s[id];
                                    }
                        }
                }
        }
    }
}

// Transform a block with index layout [k0, c0, k1, c1, k2, c2, k3, c3] to spherical
// functions; ls[i] < 0 marks a unit partner (one component, untouched).
std::vector<double> to_spherical(const std::vector<double>& block, const int ls[4], const int ks[4],
                                 const Transforms& tr) {
    std::vector<double> cur = block, nxt;
    int shape[8];
    for (int i = 0; i < 4; ++i) {
        shape[2 * i] = ks[i];
        shape[2 * i + 1] = ls[i] >= 0 ? n_cart(ls[i]) : 1;
    }
    for (int i = 0; i < 4; ++i) {
        if (ls[i] < 0) continue;
        const int axis = 2 * i + 1;
        long left = 1, right = 1;
        for (int a = 0; a < axis; ++a) left *= shape[a];
        for (int a = axis + 1; a < 8; ++a) right *= shape[a];
        const int ncart = shape[axis];
        const int nsph = 2 * ls[i] + 1;
        const auto& T = tr.t[ls[i]];
        nxt.assign(left * nsph * right, 0.0);
        for (long l0 = 0; l0 < left; ++l0)
            for (int m = 0; m < nsph; ++m) {
                double* tgt = &nxt[(l0 * nsph + m) * right];
                for (int c = 0; c < ncart; ++c) {
                    const double wgt = T[m * ncart + c];
                    if (wgt == 0.0) continue;
                    const double* src = &cur[(l0 * ncart + c) * right];
                    for (long r = 0; r < right; ++r) tgt[r] += wgt * src[r];
                }
            }
        std::swap(cur, nxt);
        shape[axis] = nsph;
    }
    return cur;
}

int nfunc(const ShellView& s) { return s.ncontr * (2 * s.l + 1); }

// ------------------------------------------------------ derivative blocks
// Derivatives of (ab|cd) as in the reference's coulomb_block_derivative
// (two_electron.rs:1138-1247). A Hermite centre (the centre of a lone
// function) by the shift of the Hermite integrals: d/dP R_tuv = R_{t+1,u,v}
// for the bra pair and the negative for the ket pair, since R_PQ = P - Q. The
// centre of the bra's first function by raising and lowering its angular
// momentum: d/dA_x x_A^i exp(-a x_A^2) = 2a x_A^(i+1) exp(..) - i x_A^(i-1) exp(..),
// for which the bra pair carries one extra order on its first function.
enum Deriv : int { kBraHermite = 0, kKetHermite = 1, kBraFunction = 2 };

struct HTerm {
    int t, u, v;
    double c;
};

// E^{ij}_t of one axis, with the raise/lower rule applied when `raise`.
double axis_coef(const PrimPair& P, int axis, int i, int j, int t, bool raise) {
    if (!raise) return P.e[axis].get(i, j, t);
    double v = 2.0 * P.ea * P.e[axis].get(i + 1, j, t);
    if (i > 0) v -= i * P.e[axis].get(i - 1, j, t);
    return v;
}

// Hermite terms of the Cartesian pair (a, b); the first function differentiated
// along `axis` when `raise`.
void pair_terms(const PrimPair& P, const std::array<int, 3>& a, const std::array<int, 3>& b, bool raise, int axis,
                double sign_per_order, std::vector<HTerm>& out) {
    out.clear();
    const int ext = raise ? 1 : 0;
    for (int t = 0; t <= a[0] + b[0] + (axis == 0 ? ext : 0); ++t) {
        const double ex = axis_coef(P, 0, a[0], b[0], t, raise && axis == 0);
        if (ex == 0.0) continue;
        for (int u = 0; u <= a[1] + b[1] + (axis == 1 ? ext : 0); ++u) {
            const double ey = ex * axis_coef(P, 1, a[1], b[1], u, raise && axis == 1);
            if (ey == 0.0) continue;
            for (int v = 0; v <= a[2] + b[2] + (axis == 2 ? ext : 0); ++v) {
                const double ez = ey * axis_coef(P, 2, a[2], b[2], v, raise && axis == 2);
                if (ez == 0.0) continue;
                const double sg = (sign_per_order < 0.0 && ((t + u + v) & 1)) ? -1.0 : 1.0;
                out.push_back({t, u, v, sg * ez});
            }
        }
    }
}

// out[axis] (layout of coulomb_block) += d/dX (ab|cd) for the centre `mode` selects;
// for kBraFunction the bra pair must carry one extra order on its first function.
void coulomb_block_derivative(const Pair& bra, const Pair& ket, const Transforms& tr, int kernel, double omega,
                              int mode, RWork& w, std::vector<double>* out) {
    const auto& ca = tr.comps[bra.la];
    const auto& cb = tr.comps[bra.lb];
    const auto& cc = tr.comps[ket.la];
    const auto& cd = tr.comps[ket.lb];
    const int na = (int)ca.size(), nb = (int)cb.size(), nc = (int)cc.size(), nd = (int)cd.size();
    const int L = bra.la + bra.lb + ket.la + ket.lb + 1;
    const int s1 = L + 1;
    std::vector<double> R(s1 * s1 * s1);
    std::vector<std::vector<HTerm>> kterms(nc * nd);
    std::vector<HTerm> bt;
    std::vector<double> val(3 * na * nb * nc * nd);
    const int sc = ket.kb * nd, sb = ket.ka * nc * sc, sa = bra.kb * nb * sb;
    const double hsign = mode == kKetHermite ? -1.0 : 1.0;
    for (size_t ib = 0; ib < bra.prims.size(); ++ib) {
        const PrimPair& P = bra.prims[ib];
        for (size_t ik = 0; ik < ket.prims.size(); ++ik) {
            const PrimPair& Q = ket.prims[ik];
            const double p = P.p, q = Q.p;
            const double alpha = p * q / (p + q);
            const double pq[3] = {P.P[0] - Q.P[0], P.P[1] - Q.P[1], P.P[2] - Q.P[2]};
            hermite_r_kernel(L, alpha, kernel, omega, pq, w, R.data());
            for (int ic = 0; ic < nc; ++ic)
                for (int id = 0; id < nd; ++id) pair_terms(Q, cc[ic], cd[id], false, 0, -1.0, kterms[ic * nd + id]);
            for (int axis = 0; axis < 3; ++axis) {
                const int dx = (mode != kBraFunction && axis == 0) ? 1 : 0;
                const int dy = (mode != kBraFunction && axis == 1) ? 1 : 0;
                const int dz = (mode != kBraFunction && axis == 2) ? 1 : 0;
                for (int ia = 0; ia < na; ++ia)
                    for (int jb = 0; jb < nb; ++jb) {
                        pair_terms(P, ca[ia], cb[jb], mode == kBraFunction, axis, 1.0, bt);
                        for (int icd = 0; icd < nc * nd; ++icd) {
                            double v = 0.0;
                            for (const HTerm& x : bt)
                                for (const HTerm& y : kterms[icd])
                                    v += x.c * y.c * R[((x.t + y.t + dx) * s1 + x.u + y.u + dy) * s1 + x.v + y.v + dz];
                            val[((axis * na + ia) * nb + jb) * nc * nd + icd] = (mode == kBraFunction ? 1.0 : hsign) * v;
                        }
                    }
            }
            const double pref = 2.0 * std::pow(kPi, 2.5) / (p * q * std::sqrt(p + q));
            for (int axis = 0; axis < 3; ++axis)
                for (int ka = 0; ka < bra.ka; ++ka)
                    for (int kb = 0; kb < bra.kb; ++kb) {
                        const double cbra = pref * bra.coef[(ib * bra.ka + ka) * bra.kb + kb];
                        for (int kc = 0; kc < ket.ka; ++kc)
                            for (int kd = 0; kd < ket.kb; ++kd) {
                                const double cf = cbra * ket.coef[(ik * ket.ka + kc) * ket.kb + kd];
                                if (cf == 0.0) continue;
                                const int base = ka * na * sa + kb * nb * sb + kc * nc * sc + kd * nd;
                                for (int ia = 0; ia < na; ++ia)
                                    for (int jb = 0; jb < nb; ++jb)
                                        for (int ic = 0; ic < nc; ++ic) {
                                            double* o = &out[axis][base + ia * sa + jb * sb + ic * sc];
                                            const double* s = &val[(((axis * na + ia) * nb + jb) * nc + ic) * nd];
                                            for (int id = 0; id < nd; ++id) o[id] += cf * s[id];
                                        }
                            }
                    }
        }
    }
}

}  // namespace

// =================================================================== C ABI
extern "C" {

struct md_shells {
    int64_t n_shells;
    const int64_t* angular_momenta;
    const double* centers;          // [n_shells][3]
    const int64_t* primitive_offsets;  // [n_shells + 1]
    const double* exponents;
    const double* coefficients;     // shell by shell, [contraction][primitive]
    const int64_t* n_contractions;
};

}  // extern "C"

namespace {
bool build_table(const md_shells* s, Table& t) {
    t.shells.clear();
    t.nfunc = 0;
    t.maxl = 0;
    long coff = 0;
    for (int64_t i = 0; i < s->n_shells; ++i) {
        ShellView v;
        v.l = (int)s->angular_momenta[i];
        if (v.l < 0 || v.l > kMaxL) return false;
        for (int x = 0; x < 3; ++x) v.center[x] = s->centers[3 * i + x];
        const int64_t p0 = s->primitive_offsets[i], p1 = s->primitive_offsets[i + 1];
        v.nprim = (int)(p1 - p0);
        if (v.nprim < 1) return false;
        v.exps = s->exponents + p0;
        v.ncontr = (int)s->n_contractions[i];
        if (v.ncontr < 1) return false;
        v.coefs = s->coefficients + coff;
        coff += (long)v.ncontr * v.nprim;
        v.first_function = t.nfunc;
        t.nfunc += nfunc(v);
        t.maxl = std::max(t.maxl, v.l);
        t.shells.push_back(v);
    }
    return true;
}
}  // namespace

extern "C" {

int md_version() { return 1; }

int md_boys(int nmax, double t, double* out) {
    if (!(t >= 0.0) || nmax < 0) return 1;
    boys(nmax, t, out);
    return 0;
}

int md_spherical_transformation(int l, double* out) {
    if (l < 0 || l > 16) return 1;
    auto m = sph_transform(l);
    std::memcpy(out, m.data(), sizeof(double) * m.size());
    return 0;
}

int md_n_functions(const md_shells* s) {
    Table t;
    if (!build_table(s, t)) return -1;
    return t.nfunc;
}

// kind: 0 overlap, 1 kinetic, 2 nuclear attraction
static int one_electron(int kind, const md_shells* bs, const md_shells* ks, int64_t ntr, const double* tr,
                        int64_t ncharge, const double* charges, const double* positions, int kernel,
                        double omega, double* out) {
    Table bra, ket;
    if (!build_table(bs, bra) || !build_table(ks, ket)) return 1;
    const int maxl = std::max(bra.maxl, ket.maxl);
    Transforms T(maxl + 2);
    const long nb = bra.nfunc, nk = ket.nfunc;
    for (int64_t it = 0; it < ntr; ++it) {
        double* img = out + it * nb * nk;
#pragma omp parallel
        {
            RWork w;
#pragma omp for schedule(dynamic)
            for (int ia = 0; ia < (int)bra.shells.size(); ++ia) {
                const ShellView& a = bra.shells[ia];
                for (int ib = 0; ib < (int)ket.shells.size(); ++ib) {
                    const ShellView& b = ket.shells[ib];
                    double cbt[3];
                    for (int x = 0; x < 3; ++x) cbt[x] = b.center[x] + tr[3 * it + x];
                    Pair pr = make_pair(a, a.center, b, cbt, 0, kind == 1 ? 2 : 0);
                    const auto& ca = T.comps[a.l];
                    const auto& cb = T.comps[b.l];
                    const int na = (int)ca.size(), nbb = (int)cb.size();
                    std::vector<double> block(a.ncontr * na * b.ncontr * nbb, 0.0);
                    std::vector<double> vals(na * nbb);
                    const int L = a.l + b.l;
                    std::vector<double> R((L + 1) * (L + 1) * (L + 1)), Rs;
                    for (size_t ip = 0; ip < pr.prims.size(); ++ip) {
                        const PrimPair& P = pr.prims[ip];
                        const double p = P.p;
                        if (kind == 2) {
                            Rs.assign(R.size(), 0.0);
                            for (int64_t c = 0; c < ncharge; ++c) {
                                const double pc[3] = {P.P[0] - positions[3 * c], P.P[1] - positions[3 * c + 1],
                                                      P.P[2] - positions[3 * c + 2]};
                                hermite_r_kernel(L, p, kernel, omega, pc, w, R.data());
                                for (size_t i = 0; i < R.size(); ++i) Rs[i] -= charges[c] * R[i];
                            }
                        }
                        const double ov = std::pow(kPi / p, 1.5);
                        for (int i = 0; i < na; ++i)
                            for (int j = 0; j < nbb; ++j) {
                                const auto& ai = ca[i];
                                const auto& bj = cb[j];
                                double v = 0.0;
                                if (kind == 0) {
                                    v = ov * P.e[0].get(ai[0], bj[0], 0) * P.e[1].get(ai[1], bj[1], 0) *
                                        P.e[2].get(ai[2], bj[2], 0);
                                } else if (kind == 1) {
                                    double s[3], d2[3];
                                    const double b2 = P.eb;
                                    for (int x = 0; x < 3; ++x) {
                                        const int ii = ai[x], jj = bj[x];
                                        s[x] = P.e[x].get(ii, jj, 0);
                                        d2[x] = 4.0 * b2 * b2 * P.e[x].get(ii, jj + 2, 0) -
                                                2.0 * b2 * (2 * jj + 1) * P.e[x].get(ii, jj, 0) +
                                                (jj >= 2 ? jj * (jj - 1) * P.e[x].get(ii, jj - 2, 0) : 0.0);
                                    }
                                    v = -0.5 * ov * (d2[0] * s[1] * s[2] + s[0] * d2[1] * s[2] + s[0] * s[1] * d2[2]);
                                } else {
                                    const int s1 = L + 1;
                                    for (int t = 0; t <= ai[0] + bj[0]; ++t)
                                        for (int u = 0; u <= ai[1] + bj[1]; ++u)
                                            for (int vv = 0; vv <= ai[2] + bj[2]; ++vv)
                                                v += P.e[0].get(ai[0], bj[0], t) * P.e[1].get(ai[1], bj[1], u) *
                                                     P.e[2].get(ai[2], bj[2], vv) * Rs[(t * s1 + u) * s1 + vv];
                                    v *= 2.0 * kPi / p;
                                }
                                vals[i * nbb + j] = v;
                            }
                        for (int ka = 0; ka < a.ncontr; ++ka)
                            for (int kb = 0; kb < b.ncontr; ++kb) {
                                const double cf = pr.coef[(ip * a.ncontr + ka) * b.ncontr + kb];
                                for (int i = 0; i < na; ++i)
                                    for (int j = 0; j < nbb; ++j)
                                        block[((ka * na + i) * b.ncontr + kb) * nbb + j] += cf * vals[i * nbb + j];
                            }
                    }
                    const int ls[4] = {a.l, b.l, -1, -1};
                    const int kk[4] = {a.ncontr, b.ncontr, 1, 1};
                    auto sph = to_spherical(block, ls, kk, T);
                    const int fa = nfunc(a), fb = nfunc(b);
                    for (int i = 0; i < fa; ++i)
                        for (int j = 0; j < fb; ++j)
                            img[(long)(a.first_function + i) * nk + b.first_function + j] = sph[i * fb + j];
                }
            }
        }
    }
    return 0;
}

int md_overlap(const md_shells* b, const md_shells* k, int64_t ntr, const double* tr, double* out) {
    return one_electron(0, b, k, ntr, tr, 0, nullptr, nullptr, 0, 0.0, out);
}
int md_kinetic(const md_shells* b, const md_shells* k, int64_t ntr, const double* tr, double* out) {
    return one_electron(1, b, k, ntr, tr, 0, nullptr, nullptr, 0, 0.0, out);
}
int md_nuclear_attraction(const md_shells* b, const md_shells* k, int64_t ntr, const double* tr,
                          int64_t ncharge, const double* charges, const double* positions, int kernel,
                          double omega, double* out) {
    return one_electron(2, b, k, ntr, tr, ncharge, charges, positions, kernel, omega, out);
}

// (P|Q(r - T)) -> out[image][bra][ket]
int md_coulomb_two_center(const md_shells* bs, const md_shells* ks, int64_t ntr, const double* tr, int kernel,
                          double omega, double* out) {
    Table bra, ket;
    if (!build_table(bs, bra) || !build_table(ks, ket)) return 1;
    Transforms T(std::max(bra.maxl, ket.maxl));
    const long nb = bra.nfunc, nk = ket.nfunc;
    for (int64_t it = 0; it < ntr; ++it) {
        double* img = out + it * nb * nk;
#pragma omp parallel
        {
            RWork w;
#pragma omp for schedule(dynamic)
            for (int ia = 0; ia < (int)bra.shells.size(); ++ia) {
                const ShellView& a = bra.shells[ia];
                Pair pa = single_pair(a, a.center);
                for (int ic = 0; ic < (int)ket.shells.size(); ++ic) {
                    const ShellView& c = ket.shells[ic];
                    double cc[3];
                    for (int x = 0; x < 3; ++x) cc[x] = c.center[x] + tr[3 * it + x];
                    Pair pc = single_pair(c, cc);
                    std::vector<double> block(a.ncontr * n_cart(a.l) * c.ncontr * n_cart(c.l), 0.0);
                    coulomb_block(pa, pc, T, kernel, omega, w, block);
                    const int ls[4] = {a.l, -1, c.l, -1};
                    const int kk[4] = {a.ncontr, 1, c.ncontr, 1};
                    auto sph = to_spherical(block, ls, kk, T);
                    const int fa = nfunc(a), fc = nfunc(c);
                    for (int i = 0; i < fa; ++i)
                        for (int j = 0; j < fc; ++j)
                            img[(long)(a.first_function + i) * nk + c.first_function + j] = sph[i * fc + j];
                }
            }
        }
    }
    return 0;
}

// (P(r - T_P)| mu nu(r - T_nu)) -> out[image][aux][bra][ket]; tr[image][2][3]
int md_coulomb_three_center(const md_shells* as, const md_shells* bs, const md_shells* ks, int64_t ntr,
                            const double* tr, int kernel, double omega, double* out) {
    Table aux, bra, ket;
    if (!build_table(as, aux) || !build_table(bs, bra) || !build_table(ks, ket)) return 1;
    Transforms T(std::max(aux.maxl, std::max(bra.maxl, ket.maxl)));
    const long na = aux.nfunc, nb = bra.nfunc, nk = ket.nfunc;
    for (int64_t it = 0; it < ntr; ++it) {
        const double* tp = tr + 6 * it;
        const double* tn = tr + 6 * it + 3;
        double* img = out + it * na * nb * nk;
#pragma omp parallel
        {
            RWork w;
#pragma omp for schedule(dynamic)
            for (int ip = 0; ip < (int)aux.shells.size(); ++ip) {
                const ShellView& P = aux.shells[ip];
                double cp[3];
                for (int x = 0; x < 3; ++x) cp[x] = P.center[x] + tp[x];
                Pair pp = single_pair(P, cp);
                for (int ia = 0; ia < (int)bra.shells.size(); ++ia) {
                    const ShellView& a = bra.shells[ia];
                    for (int ib = 0; ib < (int)ket.shells.size(); ++ib) {
                        const ShellView& b = ket.shells[ib];
                        double cb[3];
                        for (int x = 0; x < 3; ++x) cb[x] = b.center[x] + tn[x];
                        Pair pab = make_pair(a, a.center, b, cb);
                        std::vector<double> block(
                            a.ncontr * n_cart(a.l) * b.ncontr * n_cart(b.l) * P.ncontr * n_cart(P.l), 0.0);
                        coulomb_block(pab, pp, T, kernel, omega, w, block);
                        const int ls[4] = {a.l, b.l, P.l, -1};
                        const int kk[4] = {a.ncontr, b.ncontr, P.ncontr, 1};
                        auto sph = to_spherical(block, ls, kk, T);
                        const int fa = nfunc(a), fb = nfunc(b), fp = nfunc(P);
                        for (int i = 0; i < fa; ++i)
                            for (int j = 0; j < fb; ++j)
                                for (int m = 0; m < fp; ++m)
                                    img[((long)(P.first_function + m) * nb + a.first_function + i) * nk +
                                        b.first_function + j] = sph[(i * fb + j) * fp + m];
                    }
                }
            }
        }
    }
    return 0;
}

// Spherical diagonal (ab|ab) of a shell pair -> sqrt of its maximum.
static double schwarz_pair(const Pair& pr, const Transforms& T, int kernel, double omega, RWork& w) {
    const int n = pr.ka * n_cart(pr.la) * pr.kb * n_cart(pr.lb);
    std::vector<double> block(n * n, 0.0);
    coulomb_block(pr, pr, T, kernel, omega, w, block);
    const int ls[4] = {pr.la, pr.lb, pr.la, pr.lb};
    const int kk[4] = {pr.ka, pr.kb, pr.ka, pr.kb};
    auto sph = to_spherical(block, ls, kk, T);
    const int ns = pr.ka * (2 * pr.la + 1) * pr.kb * (2 * pr.lb + 1);
    double m = 0.0;
    for (int i = 0; i < ns; ++i) m = std::max(m, sph[(long)i * ns + i]);
    return std::sqrt(m);
}

int md_schwarz_bounds(const md_shells* bs, const md_shells* ks, int64_t ntr, const double* tr, int kernel,
                      double omega, double* out) {
    Table bra, ket;
    if (!build_table(bs, bra) || !build_table(ks, ket)) return 1;
    Transforms T(std::max(bra.maxl, ket.maxl));
    const long nsb = bra.shells.size(), nsk = ket.shells.size();
    for (int64_t it = 0; it < ntr; ++it) {
#pragma omp parallel
        {
            RWork w;
#pragma omp for schedule(dynamic)
            for (long ia = 0; ia < nsb; ++ia)
                for (long ib = 0; ib < nsk; ++ib) {
                    const ShellView& a = bra.shells[ia];
                    const ShellView& b = ket.shells[ib];
                    double cb[3];
                    for (int x = 0; x < 3; ++x) cb[x] = b.center[x] + tr[3 * it + x];
                    Pair pr = make_pair(a, a.center, b, cb);
                    out[(it * nsb + ia) * nsk + ib] = schwarz_pair(pr, T, kernel, omega, w);
                }
        }
    }
    return 0;
}

// (a b(r - T_b) | c(r - T_c) d(r - T_d)) -> out[image][a][b][c][d]; tr[image][3][3].
// Shell quartets with Q_ab Q_cd < threshold stay zero.
int md_coulomb_four_center(const md_shells* s0, const md_shells* s1, const md_shells* s2, const md_shells* s3,
                           int64_t ntr, const double* tr, int kernel, double omega, double threshold,
                           double* out) {
    Table t0, t1, t2, t3;
    if (!build_table(s0, t0) || !build_table(s1, t1) || !build_table(s2, t2) || !build_table(s3, t3)) return 1;
    const int maxl = std::max(std::max(t0.maxl, t1.maxl), std::max(t2.maxl, t3.maxl));
    Transforms T(maxl);
    const long n0 = t0.nfunc, n1 = t1.nfunc, n2 = t2.nfunc, n3 = t3.nfunc;
    const long size = n0 * n1 * n2 * n3;
    for (int64_t it = 0; it < ntr; ++it) {
        const double* tb = tr + 9 * it;
        const double* tc = tb + 3;
        const double* td = tb + 6;
        double* img = out + it * size;
        std::memset(img, 0, sizeof(double) * size);
        // Shell pairs with their Schwarz bounds.
        std::vector<Pair> bra_pairs, ket_pairs;
        std::vector<std::array<int, 2>> bra_idx, ket_idx;
        for (int a = 0; a < (int)t0.shells.size(); ++a)
            for (int b = 0; b < (int)t1.shells.size(); ++b) {
                double cb[3];
                for (int x = 0; x < 3; ++x) cb[x] = t1.shells[b].center[x] + tb[x];
                bra_pairs.push_back(make_pair(t0.shells[a], t0.shells[a].center, t1.shells[b], cb));
                bra_idx.push_back({a, b});
            }
        for (int c = 0; c < (int)t2.shells.size(); ++c)
            for (int d = 0; d < (int)t3.shells.size(); ++d) {
                double cc[3], cd[3];
                for (int x = 0; x < 3; ++x) {
                    cc[x] = t2.shells[c].center[x] + tc[x];
                    cd[x] = t3.shells[d].center[x] + td[x];
                }
                ket_pairs.push_back(make_pair(t2.shells[c], cc, t3.shells[d], cd));
                ket_idx.push_back({c, d});
            }
        std::vector<double> qb(bra_pairs.size()), qk(ket_pairs.size());
#pragma omp parallel
        {
            RWork w;
#pragma omp for schedule(dynamic)
            for (long i = 0; i < (long)bra_pairs.size(); ++i) qb[i] = schwarz_pair(bra_pairs[i], T, kernel, omega, w);
#pragma omp for schedule(dynamic)
            for (long i = 0; i < (long)ket_pairs.size(); ++i) qk[i] = schwarz_pair(ket_pairs[i], T, kernel, omega, w);
#pragma omp for schedule(dynamic)
            for (long ibp = 0; ibp < (long)bra_pairs.size(); ++ibp) {
                const Pair& B = bra_pairs[ibp];
                const ShellView& a = t0.shells[bra_idx[ibp][0]];
                const ShellView& b = t1.shells[bra_idx[ibp][1]];
                for (long ikp = 0; ikp < (long)ket_pairs.size(); ++ikp) {
                    if (qb[ibp] * qk[ikp] < threshold) continue;
                    const Pair& K = ket_pairs[ikp];
                    const ShellView& c = t2.shells[ket_idx[ikp][0]];
                    const ShellView& d = t3.shells[ket_idx[ikp][1]];
                    std::vector<double> block((long)B.ka * n_cart(B.la) * B.kb * n_cart(B.lb) * K.ka * n_cart(K.la) *
                                                  K.kb * n_cart(K.lb),
                                              0.0);
                    coulomb_block(B, K, T, kernel, omega, w, block);
                    const int ls[4] = {B.la, B.lb, K.la, K.lb};
                    const int kk[4] = {B.ka, B.kb, K.ka, K.kb};
                    auto sph = to_spherical(block, ls, kk, T);
                    const int fa = nfunc(a), fb = nfunc(b), fc = nfunc(c), fd = nfunc(d);
                    for (int i = 0; i < fa; ++i)
                        for (int j = 0; j < fb; ++j)
                            for (int k = 0; k < fc; ++k)
                                for (int l = 0; l < fd; ++l)
                                    img[(((long)(a.first_function + i) * n1 + b.first_function + j) * n2 +
                                         c.first_function + k) *
                                            n3 +
                                        d.first_function + l] = sph[((i * fb + j) * fc + k) * fd + l];
                }
            }
        }
    }
    return 0;
}

// <d/dA mu | O | nu> for O = 1 (kind 0), -1/2 nabla^2 (kind 1) or the point
// charges (kind 2) -> out[image][3][bra][ket]; for kind 2 also
// <mu | d/dC V_C | nu> -> nuclei[image][charge][3][bra][ket]
// (one_electron.rs derivatives; the bra function by raising and lowering its
// angular momentum, a charge position by the shift of the Hermite integrals).
static int one_electron_derivative(int kind, const md_shells* bs, const md_shells* ks, int64_t ntr, const double* tr,
                                   int64_t ncharge, const double* charges, const double* positions, int kernel,
                                   double omega, double* out, double* nuclei) {
    Table bra, ket;
    if (!build_table(bs, bra) || !build_table(ks, ket)) return 1;
    const int maxl = std::max(bra.maxl, ket.maxl);
    Transforms T(maxl);
    const long nb = bra.nfunc, nk = ket.nfunc;
    const long plane = nb * nk;
    for (int64_t it = 0; it < ntr; ++it) {
        double* img = out + it * 3 * plane;
        double* nimg = nuclei ? nuclei + it * ncharge * 3 * plane : nullptr;
#pragma omp parallel
        {
            RWork w;
#pragma omp for schedule(dynamic)
            for (int ia = 0; ia < (int)bra.shells.size(); ++ia) {
                const ShellView& a = bra.shells[ia];
                for (int ib = 0; ib < (int)ket.shells.size(); ++ib) {
                    const ShellView& b = ket.shells[ib];
                    double cbt[3];
                    for (int x = 0; x < 3; ++x) cbt[x] = b.center[x] + tr[3 * it + x];
                    Pair pr = make_pair(a, a.center, b, cbt, 1, kind == 1 ? 2 : 0);
                    const auto& ca = T.comps[a.l];
                    const auto& cb = T.comps[b.l];
                    const int na = (int)ca.size(), nbb = (int)cb.size();
                    const long bsz = (long)a.ncontr * na * b.ncontr * nbb;
                    std::vector<double> block(3 * bsz, 0.0);
                    std::vector<double> nblock(kind == 2 ? ncharge * 3 * bsz : 0, 0.0);
                    std::vector<double> vals(3 * na * nbb), nvals(kind == 2 ? ncharge * 3 * na * nbb : 0);
                    const int L = a.l + b.l + 1;
                    const int s1 = L + 1;
                    std::vector<double> R(s1 * s1 * s1), Rs;
                    std::vector<std::vector<double>> Rc(kind == 2 ? ncharge : 0);
                    std::vector<HTerm> terms;
                    for (size_t ip = 0; ip < pr.prims.size(); ++ip) {
                        const PrimPair& P = pr.prims[ip];
                        const double p = P.p;
                        if (kind == 2) {
                            Rs.assign(R.size(), 0.0);
                            for (int64_t c = 0; c < ncharge; ++c) {
                                const double pc[3] = {P.P[0] - positions[3 * c], P.P[1] - positions[3 * c + 1],
                                                      P.P[2] - positions[3 * c + 2]};
                                hermite_r_kernel(L, p, kernel, omega, pc, w, R.data());
                                Rc[c] = R;
                                for (size_t i = 0; i < R.size(); ++i) Rs[i] -= charges[c] * R[i];
                            }
                        }
                        const double ov = std::pow(kPi / p, 1.5);
                        const double b2 = P.eb;
                        auto s1d = [&](int x, int i, int j) { return P.e[x].get(i, j, 0); };
                        auto d2 = [&](int x, int i, int j) {
                            return 4.0 * b2 * b2 * P.e[x].get(i, j + 2, 0) - 2.0 * b2 * (2 * j + 1) * P.e[x].get(i, j, 0) +
                                   (j >= 2 ? j * (j - 1) * P.e[x].get(i, j - 2, 0) : 0.0);
                        };
                        auto raise = [&](auto f, int x, int i, int j) {
                            double v = 2.0 * P.ea * f(x, i + 1, j);
                            if (i > 0) v -= i * f(x, i - 1, j);
                            return v;
                        };
                        for (int axis = 0; axis < 3; ++axis)
                            for (int i = 0; i < na; ++i)
                                for (int j = 0; j < nbb; ++j) {
                                    const auto& ai = ca[i];
                                    const auto& bj = cb[j];
                                    double v = 0.0;
                                    if (kind == 0) {
                                        v = ov;
                                        for (int x = 0; x < 3; ++x)
                                            v *= x == axis ? raise(s1d, x, ai[x], bj[x]) : s1d(x, ai[x], bj[x]);
                                    } else if (kind == 1) {
                                        double s[3], t[3];
                                        for (int x = 0; x < 3; ++x) {
                                            s[x] = x == axis ? raise(s1d, x, ai[x], bj[x]) : s1d(x, ai[x], bj[x]);
                                            t[x] = x == axis ? raise(d2, x, ai[x], bj[x]) : d2(x, ai[x], bj[x]);
                                        }
                                        v = -0.5 * ov * (t[0] * s[1] * s[2] + s[0] * t[1] * s[2] + s[0] * s[1] * t[2]);
                                    } else {
                                        pair_terms(P, ai, bj, true, axis, 1.0, terms);
                                        for (const HTerm& h : terms) v += h.c * Rs[(h.t * s1 + h.u) * s1 + h.v];
                                        v *= 2.0 * kPi / p;
                                        pair_terms(P, ai, bj, false, 0, 1.0, terms);
                                        const int dx = axis == 0, dy = axis == 1, dz = axis == 2;
                                        for (int64_t c = 0; c < ncharge; ++c) {
                                            double vc = 0.0;
                                            for (const HTerm& h : terms)
                                                vc += h.c * Rc[c][((h.t + dx) * s1 + h.u + dy) * s1 + h.v + dz];
                                            nvals[((c * 3 + axis) * na + i) * nbb + j] = charges[c] * 2.0 * kPi / p * vc;
                                        }
                                    }
                                    vals[(axis * na + i) * nbb + j] = v;
                                }
                        for (int ka = 0; ka < a.ncontr; ++ka)
                            for (int kb = 0; kb < b.ncontr; ++kb) {
                                const double cf = pr.coef[(ip * a.ncontr + ka) * b.ncontr + kb];
                                for (int axis = 0; axis < 3; ++axis)
                                    for (int i = 0; i < na; ++i)
                                        for (int j = 0; j < nbb; ++j)
                                            block[axis * bsz + ((ka * na + i) * b.ncontr + kb) * nbb + j] +=
                                                cf * vals[(axis * na + i) * nbb + j];
                                if (kind == 2)
                                    for (int64_t c = 0; c < ncharge; ++c)
                                        for (int axis = 0; axis < 3; ++axis)
                                            for (int i = 0; i < na; ++i)
                                                for (int j = 0; j < nbb; ++j)
                                                    nblock[(c * 3 + axis) * bsz + ((ka * na + i) * b.ncontr + kb) * nbb + j] +=
                                                        cf * nvals[((c * 3 + axis) * na + i) * nbb + j];
                            }
                    }
                    const int ls[4] = {a.l, b.l, -1, -1};
                    const int kk[4] = {a.ncontr, b.ncontr, 1, 1};
                    const int fa = nfunc(a), fb = nfunc(b);
                    const long nsets = kind == 2 ? 3 + 3 * ncharge : 3;
                    for (long set = 0; set < nsets; ++set) {
                        std::vector<double> part(set < 3 ? block.begin() + set * bsz : nblock.begin() + (set - 3) * bsz,
                                                 set < 3 ? block.begin() + (set + 1) * bsz
                                                         : nblock.begin() + (set - 2) * bsz);
                        auto sph = to_spherical(part, ls, kk, T);
                        double* tgt = set < 3 ? img + set * plane : nimg + (set - 3) * plane;
                        for (int i = 0; i < fa; ++i)
                            for (int j = 0; j < fb; ++j)
                                tgt[(long)(a.first_function + i) * nk + b.first_function + j] = sph[i * fb + j];
                    }
                }
            }
        }
    }
    return 0;
}

int md_overlap_derivative(const md_shells* b, const md_shells* k, int64_t ntr, const double* tr, double* out) {
    return one_electron_derivative(0, b, k, ntr, tr, 0, nullptr, nullptr, 0, 0.0, out, nullptr);
}
int md_kinetic_derivative(const md_shells* b, const md_shells* k, int64_t ntr, const double* tr, double* out) {
    return one_electron_derivative(1, b, k, ntr, tr, 0, nullptr, nullptr, 0, 0.0, out, nullptr);
}
int md_nuclear_attraction_derivative(const md_shells* b, const md_shells* k, int64_t ntr, const double* tr,
                                     int64_t ncharge, const double* charges, const double* positions, int kernel,
                                     double omega, double* by_center, double* by_nucleus) {
    return one_electron_derivative(2, b, k, ntr, tr, ncharge, charges, positions, kernel, omega, by_center,
                                   by_nucleus);
}

// (d/dP P | Q(r - T)) -> out[image][3][bra][ket] (two_electron.rs:132-190)
int md_coulomb_two_center_derivative(const md_shells* bs, const md_shells* ks, int64_t ntr, const double* tr,
                                     int kernel, double omega, double* out) {
    Table bra, ket;
    if (!build_table(bs, bra) || !build_table(ks, ket)) return 1;
    Transforms T(std::max(bra.maxl, ket.maxl));
    const long nb = bra.nfunc, nk = ket.nfunc;
    for (int64_t it = 0; it < ntr; ++it) {
        double* img = out + it * 3 * nb * nk;
#pragma omp parallel
        {
            RWork w;
#pragma omp for schedule(dynamic)
            for (int ia = 0; ia < (int)bra.shells.size(); ++ia) {
                const ShellView& a = bra.shells[ia];
                Pair pa = single_pair(a, a.center);
                for (int ic = 0; ic < (int)ket.shells.size(); ++ic) {
                    const ShellView& c = ket.shells[ic];
                    double cc[3];
                    for (int x = 0; x < 3; ++x) cc[x] = c.center[x] + tr[3 * it + x];
                    Pair pc = single_pair(c, cc);
                    const long bsz = (long)a.ncontr * n_cart(a.l) * c.ncontr * n_cart(c.l);
                    std::vector<double> blocks[3] = {std::vector<double>(bsz, 0.0), std::vector<double>(bsz, 0.0),
                                                     std::vector<double>(bsz, 0.0)};
                    coulomb_block_derivative(pa, pc, T, kernel, omega, kBraHermite, w, blocks);
                    const int ls[4] = {a.l, -1, c.l, -1};
                    const int kk[4] = {a.ncontr, 1, c.ncontr, 1};
                    const int fa = nfunc(a), fc = nfunc(c);
                    for (int axis = 0; axis < 3; ++axis) {
                        auto sph = to_spherical(blocks[axis], ls, kk, T);
                        for (int i = 0; i < fa; ++i)
                            for (int j = 0; j < fc; ++j)
                                img[((long)axis * nb + a.first_function + i) * nk + c.first_function + j] = sph[i * fc + j];
                    }
                }
            }
        }
    }
    return 0;
}

// (d/dP P(r - T_P) | mu nu(r - T_nu)) in slots 0..2 and (P | d/dA mu nu) in slots
// 3..5 -> out[image][6][aux][bra][ket]; tr[image][2][3] (two_electron.rs:300-394)
int md_coulomb_three_center_derivative(const md_shells* as, const md_shells* bs, const md_shells* ks, int64_t ntr,
                                       const double* tr, int kernel, double omega, double* out) {
    Table aux, bra, ket;
    if (!build_table(as, aux) || !build_table(bs, bra) || !build_table(ks, ket)) return 1;
    Transforms T(std::max(aux.maxl, std::max(bra.maxl, ket.maxl)));
    const long na = aux.nfunc, nb = bra.nfunc, nk = ket.nfunc;
    const long vol = na * nb * nk;
    for (int64_t it = 0; it < ntr; ++it) {
        const double* tp = tr + 6 * it;
        const double* tn = tr + 6 * it + 3;
        double* img = out + it * 6 * vol;
#pragma omp parallel
        {
            RWork w;
#pragma omp for schedule(dynamic)
            for (int ip = 0; ip < (int)aux.shells.size(); ++ip) {
                const ShellView& P = aux.shells[ip];
                double cp[3];
                for (int x = 0; x < 3; ++x) cp[x] = P.center[x] + tp[x];
                Pair pp = single_pair(P, cp);
                for (int ia = 0; ia < (int)bra.shells.size(); ++ia) {
                    const ShellView& a = bra.shells[ia];
                    for (int ib = 0; ib < (int)ket.shells.size(); ++ib) {
                        const ShellView& b = ket.shells[ib];
                        double cb[3];
                        for (int x = 0; x < 3; ++x) cb[x] = b.center[x] + tn[x];
                        Pair pab = make_pair(a, a.center, b, cb, 1, 0);
                        const long bsz = (long)a.ncontr * n_cart(a.l) * b.ncontr * n_cart(b.l) * P.ncontr * n_cart(P.l);
                        const int ls[4] = {a.l, b.l, P.l, -1};
                        const int kk[4] = {a.ncontr, b.ncontr, P.ncontr, 1};
                        const int fa = nfunc(a), fb = nfunc(b), fp = nfunc(P);
                        for (int which = 0; which < 2; ++which) {
                            std::vector<double> blocks[3] = {std::vector<double>(bsz, 0.0),
                                                             std::vector<double>(bsz, 0.0),
                                                             std::vector<double>(bsz, 0.0)};
                            coulomb_block_derivative(pab, pp, T, kernel, omega, which == 0 ? kKetHermite : kBraFunction,
                                                     w, blocks);
                            for (int axis = 0; axis < 3; ++axis) {
                                auto sph = to_spherical(blocks[axis], ls, kk, T);
                                double* slab = img + (long)(3 * which + axis) * vol;
                                for (int i = 0; i < fa; ++i)
                                    for (int j = 0; j < fb; ++j)
                                        for (int m = 0; m < fp; ++m)
                                            slab[((long)(P.first_function + m) * nb + a.first_function + i) * nk +
                                                 b.first_function + j] = sph[(i * fb + j) * fp + m];
                            }
                        }
                    }
                }
            }
        }
    }
    return 0;
}

void md_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int md_get_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
