// McMurchie–Davidson integral kernels for sm_100a, FP64.
//
// Reference counterparts (crates/hafnium-core/src/integrals/):
//   (P|Q)        two_electron.rs:74-130  coulomb_two_center, Full kernel, threshold 0
//   (P|mu nu)    two_electron.rs:212-297 coulomb_three_center, mu<=nu symmetric path
//   S, T, V      one_electron.rs:40-190
// The primitive-quartet contraction follows two_electron.rs:1398-1580 with the
// prefactor 2 pi^(5/2) / (p q sqrt(p+q)); the Cartesian-to-spherical transform is
// applied to the bra pair's Hermite coefficients once per primitive pair instead
// of to every output block (cartesian.rs:93-110, two_electron.rs:1028-1060).
#include <cmath>
#include <mutex>
#include <vector>

#include "integrals.cuh"
#include "md.cuh"

namespace hf {

__constant__ double c_c2s[kC2sSize];
// (t, u, v) of each tetrahedral index up to order 8, and Cartesian exponents per l.
__constant__ int c_tet_t[ntet(8)];
__constant__ int c_tet_u[ntet(8)];
__constant__ int c_tet_v[ntet(8)];
__constant__ int c_cart[kMaxAuxL + 1][15][3];

namespace {

double fact(int n) {
    double v = 1.0;
    for (int k = 2; k <= n; ++k) v *= k;
    return v;
}
double binom(int n, int k) {
    if (k < 0 || k > n) return 0.0;
    double v = 1.0;
    for (int i = 0; i < k; ++i) v = v * (n - i) / (i + 1);
    return std::round(v);
}
// Row-major [2l+1][ncart(l)] sphere-normalised solid harmonics (Helgaker 6.4.47).
std::vector<double> c2s_host(int l) {
    const int nc = ncart(l);
    std::vector<double> m(nsph(l) * nc, 0.0);
    const double sphere = std::sqrt((2.0 * l + 1.0) / (4.0 * kPi));
    std::vector<int> ms;
    if (l == 1) ms = {1, -1, 0};
    else
        for (int v = -l; v <= l; ++v) ms.push_back(v);
    for (int row = 0; row < (int)ms.size(); ++row) {
        const int mv = ms[row], am = std::abs(mv);
        const bool neg = mv < 0;
        const double norm = std::sqrt(2.0 * fact(l + am) * fact(l - am) / (mv == 0 ? 2.0 : 1.0)) /
                            (std::pow(2.0, am) * fact(l));
        for (int t = 0; t <= (l - am) / 2; ++t)
            for (int u = 0; u <= t; ++u) {
                const int vmax = neg ? (am - 1) / 2 : am / 2;
                for (int vh = 0; vh <= vmax; ++vh) {
                    const int two_v = neg ? 2 * vh + 1 : 2 * vh;
                    if (two_v > am) continue;
                    const double sign = ((t + vh) % 2 == 0) ? 1.0 : -1.0;
                    const double coef = sign * std::pow(0.25, t) * binom(l, t) * binom(l - t, am + t) *
                                        binom(t, u) * binom(am, two_v);
                    const int py = 2 * u + two_v, px = 2 * t + am - py, pz = l - 2 * t - am;
                    for (int c = 0; c < nc; ++c)
                        if (cart_x(l, c) == px && cart_y(l, c) == py && cart_z(l, c) == pz)
                            m[row * nc + c] += sphere * norm * coef;
                }
            }
    }
    return m;
}
}  // namespace

ConstantTables constant_tables_host() {
    ConstantTables t{};
    std::vector<double> all;
    for (int l = 0; l <= kMaxAuxL; ++l) {
        auto m = c2s_host(l);
        all.insert(all.end(), m.begin(), m.end());
    }
    for (size_t k = 0; k < all.size() && k < (size_t)kC2sSize; ++k) t.c2s[k] = all[k];
    for (int s = 0; s <= 8; ++s)
        for (int tt = 0; tt <= s; ++tt)
            for (int u = 0; u <= s - tt; ++u) {
                const int v = s - tt - u;
                t.tet_t[tet(tt, u, v)] = tt;
                t.tet_u[tet(tt, u, v)] = u;
                t.tet_v[tet(tt, u, v)] = v;
            }
    for (int l = 0; l <= kMaxAuxL; ++l)
        for (int c = 0; c < ncart(l); ++c) {
            t.cart[l][c][0] = cart_x(l, c);
            t.cart[l][c][1] = cart_y(l, c);
            t.cart[l][c][2] = cart_z(l, c);
        }
    return t;
}

void upload_c2s(cudaStream_t stream) {
    // the tables are constants of the library: written once per device
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

// F_m(T_j) for T_j = j * step, m < kBoysOrders, by the series of special.rs:67-81
// for the highest order and the downward recursion for the rest.
std::vector<double> boys_grid_host() {
    static std::mutex mutex;
    static std::vector<double> cached;
    std::lock_guard<std::mutex> lock(mutex);
    if (!cached.empty()) return cached;
    std::vector<double> g(kBoysGrid * kBoysOrders);
    const int nmax = kBoysOrders - 1;
    for (int j = 0; j < kBoysGrid; ++j) {
        const double t = j * kBoysStep;
        const double et = std::exp(-t);
        double term = 1.0 / (2 * nmax + 1), sum = term;
        for (int i = 1;; ++i) {
            term *= 2.0 * t / (2 * nmax + 2 * i + 1);
            sum += term;
            if (term < sum * 1e-17) break;
        }
        double* row = &g[j * kBoysOrders];
        row[nmax] = et * sum;
        for (int n = nmax; n >= 1; --n) row[n - 1] = (2.0 * t * row[n] + et) / (2 * n - 1);
    }
    cached = g;
    return g;
}

// F_0..F_L(T) of the device evaluation the integral kernels use, one argument
// per thread, into out[i][0..L] (the values special.rs:34-51 fill_boys gives).
template <int L>
__global__ void k_boys_values(const double* __restrict__ t, int64_t count, const double* __restrict__ btable,
                              double* __restrict__ out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= count) return;
    double F[L + 1];
    boys<L>(t[i], btable, F);
#pragma unroll
    for (int n = 0; n <= L; ++n) out[i * (L + 1) + n] = F[n];
}

template <int L>
cudaError_t boys_values_l(const double* t, int64_t count, const double* btable, double* out, cudaStream_t stream) {
    k_boys_values<L><<<(unsigned)((count + 127) / 128), 128, 0, stream>>>(t, count, btable, out);
    return cudaGetLastError();
}

cudaError_t launch_boys_values(const double* t, int64_t count, int n_max, const double* btable, double* out,
                               cudaStream_t stream) {
    if (count <= 0) return cudaSuccess;
    switch (n_max) {
        case 0: return boys_values_l<0>(t, count, btable, out, stream);
        case 1: return boys_values_l<1>(t, count, btable, out, stream);
        case 2: return boys_values_l<2>(t, count, btable, out, stream);
        case 3: return boys_values_l<3>(t, count, btable, out, stream);
        case 4: return boys_values_l<4>(t, count, btable, out, stream);
        case 5: return boys_values_l<5>(t, count, btable, out, stream);
        case 6: return boys_values_l<6>(t, count, btable, out, stream);
        case 7: return boys_values_l<7>(t, count, btable, out, stream);
        case 8: return boys_values_l<8>(t, count, btable, out, stream);
        case 9: return boys_values_l<9>(t, count, btable, out, stream);
        default: return cudaErrorInvalidValue;
    }
}
static_assert(kBoysOrders - kBoysTerms == 9, "launch_boys_values covers orders 0..9");

// ------------------------------------------------------------- (P|Q) metric
template <int LP, int LQ>
__global__ void __launch_bounds__(128) k_metric(const DevShell* __restrict__ aux, const double* __restrict__ exps,
                                                const double* __restrict__ coefs, const int* __restrict__ plist,
                                                int np, const int* __restrict__ qlist, int nq,
                                                const double* __restrict__ btable, double* __restrict__ M,
                                                int64_t ldm) {
    constexpr int L = LP + LQ;
    constexpr int NCP = ncart(LP), NCQ = ncart(LQ), NSP = nsph(LP), NSQ = nsph(LQ);
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)np * NSP * nq) return;
    const int iq = (int)(idx % nq);
    const int64_t rest = idx / nq;
    const int mp = (int)(rest % NSP);
    const int ip = (int)(rest / NSP);
    const DevShell P = aux[plist[ip]];
    const DevShell Q = aux[qlist[iq]];
    double crow[NCP];
#pragma unroll
    for (int c = 0; c < NCP; ++c) crow[c] = c_c2s[c2s_offset(LP) + mp * NCP + c];
    double acc[NSQ];
#pragma unroll
    for (int m = 0; m < NSQ; ++m) acc[m] = 0.0;
    const double X = P.x - Q.x, Y = P.y - Q.y, Z = P.z - Q.z;
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
            double h[NCQ];
#pragma unroll
            for (int b = 0; b < NCQ; ++b) {
                double s = 0.0;
#pragma unroll
                for (int a = 0; a < NCP; ++a)
                    s += crow[a] * R[tet(cart_x(LP, a) + cart_x(LQ, b), cart_y(LP, a) + cart_y(LQ, b),
                                         cart_z(LP, a) + cart_z(LQ, b))];
                h[b] = s;
            }
#pragma unroll
            for (int m = 0; m < NSQ; ++m) {
                double s = 0.0;
#pragma unroll
                for (int b = 0; b < NCQ; ++b) s += c_c2s[c2s_offset(LQ) + m * NCQ + b] * h[b];
                acc[m] += pref * s;
            }
        }
    }
    double* row = M + (int64_t)(P.fn + mp) * ldm + Q.fn;
#pragma unroll
    for (int m = 0; m < NSQ; ++m) row[m] = acc[m];
}

template <int LP, int LQ>
static cudaError_t metric_one(const DevShell* aux, const double* exps, const double* coefs, const int* plist, int np,
                              const int* qlist, int nq, const double* btable, double* M, int64_t ldm,
                              cudaStream_t stream) {
    const int64_t total = (int64_t)np * nsph(LP) * nq;
    if (total == 0) return cudaSuccess;
    const int64_t blocks = (total + 127) / 128;
    k_metric<LP, LQ><<<(unsigned)blocks, 128, 0, stream>>>(aux, exps, coefs, plist, np, qlist, nq, btable, M, ldm);
    return cudaGetLastError();
}

cudaError_t launch_metric(const DevShell* aux, const double* exps, const double* coefs,
                          const int* const* aux_by_l, const int* count, const double* btable, double* M,
                          int64_t ldm, cudaStream_t stream) {
    cudaError_t e = cudaSuccess;
#define HF_METRIC(LP, LQ)                                                                                    \
    if (e == cudaSuccess)                                                                                    \
        e = metric_one<LP, LQ>(aux, exps, coefs, aux_by_l[LP], count[LP], aux_by_l[LQ], count[LQ], btable, M, \
                               ldm, stream);
#define HF_METRIC_ROW(LP) HF_METRIC(LP, 0) HF_METRIC(LP, 1) HF_METRIC(LP, 2) HF_METRIC(LP, 3) HF_METRIC(LP, 4)
    HF_METRIC_ROW(0)
    HF_METRIC_ROW(1)
    HF_METRIC_ROW(2)
    HF_METRIC_ROW(3)
    HF_METRIC_ROW(4)
#undef HF_METRIC_ROW
#undef HF_METRIC
    return e;
}

// ------------------------------------------------------------ (P|mu nu)
// One CTA per orbital shell pair of class (LA <= LB); its threads run over the
// auxiliary shells of class LP, one thread per (aux shell, m_P). The pair's
// primitive data and spherical Hermite coefficients sit in shared memory and
// are read by every thread at the same address (broadcast).
template <int LA, int LB>
struct PairLayout {
    static constexpr int NSA = nsph(LA), NSB = nsph(LB), NSAB = NSA * NSB;
    static constexpr int KA = kMaxOrbContr[LA], KB = kMaxOrbContr[LB], KK = KA * KB;
    static constexpr int NH = ntet(LA + LB);
    // per primitive pair: p, Px, Py, Pz, 1/p, cc[KK], Etil[NSAB][NH]
    static constexpr int CC = 5, ET = CC + KK;
    static constexpr int STRIDE = ET + NSAB * NH;
};


// s_pos holds 2 kMaxPrimPairs + 1 ints: [pp0] -> compacted index or -1, the count
// at [kMaxPrimPairs], and compacted index -> pp0 from [kMaxPrimPairs + 1].
template <int LA, int LB>
__device__ int pair_prologue(const DevShell& A, const DevShell& B, const double* __restrict__ exps,
                             const double* __restrict__ coefs, double* smem, int* s_pos) {
    using PL = PairLayout<LA, LB>;
    constexpr int NCA = ncart(LA), NCB = ncart(LB);
    const int npp = A.nprim * B.nprim;
    const double abx = A.x - B.x, aby = A.y - B.y, abz = A.z - B.z;
    const double rab2 = abx * abx + aby * aby + abz * abz;
    int* s_src = s_pos + kMaxPrimPairs + 1;
    // significance flags, then a serial prefix (npp <= 256) for a deterministic order
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
            if (keep) s_src[k] = pp0;
            k += keep;
        }
        s_pos[kMaxPrimPairs] = k;
    }
    __syncthreads();
    // One task per (surviving primitive pair, spherical component pair m): the
    // pair's row Etil[m][*] (each task builds that pair's Cartesian Hermite
    // tables itself), and for m = 0 the pair's scalars. Spreading the rows over
    // the threads matters for the high angular momenta, whose shells have one or
    // few primitives.
    const int nk = s_pos[kMaxPrimPairs];
    for (int w = threadIdx.x; w < nk * PL::NSAB; w += blockDim.x) {
        const int pp = w / PL::NSAB, m = w - pp * PL::NSAB;
        const int ma = m / PL::NSB, mb = m - ma * PL::NSB;
        const int pp0 = s_src[pp];
        const int i = pp0 / B.nprim, j = pp0 % B.nprim;
        const double a = exps[A.prim + i], b = exps[B.prim + j];
        const double p = a + b;
        const double mu = a * b / p;
        const double px = (a * A.x + b * B.x) / p, py = (a * A.y + b * B.y) / p, pz = (a * A.z + b * B.z) / p;
        double* s = smem + pp * PL::STRIDE;
        if (m == 0) {
            s[0] = p;
            s[1] = px;
            s[2] = py;
            s[3] = pz;
            s[4] = 1.0 / p;
#pragma unroll
            for (int ka = 0; ka < PL::KA; ++ka)
#pragma unroll
                for (int kb = 0; kb < PL::KB; ++kb)
                    s[PL::CC + ka * PL::KB + kb] = (ka < A.ncontr && kb < B.ncontr)
                                                  ? coefs[A.coef + ka * A.nprim + i] * coefs[B.coef + kb * B.nprim + j]
                                                  : 0.0;
        }
        Hermite1D<LA, LB> ex, ey, ez;
        const double e00 = exp(-mu * rab2);
        ex.build(p, e00, px - A.x, px - B.x);
        ey.build(p, 1.0, py - A.y, py - B.y);
        ez.build(p, 1.0, pz - A.z, pz - B.z);
        double* et = s + PL::ET + m * PL::NH;
        for (int h = 0; h < PL::NH; ++h) et[h] = 0.0;
#pragma unroll 1
        for (int ca = 0; ca < NCA; ++ca) {
            const double ra = c_c2s[c2s_offset(LA) + ma * NCA + ca];
            if (ra == 0.0) continue;
#pragma unroll 1
            for (int cb = 0; cb < NCB; ++cb) {
                const double w2 = ra * c_c2s[c2s_offset(LB) + mb * NCB + cb];
                if (w2 == 0.0) continue;
                const int ix = c_cart[LA][ca][0], iy = c_cart[LA][ca][1], iz = c_cart[LA][ca][2];
                const int jx = c_cart[LB][cb][0], jy = c_cart[LB][cb][1], jz = c_cart[LB][cb][2];
#pragma unroll 1
                for (int t = 0; t <= ix + jx; ++t)
#pragma unroll 1
                    for (int u = 0; u <= iy + jy; ++u)
#pragma unroll 1
                        for (int v = 0; v <= iz + jz; ++v)
                            et[tet(t, u, v)] += w2 * ex.e[ix][jx][t] * ey.e[iy][jy][u] * ez.e[iz][jz][v];
            }
        }
    }
    __syncthreads();
    return nk;
}

// Shapes of one (P|mu nu) class. The threads of an auxiliary shell (one per
// m_P, all in one warp) share each primitive triple's R table: per round, TPR
// of them each evaluate the Boys function and R table of one triple into
// shared memory, and after a warp barrier every thread contracts all TPR tables
// with its own m_P row of the Cartesian-to-spherical matrix. TPR is NSP unless
// the tables would pass kRTableBytes (the high classes, whose tables hold up to
// 165 entries). For l_P = 0 each shell has one thread, which keeps its table in
// registers.
constexpr int kRTableBytes = 48 * 1024;
template <int LA, int LB, int LP>
struct ThreeCenterShape {
    static constexpr int L = LA + LB + LP;
    static constexpr int NCP = ncart(LP), NSP = nsph(LP);
    static constexpr int SPW = 32 / NSP;  // auxiliary shells per warp
    static constexpr int SPB = 4 * SPW;   // ... per 128-thread CTA
    static constexpr int NH = ntet(LA + LB);
    static constexpr int NR = ntet(L);
    // the table and its prefactor, padded to an odd count of doubles so that
    // rows of consecutive threads fall in different banks
    static constexpr int RS = (NR + 1) | 1;
    static constexpr int FIT = kRTableBytes / (SPB * RS * 8);
    static constexpr int TPR = NSP == 1 ? 1 : (FIT < 1 ? 1 : (FIT > NSP ? NSP : FIT));
    static constexpr int R_DOUBLES = NSP == 1 ? 0 : SPB * TPR * RS;
};

// One CTA per orbital shell pair of class (LA <= LB) and a slab of SPB auxiliary
// shells of class LP; thread (slot, m_P) accumulates the pair's NSAB x KK block
// of (P m_P | mu nu) for the slot's shell. The pair's primitive data and
// spherical Hermite coefficients sit in shared memory (broadcast reads), so do
// the round's R tables (rows of RS doubles, read by the slot's threads).
template <int LA, int LB, int LP>
__global__ void __launch_bounds__(128) k_three_center(const PairTask* __restrict__ tasks,
                                                      const DevShell* __restrict__ orb,
                                                      const DevShell* __restrict__ aux,
                                                      const double* __restrict__ exps,
                                                      const double* __restrict__ coefs,
                                                      const int* __restrict__ alist, int nalist,
                                                      const double* __restrict__ btable, ChunkDesc chunk,
                                                      int r_offset, double* __restrict__ T) {
    using PL = PairLayout<LA, LB>;
    using SH = ThreeCenterShape<LA, LB, LP>;
    constexpr int L = SH::L, NCP = SH::NCP, NSP = SH::NSP, SPW = SH::SPW, NH = SH::NH, TPR = SH::TPR;
    constexpr int RS = SH::RS, NR = SH::NR;
    extern __shared__ double smem[];
    __shared__ int s_pos[2 * kMaxPrimPairs + 1];
    __shared__ int s_idx[NCP * NH];      // tet(h + c) for Cartesian c of l_P, Hermite h of the pair
    __shared__ int s_nzc[NSP * NCP];     // per m_P: the Cartesian components with a nonzero weight
    __shared__ double s_nzw[NSP * NCP];  // ... and the weights
    __shared__ int s_nnz[NSP];
    __shared__ int s_tp[SH::SPB * TPR];  // primitive pair of each table of the round, -1 past the end
    double* sR = smem + r_offset;

    for (int e = threadIdx.x; e < NCP * NH; e += blockDim.x) {
        const int c = e / NH, h = e - c * NH;
        s_idx[e] = tet(c_tet_t[h] + c_cart[LP][c][0], c_tet_u[h] + c_cart[LP][c][1], c_tet_v[h] + c_cart[LP][c][2]);
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

    const PairTask task = tasks[blockIdx.x];
    const DevShell A = orb[task.swap ? task.second : task.first];
    const DevShell B = orb[task.swap ? task.first : task.second];
    const int npp = pair_prologue<LA, LB>(A, B, exps, coefs, smem, s_pos);  // ends with a barrier
    if (npp == 0) return;  // the same for the whole CTA; the chunk was zeroed

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wslot = lane / NSP, mp = lane - wslot * NSP;
    const int slot = warp * SPW + wslot;
    const int ia = blockIdx.y * SH::SPB + slot;
    const bool active = wslot < SPW && ia < nalist;
    DevShell P{};
    int ntrip = 0;
    if (active) {
        P = aux[alist[ia]];
        ntrip = P.nprim * npp;
    }
    // rounds of this warp: its slowest shell's triples over TPR
    const int rounds = __reduce_max_sync(0xffffffffu, (ntrip + TPR - 1) / TPR);
    const int nnz = s_nnz[active ? mp : 0];

    double acc[PL::KK][PL::NSAB];
#pragma unroll
    for (int k = 0; k < PL::KK; ++k)
#pragma unroll
        for (int m = 0; m < PL::NSAB; ++m) acc[k][m] = 0.0;

    // this thread's triple t = r TPR + mp as (auxiliary primitive i, primitive pair pp),
    // advanced by TPR per round; the auxiliary primitive's factors are kept while i stays
    int ti = mp / npp, tpp = mp - (mp / npp) * npp;
    int ci = -1;
    double q = 0.0, cq = 0.0;
    for (int r = 0; r < rounds; ++r) {
        int pp = -1;
        double R[NSP == 1 ? NR : 1];
        if (active && mp < TPR && ti < P.nprim) {
            pp = tpp;
            if (ti != ci) {
                ci = ti;
                q = exps[P.prim + ti];
                const double inv_q = 1.0 / q;
                // c_P (2q)^-l_P (-1)^l_P 2 pi^(5/2) / q
                cq = coefs[P.coef + ti] * kTwoPi52 * inv_q;
                const double h2q = 0.5 * inv_q;
#pragma unroll
                for (int k = 0; k < LP; ++k) cq *= h2q;
                if (LP & 1) cq = -cq;
            }
            const double* s = smem + pp * PL::STRIDE;
            const double p = s[0];
            // one division per primitive triple: 1/(p+q) gives both the reduced
            // exponent and the prefactor 2 pi^(5/2) / (p q sqrt(p+q))
            const double inv_pq = 1.0 / (p + q);
            const double alpha = p * q * inv_pq;
            const double pref = s[4] * sqrt(inv_pq) * cq;
            if constexpr (NSP == 1) {
                hermite_r<L>(alpha, s[1] - P.x, s[2] - P.y, s[3] - P.z, btable, R);
                const double scale = pref * c_c2s[c2s_offset(LP)];  // the single weight of l_P = 0
#pragma unroll
                for (int e = 0; e < NR; ++e) R[e] *= scale;
            } else {
                double* row = sR + (slot * TPR + mp) * RS;
                if constexpr (L <= 4) {
                    double Rr[NR];
                    hermite_r<L>(alpha, s[1] - P.x, s[2] - P.y, s[3] - P.z, btable, Rr);
#pragma unroll
                    for (int e = 0; e < NR; ++e) row[e] = Rr[e];
                } else {
                    hermite_r<L>(alpha, s[1] - P.x, s[2] - P.y, s[3] - P.z, btable, row);
                }
                row[NR] = pref;
            }
            tpp += TPR;
            while (tpp >= npp) {
                tpp -= npp;
                ++ti;
            }
        }
        if constexpr (NSP == 1) {
            // l_P = 0: one thread per shell, the table (weight and prefactor
            // applied) in registers
            if (pp >= 0) {
                const double* s = smem + pp * PL::STRIDE;
                const double* et = s + PL::ET;
#pragma unroll
                for (int m = 0; m < PL::NSAB; ++m) {
                    double val = 0.0;
#pragma unroll
                    for (int h = 0; h < NH; ++h) val += et[m * NH + h] * R[h];
#pragma unroll
                    for (int k = 0; k < PL::KK; ++k) acc[k][m] += s[PL::CC + k] * val;
                }
            }
        } else {
            if (active && mp < TPR) s_tp[slot * TPR + mp] = pp;
            __syncwarp();
            if (active) {
#pragma unroll 1
                for (int j = 0; j < TPR; ++j) {
                    const int pj = s_tp[slot * TPR + j];
                    if (pj < 0) break;
                    const double* row = sR + (slot * TPR + j) * RS;
                    double G[NH];
#pragma unroll
                    for (int h = 0; h < NH; ++h) G[h] = 0.0;
#pragma unroll 1
                    for (int k = 0; k < nnz; ++k) {
                        const int* ix = s_idx + s_nzc[mp * NCP + k] * NH;
                        const double w = s_nzw[mp * NCP + k];
#pragma unroll
                        for (int h = 0; h < NH; ++h) G[h] += w * row[ix[h]];
                    }
                    const double pref = row[NR];
                    const double* s = smem + pj * PL::STRIDE;
                    const double* et = s + PL::ET;
#pragma unroll
                    for (int m = 0; m < PL::NSAB; ++m) {
                        double val = 0.0;
#pragma unroll
                        for (int h = 0; h < NH; ++h) val += et[m * NH + h] * G[h];
                        val *= pref;
#pragma unroll
                        for (int k = 0; k < PL::KK; ++k) acc[k][m] += s[PL::CC + k] * val;
                    }
                }
            }
            __syncwarp();
        }
    }
    if (!active) return;

    // Scatter into the chunk: element (mu, nu) in AO order, both orders where the
    // tile is on or above the diagonal and its row belongs to this chunk.
    const int same = task.first == task.second;
    const int q0 = P.fn + mp;
#pragma unroll
    for (int ka = 0; ka < PL::KA; ++ka)
#pragma unroll
        for (int kb = 0; kb < PL::KB; ++kb) {
            if (ka >= A.ncontr || kb >= B.ncontr) continue;
#pragma unroll
            for (int ma = 0; ma < PL::NSA; ++ma)
#pragma unroll
                for (int mb = 0; mb < PL::NSB; ++mb) {
                    const double v = acc[ka * PL::KB + kb][ma * PL::NSB + mb];
                    int mu = A.fn + ka * PL::NSA + ma;
                    int nu = B.fn + kb * PL::NSB + mb;
                    if (task.swap) {
                        const int tmp = mu;
                        mu = nu;
                        nu = tmp;
                    }
                    if (same && mu > nu) continue;
#pragma unroll
                    for (int o = 0; o < 2; ++o) {
                        const int r = (o ? nu : mu), c = (o ? mu : nu);
                        if (o && r == c) break;
                        const int tr = r >> 6, tc = c >> 6;
                        if (tr < chunk.row0 || tr >= chunk.row1 || tc < tr) continue;
                        const int64_t col = (tile_index(tr, tc, chunk.nt) - chunk.tile_base) * 4096 +
                                            (r & 63) * 64 + (c & 63);
                        T[col * chunk.ld + q0] = v;
                    }
                }
        }
}

template <int LA, int LB, int LP>
static cudaError_t three_center_one(const PairTask* tasks, int ntasks, int max_npp, const DevShell* orb,
                                    const DevShell* aux, const double* exps, const double* coefs,
                                    const int* alist, int nalist, const double* btable, ChunkDesc chunk,
                                    double* T, cudaStream_t stream) {
    if (ntasks == 0 || nalist == 0) return cudaSuccess;
    using SH = ThreeCenterShape<LA, LB, LP>;
    const int r_offset = max_npp * PairLayout<LA, LB>::STRIDE;
    const size_t smem = sizeof(double) * ((size_t)r_offset + SH::R_DOUBLES);
    // the attribute covers the dynamic part; the static tables count against
    // the 48 KB default too
    if (smem > 40 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_three_center<LA, LB, LP>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    dim3 grid(ntasks, (nalist + SH::SPB - 1) / SH::SPB);  // 4 warps of SPW shells
    k_three_center<LA, LB, LP><<<grid, 128, smem, stream>>>(tasks, orb, aux, exps, coefs, alist, nalist, btable,
                                                            chunk, r_offset, T);
    return cudaGetLastError();
}

cudaError_t launch_three_center(int la, int lb, const PairTask* tasks, int ntasks, int max_npp, const DevShell* orb,
                                const DevShell* aux, const double* exps, const double* coefs,
                                const int* const* aux_by_l, const int* count, const double* btable,
                                ChunkDesc chunk, double* T, cudaStream_t stream) {
    cudaError_t e = cudaSuccess;
#define HF_3C(LA, LB, LP)                                                                                     \
    if (e == cudaSuccess && la == LA && lb == LB)                                                             \
        e = three_center_one<LA, LB, LP>(tasks, ntasks, max_npp, orb, aux, exps, coefs, aux_by_l[LP], count[LP], \
                                         btable, chunk, T, stream);
#define HF_3C_P(LA, LB) HF_3C(LA, LB, 0) HF_3C(LA, LB, 1) HF_3C(LA, LB, 2) HF_3C(LA, LB, 3) HF_3C(LA, LB, 4)
    HF_3C_P(0, 0)
    HF_3C_P(0, 1)
    HF_3C_P(0, 2)
    HF_3C_P(1, 1)
    HF_3C_P(1, 2)
    HF_3C_P(2, 2)
#undef HF_3C_P
#undef HF_3C
    return e;
}

// ---------------------------------------------------------- S, T and V
template <int LA, int LB, int KIND>
__global__ void __launch_bounds__(128) k_one_electron(const int2* __restrict__ tasks, int ntasks,
                                                      const DevShell* __restrict__ orb,
                                                      const double* __restrict__ exps,
                                                      const double* __restrict__ coefs,
                                                      const double* __restrict__ charges,
                                                      const double* __restrict__ positions, int natoms,
                                                      const double* __restrict__ btable, double* __restrict__ out,
                                                      int64_t n) {
    constexpr int NCA = ncart(LA), NCB = ncart(LB), NSA = nsph(LA), NSB = nsph(LB);
    constexpr int KA = kMaxOrbContr[LA], KB = kMaxOrbContr[LB];
    constexpr int XB = (KIND == 1) ? 2 : 0;
    constexpr int LAB = LA + LB;
    // the attraction spreads its sum over the nuclei across the 32 lanes of a warp
    // (one warp per shell pair; small molecules otherwise leave most SMs idle)
    constexpr int LANES = (KIND == 2) ? 32 : 1;
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    const int t = gt / LANES, lane = gt % LANES;
    if (t >= ntasks) return;  // a whole warp at a time when LANES = 32
    const int2 task = tasks[t];
    const DevShell A = orb[task.x];
    const DevShell B = orb[task.y];
    double acc[KA * KB][NSA * NSB];
#pragma unroll
    for (int k = 0; k < KA * KB; ++k)
#pragma unroll
        for (int m = 0; m < NSA * NSB; ++m) acc[k][m] = 0.0;
    const double abx = A.x - B.x, aby = A.y - B.y, abz = A.z - B.z;
    const double rab2 = abx * abx + aby * aby + abz * abz;
    for (int i = 0; i < A.nprim; ++i)
        for (int j = 0; j < B.nprim; ++j) {
            const double a = exps[A.prim + i], b = exps[B.prim + j];
            const double p = a + b, mu = a * b / p;
            const double px = (a * A.x + b * B.x) / p, py = (a * A.y + b * B.y) / p, pz = (a * A.z + b * B.z) / p;
            Hermite1D<LA, LB + XB> ex, ey, ez;
            ex.build(p, exp(-mu * rab2), px - A.x, px - B.x);
            ey.build(p, 1.0, py - A.y, py - B.y);
            ez.build(p, 1.0, pz - A.z, pz - B.z);
            double cart[NCA][NCB];
            if (KIND == 2) {
                double Rs[ntet(LAB)];
#pragma unroll
                for (int h = 0; h < ntet(LAB); ++h) Rs[h] = 0.0;
                for (int c = lane; c < natoms; c += LANES) {
                    double R[ntet(LAB)];
                    hermite_r<LAB>(p, px - positions[3 * c], py - positions[3 * c + 1], pz - positions[3 * c + 2],
                                   btable, R);
                    const double z = charges[c];
#pragma unroll
                    for (int h = 0; h < ntet(LAB); ++h) Rs[h] -= z * R[h];
                }
                if constexpr (LANES > 1) {
#pragma unroll
                    for (int h = 0; h < ntet(LAB); ++h)
#pragma unroll
                        for (int o = LANES / 2; o > 0; o >>= 1) Rs[h] += __shfl_xor_sync(0xffffffffu, Rs[h], o);
                }
                const double pref = 2.0 * kPi / p;
#pragma unroll
                for (int ca = 0; ca < NCA; ++ca)
#pragma unroll
                    for (int cb = 0; cb < NCB; ++cb) {
                        const int ix = cart_x(LA, ca), iy = cart_y(LA, ca), iz = cart_z(LA, ca);
                        const int jx = cart_x(LB, cb), jy = cart_y(LB, cb), jz = cart_z(LB, cb);
                        double s = 0.0;
#pragma unroll
                        for (int tt = 0; tt <= ix + jx; ++tt)
#pragma unroll
                            for (int u = 0; u <= iy + jy; ++u)
#pragma unroll
                                for (int v = 0; v <= iz + jz; ++v)
                                    s += ex.e[ix][jx][tt] * ey.e[iy][jy][u] * ez.e[iz][jz][v] * Rs[tet(tt, u, v)];
                        cart[ca][cb] = pref * s;
                    }
            } else {
                const double ov = pow(kPi / p, 1.5);
#pragma unroll
                for (int ca = 0; ca < NCA; ++ca)
#pragma unroll
                    for (int cb = 0; cb < NCB; ++cb) {
                        const int ix = cart_x(LA, ca), iy = cart_y(LA, ca), iz = cart_z(LA, ca);
                        const int jx = cart_x(LB, cb), jy = cart_y(LB, cb), jz = cart_z(LB, cb);
                        const double sx = ex.e[ix][jx][0], sy = ey.e[iy][jy][0], sz = ez.e[iz][jz][0];
                        if (KIND == 0) {
                            cart[ca][cb] = ov * sx * sy * sz;
                        } else {
                            // <x^i | d^2/dx^2 | x^j> / sqrt(pi/p) (pairs.rs:41-52, Helgaker 9.3.33)
                            auto d2 = [&](const Hermite1D<LA, LB + XB>& e, int ii, int jj) {
                                double v = 4.0 * b * b * e.e[ii][jj + 2 < LB + XB + 1 ? jj + 2 : 0][0] -
                                           2.0 * b * (2 * jj + 1) * e.e[ii][jj][0];
                                if (jj >= 2) v += jj * (jj - 1) * e.e[ii][jj - 2][0];
                                return v;
                            };
                            cart[ca][cb] = -0.5 * ov *
                                           (d2(ex, ix, jx) * sy * sz + sx * d2(ey, iy, jy) * sz + sx * sy * d2(ez, iz, jz));
                        }
                    }
            }
#pragma unroll
            for (int ma = 0; ma < NSA; ++ma)
#pragma unroll
                for (int mb = 0; mb < NSB; ++mb) {
                    double s = 0.0;
#pragma unroll
                    for (int ca = 0; ca < NCA; ++ca) {
                        const double ta = c_c2s[c2s_offset(LA) + ma * NCA + ca];
                        if (ta == 0.0) continue;
#pragma unroll
                        for (int cb = 0; cb < NCB; ++cb) s += ta * c_c2s[c2s_offset(LB) + mb * NCB + cb] * cart[ca][cb];
                    }
#pragma unroll
                    for (int ka = 0; ka < KA; ++ka)
#pragma unroll
                        for (int kb = 0; kb < KB; ++kb) {
                            if (ka >= A.ncontr || kb >= B.ncontr) continue;
                            acc[ka * KB + kb][ma * NSB + mb] +=
                                coefs[A.coef + ka * A.nprim + i] * coefs[B.coef + kb * B.nprim + j] * s;
                        }
                }
        }
    if (lane != 0) return;
#pragma unroll
    for (int ka = 0; ka < KA; ++ka)
#pragma unroll
        for (int kb = 0; kb < KB; ++kb) {
            if (ka >= A.ncontr || kb >= B.ncontr) continue;
#pragma unroll
            for (int ma = 0; ma < NSA; ++ma)
#pragma unroll
                for (int mb = 0; mb < NSB; ++mb)
                    out[(int64_t)(A.fn + ka * NSA + ma) * n + B.fn + kb * NSB + mb] = acc[ka * KB + kb][ma * NSB + mb];
        }
}

template <int LA, int LB, int KIND>
static cudaError_t one_electron_one(const int2* tasks, int ntasks, const DevShell* orb, const double* exps,
                                    const double* coefs, const double* charges, const double* positions, int natoms,
                                    const double* btable, double* out, int64_t n, cudaStream_t stream) {
    if (ntasks == 0) return cudaSuccess;
    const int64_t threads = (int64_t)ntasks * (KIND == 2 ? 32 : 1);
    k_one_electron<LA, LB, KIND><<<(unsigned)((threads + 127) / 128), 128, 0, stream>>>(
        tasks, ntasks, orb, exps, coefs, charges, positions, natoms, btable, out, n);
    return cudaGetLastError();
}

cudaError_t launch_one_electron(int kind, int la, int lb, const int2* tasks, int ntasks, const DevShell* orb,
                                const double* exps, const double* coefs, const double* charges,
                                const double* positions, int natoms, const double* btable, double* out, int64_t n,
                                cudaStream_t stream) {
    cudaError_t e = cudaSuccess;
#define HF_1E(K, LA, LB)                                                                                        \
    if (kind == K && la == LA && lb == LB)                                                                      \
        e = one_electron_one<LA, LB, K>(tasks, ntasks, orb, exps, coefs, charges, positions, natoms, btable, out, \
                                        n, stream);
#define HF_1E_K(K)                                                                                  \
    HF_1E(K, 0, 0) HF_1E(K, 0, 1) HF_1E(K, 0, 2) HF_1E(K, 1, 0) HF_1E(K, 1, 1) HF_1E(K, 1, 2) HF_1E(K, 2, 0) \
    HF_1E(K, 2, 1) HF_1E(K, 2, 2)
    HF_1E_K(0)
    HF_1E_K(1)
    HF_1E_K(2)
#undef HF_1E_K
#undef HF_1E
    return e;
}

}  // namespace hf

#include "four_center.cuh"
