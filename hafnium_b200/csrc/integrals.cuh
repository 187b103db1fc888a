// Host-visible declarations of the integral kernels' launch helpers.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "md.cuh"

namespace hf {

// One shell on the device. `fn` is the first orbital function (AO order) for
// orbital shells and the first internal auxiliary index for auxiliary shells.
struct DevShell {
    double x, y, z;
    int l, nprim, ncontr, prim, coef, fn;
};

// The part of the packed fitted tensor a three-centre launch fills: tile rows
// [row0, row1) of the upper triangle of 64x64 (mu, nu) tiles, laid out as
// T[col][q] with col = (tile - tile_base) * 4096 + (mu % 64) * 64 + nu % 64.
struct ChunkDesc {
    int row0, row1, nt;
    int64_t tile_base;
    int64_t ld;  // leading dimension (number of auxiliary functions, padded)
};

__host__ __device__ inline int64_t tile_index(int I, int J, int nt) {
    return (int64_t)I * nt - (int64_t)I * (I - 1) / 2 + (J - I);
}

// A shell pair task: orbital shells a <= b in AO order. `swap` marks a pair
// evaluated with the roles of a and b exchanged (so that l_first <= l_second).
struct PairTask {
    int first, second, swap, pad;
};

struct ShellClassLists {
    // orbital pairs bucketed by (la, lb) with la <= lb: 3x3 buckets (only la<=lb used)
    std::vector<PairTask> pairs[3][3];
    int max_npp[3][3] = {};
};

// The constant tables every integral kernel reads (each translation unit with
// such kernels holds its own __constant__ copy): Cartesian-to-spherical
// matrices, the (t, u, v) of each tetrahedral index up to order 8 and the
// Cartesian exponents per l.
struct ConstantTables {
    double c2s[kC2sSize];
    int tet_t[ntet(8)], tet_u[ntet(8)], tet_v[ntet(8)];
    int cart[kMaxAuxL + 1][15][3];
};
ConstantTables constant_tables_host();
void upload_c2s(cudaStream_t stream);
void upload_gradient_tables(cudaStream_t stream);
std::vector<double> boys_grid_host();
// The highest Boys order the device evaluation supports (the Taylor grid holds
// kBoysTerms orders above it).
constexpr int kBoysMaxOrder = kBoysOrders - kBoysTerms;
// F_0..F_n_max at count arguments t (device arrays) into out[count][n_max + 1].
cudaError_t launch_boys_values(const double* t, int64_t count, int n_max, const double* btable, double* out,
                               cudaStream_t stream);

// (P|Q) for all aux shells into M[N][N] (internal order, row-major, ld = ldm).
cudaError_t launch_metric(const DevShell* aux, const double* exps, const double* coefs,
                          const int* const* aux_by_l_dev, const int* aux_count, const double* btable,
                          double* M, int64_t ldm, cudaStream_t stream);

// (P|ab) for the given pair tasks of class (la, lb) and all aux shells, into a chunk.
cudaError_t launch_three_center(int la, int lb, const PairTask* tasks, int ntasks, int max_npp,
                                const DevShell* orb, const DevShell* aux, const double* exps,
                                const double* coefs, const int* const* aux_by_l_dev, const int* aux_count,
                                const double* btable, ChunkDesc chunk, double* T, cudaStream_t stream);

// S, T (kinetic) or V (attraction to point charges) over all ordered shell pairs
// of class (la, lb) into out[n][n] (AO order). kind: 0 S, 1 T, 2 V.
cudaError_t launch_one_electron(int kind, int la, int lb, const int2* tasks, int ntasks, const DevShell* orb,
                                const double* exps, const double* coefs, const double* charges,
                                const double* positions, int natoms, const double* btable, double* out,
                                int64_t n, cudaStream_t stream);

// Weights the contracted three-centre derivative kernels read: the total density
// D [n][n], the fitted Coulomb coefficients cfit [naux] (internal order) and the
// exchange weight GK [n][n][Pb] of the auxiliary functions [P0, P0 + Pb).
struct GradWeights {
    const double* D;
    const double* cfit;
    const double* GK;
    int64_t n;
    int P0;
    int64_t Pb;
};

// DF-RHF gradient pieces, contracted on the fly (gradient_kernels.cuh). Force
// sums per shell: gorb/gaux [shell][6] (Coulomb x y z, exchange x y z) for the
// fitted terms, gorb1 [shell][6] (one-electron, overlap) and gatom [atom][3]
// (the attraction's dependence on the nuclei).
// Per shell pair of a class: offsets[task] (doubles) into data of its Hermite
// data, npps[task] its primitive pairs kept (filled by launch_grad_pair_data).
struct GradPairData {
    const int64_t* offsets;
    double* data;
    int* npps;
};
cudaError_t launch_grad_pair_data(int la, int lb, const PairTask* tasks, int ntasks, int max_npp,
                                  const DevShell* orb, const double* exps, const double* coefs, const double* D,
                                  int64_t n, GradPairData pd, cudaStream_t stream);
cudaError_t launch_three_center_grad(int la, int lb, const PairTask* tasks, int ntasks, int max_npp,
                                     const DevShell* orb, const DevShell* aux, const double* exps,
                                     const double* coefs, const int* const* alist_by_l, const int* count_by_l,
                                     const double* btable, GradWeights g, GradPairData pd, double* gorb,
                                     double* gaux, cudaStream_t stream);
// Shared memory of one pair's data: max_npp primitive pairs of class (la, lb).
size_t three_center_grad_smem(int la, int lb, int max_npp);
// WK: only entries with row <= column are read (its upper triangle).
cudaError_t launch_metric_grad(const DevShell* aux, const double* exps, const double* coefs,
                               const int* const* aux_by_l, const int* count, const double* btable, const double* WJ,
                               const double* WK, int64_t ldw, double* gaux, cudaStream_t stream);
cudaError_t launch_one_electron_grad(int la, int lb, const int2* tasks, int ntasks, const DevShell* orb,
                                     const double* exps, const double* coefs, const double* charges,
                                     const double* positions, int natoms, const double* btable, const double* D,
                                     const double* W, int64_t n, double* gorb1, double* gatom, cudaStream_t stream);

// Exact (ab|cd) over all shell quartets of a small table into out[n][n][n][n].
cudaError_t launch_four_center(const DevShell* shells, int ns, const double* exps, const double* coefs,
                               const double* btable, double* out, int n, cudaStream_t stream);

}  // namespace hf
