/* hfbatch.h: batched, graph-resident restricted SCF over many clusters.
 *
 * A device restatement of the reference's restricted SCF driver run for many
 * molecules at once:
 *   hafnium/scf/driver.py:154-213, 331-366  solve_scf loop and finish
 *   hafnium/scf/diis.py:55-106              DIIS history, overlaps and solve
 *   hafnium/scf/hamiltonian.py:331-370      restricted Fock build and energy
 *   hafnium/scf/coulomb_exchange.py:176-190 J and K from the fitted tensor
 * Clusters of one batch share their shape (orbital and auxiliary counts and
 * occupation); each keeps its own fitted tensor in its own hf_ctx. Every SCF
 * iteration of every cluster runs inside one CUDA graph: the loop over
 * iterations is a device-side conditional (WHILE) node, so one graph launch
 * converges the whole batch. Several batches of different shapes can share
 * one graph launch (hf_batch_run_group).
 *
 * Differences from the reference driver, chosen so every step is a batched
 * kernel: the orthonormal basis is X = L^-T from the overlap's Cholesky factor
 * (S = L L^T; the reference uses the canonical X = U s^-1/2 and gives the same
 * SCF whenever no overlap eigenvalue falls below its 1e-10 drop threshold,
 * which hf_batch_load checks through a bound), and the aufbau density of each
 * Fock matrix comes from canonical purification (Palser and Manolopoulos,
 * Phys. Rev. B 58, 12704 (1998)) on FP64 tensor cores instead of an
 * eigendecomposition; both give the projector onto the n_occ lowest orbitals.
 * The DIIS system is solved as in the reference: an eigendecomposition of the
 * bordered, scaled overlap matrix with eigenvalues below 1e-14 of the largest
 * dropped.
 */
#ifndef HFBATCH_H
#define HFBATCH_H

#include <stdint.h>

#include "hfjk.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hf_batch hf_batch;

#define HF_BATCH_MAX_CLUSTERS 4096
#define HF_BATCH_MAX_DIIS 8

/* Per-cluster outcome (hf_batch_results). */
typedef enum hf_batch_state {
    HF_SCF_ITERATING = 0,
    HF_SCF_FINISHING = 1, /* converged; the final Fock build is pending */
    HF_SCF_CONVERGED = 2,
    HF_SCF_NOT_CONVERGED = 3,  /* max_iterations reached (reference: ConvergenceError) */
    HF_SCF_PURIFICATION_FAILED = 4 /* no gap: purification did not converge */
} hf_batch_state;

typedef struct hf_batch_options {
    int max_iterations;        /* reference ScfOptions default 100 */
    int diis_size;             /* 1..HF_BATCH_MAX_DIIS, reference default 8 */
    double energy_tolerance;   /* reference default 1e-10 */
    double gradient_tolerance; /* reference default 1e-6 */
    int purify_steps;          /* purification steps captured per iteration (1..128) */
    double purify_tolerance;   /* tr(P - P^2) below which one more step ends purification */
    int gemm_tile;             /* DMMA tile shape for the n x n products (0..5, see hf_dgemm_nt) */
    int use_graph;             /* 1: one CUDA graph with a device-side loop; 0: host loop */
} hf_batch_options;

/* Fills the reference defaults. */
int hf_batch_default_options(hf_batch_options* out);

/* A batch over `count` built contexts on one device with equal n_ao and n_aux;
 * n_occ doubly occupied orbitals each. Allocates all batch state. */
int hf_batch_create(hf_ctx* const* clusters, int count, int64_t n_occ, hf_batch** out);
int hf_batch_destroy(hf_batch* batch);
const char* hf_batch_last_error(const hf_batch* batch);
int hf_batch_set_stream(hf_batch* batch, void* stream);
int hf_batch_dims(const hf_batch* batch, int* count, int64_t* n_ao, int64_t* n_aux, int64_t* n_occ);

/* Per-cluster inputs, device arrays of count x n x n (row-major): overlap S,
 * core Hamiltonian H and the starting density D0 (alpha spin); host array of
 * count nuclear repulsion energies. guess_rank bounds the rank of every D0
 * (n_ao when unknown). Fails with HF_ERR_NUMERIC if some S is not positive
 * definite or may have an eigenvalue below the reference's drop threshold. */
int hf_batch_load(hf_batch* batch, const double* overlap, const double* core, const double* guess,
                  const double* nuclear_repulsion, int64_t guess_rank);

/* Converges every loaded cluster (the reference's solve_scf + finish). */
int hf_batch_run(hf_batch* batch, const hf_batch_options* options);

/* All batches in one graph launch (one stream each, forked inside the graph). */
int hf_batch_run_group(hf_batch* const* batches, int count, const hf_batch_options* options);

/* Host outputs (any may be NULL): final energies [count], Fock builds inside
 * the loop [count] (the reference's len(history)), hf_batch_state [count];
 * densities: device, count x n x n. */
int hf_batch_results(hf_batch* batch, double* energies, int* iterations, int* states, double* densities);

/* Batched J = J(scale D) and K(D) over the batch's tensors (device arrays,
 * count x n x n); K factors every D by pivoted Cholesky (rank <= max_rank). */
int hf_batch_coulomb(hf_batch* batch, const double* density, double scale, double* coulomb);
int hf_batch_exchange(hf_batch* batch, const double* density, int64_t max_rank, double* exchange);

/* Strided-batched FP64 tensor-core GEMM, C = alpha A B^T + beta C, for the
 * tile autotuner: A [m][k] (lda), B [n][k] (ldb), C [m][n] (ldc), device
 * pointers advanced by the strides per batch; tile 0..5 selects the CTA tile
 * 128x64, 64x64, 64x32, 32x32, 128x128 (3 stages of 16-wide k slices) or
 * 64x64 with 2 stages of 32-wide k slices. */
int hf_dgemm_nt(int64_t m, int64_t n, int64_t k, const double* a, int64_t lda, int64_t stride_a, const double* b,
                int64_t ldb, int64_t stride_b, double* c, int64_t ldc, int64_t stride_c, double alpha, double beta,
                int batch, int tile, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* HFBATCH_H */
