/* hfjk.h: C ABI of the B200 density-fitted Coulomb/exchange (J/K) builder.
 *
 * A drop-in for the molecular DensityFittedCoulombExchange of maxnus/hafnium:
 *   hafnium/scf/coulomb_exchange.py:53-71   CoulombExchange protocol (n_ao, coulomb, exchange)
 *   hafnium/scf/coulomb_exchange.py:125-190 DensityFittedCoulombExchange (from_molecule, J, K)
 *   hafnium/integrals/density_fitting.py:59-107 DensityFitting.build / df_tensor
 *   hafnium/integrals/native.py:16-24, 104-177 RustEngine 2c/3c + ShellTable marshalling
 *   crates/hafnium-py/src/lib.rs:66-108, 352-423 the PyO3 entry points the shell table crosses
 *
 * Conventions: plain pointers and sizes, no exceptions cross this boundary,
 * every entry point returns an hf_status. Host arrays are caller-owned; device
 * arrays passed with on_device = 1 are raw CUDA pointers on the context's device.
 * Matrices are row-major float64. One context per host thread / stream.
 */
#ifndef HFJK_H
#define HFJK_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum hf_status {
    HF_OK = 0,
    HF_ERR_ARG = 1,      /* invalid argument or shell table (reference: ValueError, lib.rs:1118) */
    HF_ERR_OOM = 2,      /* device allocation failed */
    HF_ERR_CUDA = 3,     /* CUDA runtime error; see hf_last_error */
    HF_ERR_TIMEOUT = 4,  /* a bounded device wait ran out */
    HF_ERR_NUMERIC = 5,  /* metric not positive definite, or density not factorisable */
    HF_ERR_STATE = 6     /* call order: shells not uploaded / tensor not built */
} hf_status;

typedef struct hf_ctx hf_ctx;

/* Shells in structure-of-arrays form, the layout of hafnium's ShellTable
 * (hafnium/integrals/shell_table.py:14-82, crates/.../integrals/mod.rs:63-173):
 * one entry per shell with all its contractions; coefficients of bare
 * primitives stored shell by shell as [contraction][primitive]. */
typedef struct hf_shell_table {
    int64_t n_shells;
    const int64_t* angular_momenta;   /* [n_shells] */
    const double* centers;            /* [n_shells][3], Bohr */
    const int64_t* primitive_offsets; /* [n_shells + 1] */
    const double* exponents;          /* [primitive_offsets[n_shells]] */
    const double* coefficients;       /* [sum_s n_contractions[s] * n_prim(s)] */
    const int64_t* n_contractions;    /* [n_shells] */
} hf_shell_table;

typedef enum hf_precision {
    HF_PREC_FP64 = 0,      /* FP64 DMMA tensor cores */
    HF_PREC_BF16X3 = 1     /* 3 split-BF16 products, FP32 accumulation (tcgen05) */
} hf_precision;

/* The mixed-precision exchange schedule behind hf_exchange_scheduled. */
typedef enum hf_schedule_mode {
    HF_SCHEDULE_FP64 = 0,  /* every build FP64 */
    HF_SCHEDULE_MIXED = 1  /* split-BF16, FP64 anchor, anchored increments, late re-anchor */
} hf_schedule_mode;

typedef struct hf_schedule {
    int mode;               /* hf_schedule_mode */
    double anchor_change;   /* split-BF16 while max|D_n - D_(n-1)| >= this (1e-3) */
    double final_change;    /* one more FP64 anchor once the change is below this while
                               the anchor lies farther than it (1e-5) */
} hf_schedule;

/* What a scheduled build computed. */
typedef enum hf_build_kind {
    HF_BUILD_FP64 = 0,        /* FP64 (HF_SCHEDULE_FP64) */
    HF_BUILD_BF16 = 1,        /* split-BF16 from the density's factor */
    HF_BUILD_ANCHOR = 2,      /* FP64, kept as the anchor */
    HF_BUILD_INCREMENTAL = 3  /* anchor + split-BF16 of the exactly factored difference */
} hf_build_kind;

typedef struct hf_stats {
    double ms_metric;       /* (P|Q) */
    double ms_factor;       /* Cholesky + inverse of the factor */
    double ms_three_center; /* (P|mu nu), all chunks */
    double ms_fit;          /* B = L^-1 (P|mu nu), all chunks */
    double ms_coulomb;      /* last J build */
    double ms_exchange;     /* last K build */
    double ms_factorize_density; /* last pivoted Cholesky of D (hf_exchange) */
    double min_pivot_ratio; /* min Cholesky pivot^2 / max metric diagonal */
    int64_t n_ao, n_aux, n_tiles;
    int64_t b_bytes;        /* bytes of the packed fitted tensor */
    int64_t exchange_rank;  /* columns of the last exchange factor */
    int64_t kernel_launches;/* launches issued by this context so far */
    double ms_gradient_weights; /* last gradient: densities, metric factor, Gamma, metric weights */
    double ms_gradient_metric;  /* last gradient: (dP P|Q) against the metric weights */
    double ms_gradient_three_center; /* last gradient: exchange weights and (dP P|uv), (P|dA uv) */
    double ms_gradient_one_electron; /* last gradient: S, T, V derivatives */
    int64_t device_allocations; /* cudaMalloc / cudaMallocAsync calls made for this context so far */
} hf_stats;

/* Context lifetime (no reference counterpart: the reference's kernels are
 * stateless functions over host arrays). */
int hf_ctx_create(int device, hf_ctx** out);
int hf_ctx_destroy(hf_ctx* ctx);
const char* hf_last_error(const hf_ctx* ctx);
/* Launch on this stream (cudaStream_t) from now on; NULL = the context's own.
 * Waits for the work queued on the previous stream first (unless that stream
 * is being captured), since the context's blocks are released in the order of
 * its current stream. */
int hf_set_stream(hf_ctx* ctx, void* stream);

/* The device blocks of fitted tensors, their BF16 copies and the J/K scratch
 * areas, when at least 256 MiB, are not freed when a context is destroyed or
 * rebuilt: up to eight per device are kept and handed to the next context
 * whose request fits, so a run over many geometries of one size maps them
 * once (smaller blocks come from the device's stream-ordered pool and go back
 * to it without a device-wide synchronisation). A failed allocation empties
 * the cache first. This frees the blocks kept for `device` now. No reference counterpart (the reference holds host
 * arrays only). */
int hf_release_retained(int device);

/* Limit of every device-side wait of the split-BF16 exchange's pipeline (its
 * mbarrier waits), in nanoseconds, 1 us .. 60 s; 2 s by default. A wait that
 * runs out ends the kernel cleanly (in-flight copies drained, tensor memory
 * freed) and the build returns HF_ERR_TIMEOUT; the context stays usable. With
 * stall_next_build set, the next split-BF16 build waits once on a barrier that
 * nothing completes, so that path can be tested without a fault. No reference
 * counterpart (the reference has no device code). */
int hf_set_wait_limit(hf_ctx* ctx, int64_t wait_ns, int stall_next_build);

/* Upload the orbital and auxiliary shells (replaces the _kernels.ShellTable
 * marshalling of native.py:16-24; validation of integrals/mod.rs:111-173).
 * auxiliary may be NULL when only one-electron / four-centre integrals are wanted. */
int hf_shells_upload(hf_ctx* ctx, const hf_shell_table* orbital, const hf_shell_table* auxiliary);

/* (P|Q), its Cholesky factor and (P|mu nu) -> packed B = L^-1 (P|mu nu) on the
 * device (replaces DensityFitting.build + df_tensor, density_fitting.py:59-107,
 * and the Rust coulomb_two_center / coulomb_three_center, two_electron.rs:74-297). */
int hf_build_fitted_tensor(hf_ctx* ctx);

/* Hold only rows [row0, row1) of the fitted tensor (auxiliary functions in the
 * library's internal order: shells sorted by angular momentum), for a tensor
 * sharded over devices by auxiliary index. Call after hf_shells_upload and
 * before hf_build_fitted_tensor; the rows of all shards must cover
 * 0 .. n_aux - 1 once. J and K of such a context are the sums over its rows,
 * J = sum_{q in rows} (B_q . D) B_q and K = sum_{q in rows} B_q D B_q, which the
 * caller adds over the shards (an all-reduce of n_ao^2 doubles each); the
 * metric is factored in full on every shard, and the three-centre integrals of
 * the rows below row1 are computed. MP2, the orbital-basis tensor, the fitted
 * ERIs and the gradient need every row (HF_ERR_STATE otherwise). No reference
 * counterpart (the reference is not distributed). */
int hf_set_fitted_rows(hf_ctx* ctx, int64_t row0, int64_t row1);

int hf_dims(const hf_ctx* ctx, int64_t* n_ao, int64_t* n_aux);

/* J[u][v] = sum_wx (uv|wx) D[w][x] (coulomb_exchange.py:176-182). */
int hf_coulomb(hf_ctx* ctx, const double* density, double* coulomb, int on_device);

/* The J build of hf_coulomb without any device allocation, for callers that
 * cannot call cudaMalloc (a device pool already reserved by their own
 * allocator, or a loop where an allocation's device synchronisation is not
 * allowed). No counterpart in the reference. Density and J are device pointers;
 * scratch comes from a static device array of about 19.7 MB that every GPU
 * loading this library holds until exit, so n_ao <= 1536 and n_aux <= 8192
 * (HF_ERR_ARG beyond). Calls share that array: calls that overlap on the GPU
 * race. The first call on a device resolves the array's address; make it
 * before any stream capture. That address is kept for the life of the
 * process, so no call may follow a reset of the device (cudaDeviceReset) in
 * the same process. The call returns once J is complete: it waits for the
 * context's stream. */
int hf_coulomb_static(hf_ctx* ctx, const double* density, double* coulomb);

/* K for the density of one SCF iteration with the arithmetic chosen by the
 * schedule from the sequence of densities the context has been given
 * (hafnium/scf/coulomb_exchange.py:184-190 behind the reference driver's
 * per-iteration and finishing calls, hafnium/scf/driver.py:198-205, 336):
 * split-BF16 from the density's pivoted-Cholesky factor while the largest
 * element change from the previous call is at least anchor_change; then an
 * FP64 build kept as the anchor; then K64(D_a) + K16(V+) - K16(V-) with
 * D - D_a = V+ V+^T - V- V-^T from the factors (the anchor's rotated onto the
 * current one by the polar factor of F_a^T S F, a Newton-Schulz iteration of
 * matrix products; when it does not converge the build re-anchors in FP64);
 * once the change is below final_change while the anchor lies farther, one
 * more FP64 anchor. A jump of the change back above anchor_change restarts the
 * split-BF16 phase. *kind (may be NULL) receives hf_build_kind. The state is
 * the context's: one SCF at a time per context; hf_schedule_reset clears it.
 * HF_ERR_NUMERIC for an indefinite D. No reference counterpart (the reference
 * computes every K in FP64). */
int hf_exchange_scheduled(hf_ctx* ctx, const double* density, double* exchange, int on_device,
                          const hf_schedule* schedule, int* kind);
int hf_schedule_reset(hf_ctx* ctx);

/* A factor of a symmetric positive semidefinite density, D ~= F^T F: F holds
 * *rank rows of n_ao (row-major [rank][n_ao], capacity max_rank rows) from a
 * pivoted Cholesky stopped at 1e-14 of the largest diagonal element. It is the
 * factorisation hf_exchange makes internally; the drop-in's mixed-precision
 * exchange keeps it between calls to form difference densities. HF_ERR_NUMERIC
 * for an indefinite D. No reference counterpart (the reference contracts D). */
int hf_density_factor(hf_ctx* ctx, const double* density, double* factor, int64_t max_rank, int64_t* rank,
                      int on_device);

/* K[u][v] = sum_wx (uw|xv) D[w][x] (coulomb_exchange.py:184-190) for a symmetric
 * positive semidefinite D, factorised on the device by a pivoted Cholesky;
 * HF_ERR_NUMERIC when D is indefinite (use hf_exchange_factored then). */
int hf_exchange(hf_ctx* ctx, const double* density, double* exchange, int precision, int on_device);

/* K for D = C diag(w) C^T with C [n_ao][n_cols] row-major (w = NULL: all ones);
 * weights of either sign, in both precisions. */
int hf_exchange_factored(hf_ctx* ctx, const double* factor, int64_t n_cols, const double* weights,
                         double* exchange, int precision, int on_device);

/* Parity / inspection entry points (small systems). Reference order of the
 * auxiliary functions (the order of the auxiliary shell table). */
int hf_metric(hf_ctx* ctx, double* out /* [n_aux][n_aux] host */);
int hf_three_center(hf_ctx* ctx, double* out /* [n_aux][n_ao][n_ao] host */);
/* B^T B contracted on the auxiliary index, (uv|wx) fitted, [n][n][n][n] host. */
int hf_fitted_eri(hf_ctx* ctx, double* out);

/* One-electron integrals over the orbital shells (one_electron.rs:40-190):
 * kind 0 overlap, 1 kinetic, 2 attraction to point charges (charges [n_atoms],
 * positions [n_atoms][3] Bohr). out: [n_ao][n_ao]. */
int hf_one_electron(hf_ctx* ctx, int kind, const double* charges, const double* positions, int64_t n_atoms,
                    double* out, int on_device);

/* Exact (uv|wx) over the uploaded orbital shells, [n][n][n][n], n <= 128: the
 * atoms of the superposition-of-atomic-densities guess (hafnium/scf/atoms.py:55-73
 * with the Rust coulomb_four_center, two_electron.rs:429-935). */
int hf_four_center(hf_ctx* ctx, double* out, int on_device);

/* DF-MP2 correlation energy of a closed-shell reference from the context's
 * fitted tensor (hafnium/mp/mp2.py:68-176, df_mp2 + second_order, restricted
 * class, all electrons correlated): mo_coefficients [n_ao][n_mo] with the
 * orbitals in increasing energy (the first n_occ doubly occupied),
 * mo_energies [n_mo]; host or device arrays per on_device. */
int hf_mp2_energy(hf_ctx* ctx, const double* mo_coefficients, const double* mo_energies, int64_t n_mo, int64_t n_occ,
                  double* correlation, int on_device);

/* The fitted tensor in an orbital basis (hafnium/orbitals/integrals.py:73-157,
 * transform_df_tensor for restricted real orbitals without irrep sectors):
 * out[P][p][q] = sum_uv c_bra[u][p] B[P][u][v] c_ket[v][q], with c_bra
 * [n_ao][n_bra], c_ket [n_ao][n_ket]; host or device arrays per on_device.
 * B is the context's Cholesky-fitted tensor L^-1 (P|uv), whose auxiliary index
 * is an orthogonal rotation of the reference's M^-1/2 (P|uv): every contraction
 * over P (what the tensor's consumers form) is the reference's, the single
 * elements are not. */
int hf_mo_fitted_tensor(hf_ctx* ctx, const double* c_bra, int64_t n_bra, const double* c_ket, int64_t n_ket,
                        double* out, int on_device);

/* Analytic nuclear gradient of the DF-RHF energy of a converged closed-shell
 * state (hafnium/properties/gradient.py:72-149, nuclear_gradient, restricted
 * class): terms [5][natoms][3] in Hartree/Bohr, in the order nuclear
 * repulsion, one-electron, overlap, Coulomb, exchange (NuclearGradient,
 * gradient.py:44-69; their sum is the gradient). C: the occupied orbitals
 * [n_ao][nocc] (D = C C^T per spin); W: the energy-weighted density 2 D F D
 * [n_ao][n_ao]; charges [natoms] and positions [natoms][3] (Bohr) are host
 * arrays, and every shell must sit on one of those atoms. The derivative
 * integrals are contracted with their weights as they are formed, never
 * stored. C, W and terms are device pointers when on_device, else host.
 * Frees the context's split-BF16 copy of B when the intermediates would not
 * fit beside it (it is rebuilt on its next use). */
int hf_nuclear_gradient(hf_ctx* ctx, const double* C, int64_t nocc, const double* W, const double* charges,
                        const double* positions, int64_t natoms, double* terms, int on_device);

int hf_get_stats(const hf_ctx* ctx, hf_stats* out);

/* F_n(t), n = 0..n_max, for count arguments t (host arrays; out is
 * [count][n_max + 1]) by the device evaluation the integral kernels use: an
 * 8-term Taylor expansion on a 0.05 grid below t = 36, then downward
 * recursion; the large-t form and upward recursion above. Replaces the PyO3
 * boys_function (crates/hafnium-py/src/lib.rs:39-46, special.rs:34-51) for
 * testing the device path; n_max <= 9 (the integrals' highest order plus one
 * for their derivatives); a negative or non-finite t is HF_ERR_ARG. */
int hf_boys(hf_ctx* ctx, const double* t, int64_t count, int n_max, double* out);

#ifdef __cplusplus
}
#endif
#endif /* HFJK_H */
