/* hfnn.h: device kernels of the learned initial-density network (FP32).
 *
 * No counterpart in the reference: hafnium starts its SCF from the
 * superposition of atomic densities (hafnium/scf/atoms.py:76-120); this network
 * predicts a better starting density and falls back to that guess. The
 * network's layers are composed from these kernels by
 * hafnium_b200/learned/model.py. Pointers are device pointers; matrices are
 * row-major; stream is a cudaStream_t (NULL = the legacy default stream).
 * Every entry point returns 0 on success, 3 on a CUDA error.
 */
#ifndef HFNN_H
#define HFNN_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* C[m][n] (+)= op(A) op(B) + bias[n]; ta: A stored [k][m] (use A^T); tb: B stored [n][k]. */
int hfnn_sgemm(int m, int n, int k, const float* a, int ta, const float* b, int tb, const float* bias, float* c,
               int accumulate, void* stream);
/* y (+)= silu(z) * scale[row] (scale may be NULL). */
int hfnn_silu(int64_t rows, int cols, const float* z, const float* scale, float* y, int add, void* stream);
/* dz = dy * silu'(z) * scale[row]. */
int hfnn_dsilu(int64_t rows, int cols, const float* dy, const float* z, const float* scale, float* dz, void* stream);
/* out[r][col0 + c] = in[idx[r]][c] (idx may be NULL: identity); out row stride ldo. */
int hfnn_gather(int64_t rows, int width, const float* in, const int* idx, float* out, int ldo, int col0, void* stream);
/* out[idx[r]][c] += in[r][col0 + c] * scale[r]; in row stride ldi. */
int hfnn_scatter_add(int64_t rows, int width, const float* in, int ldi, int col0, const int* idx, const float* scale,
                     float* out, void* stream);
/* out[c] = sum_r in[r][c]. */
int hfnn_colsum(int64_t rows, int cols, const float* in, float* out, void* stream);
/* g = 2 w (y - t), *loss += w |y - t|^2. */
int hfnn_sq_loss(int64_t count, const float* y, const float* t, float w, float* g, float* loss, void* stream);
/* One Adam step (bias-corrected with the 1-based step). */
int hfnn_adam(int64_t count, float* p, const float* g, float* m, float* v, float lr, float b1, float b2, float eps,
              int step, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* HFNN_H */
