/* ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the parts of the reference hot path that cannot be
 * compiled here (the reference's CUDA kernels use texture references and
 * __shfl_down, both removed in CUDA 12), plus FP64 CSR oracles that the
 * reference does not have.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load liboracle.so; the product never does.
 *
 * Each function cites the reference file:line whose behaviour it restates.
 */
#ifndef ISPM_ORACLE_H
#define ISPM_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Sliced-ELL matrix as laid out by formats/conversion.h:338-414. */
typedef struct {
  int n_rows, n_cols;
  unsigned slice_height, n_slices, hblock;
  int var_height, diags;
  const unsigned *slice_ptr;
  const unsigned *cols;
  const void *elms; /* float or double, per e_f64 */
  int e_f64;
} orc_slell;

/* y = A x following cuda/spmv/kernel.h:1-135 for launch parameters (N, H):
 * per-thread partial sums in the kernel's walk order (kernel.h:70-119), the
 * fold-upper-half-onto-lower column reduction (cuda/reduce.h:80-127) and the
 * store of rows [y0, y0 + slice size) (kernel.h:130-134).  Multiply-adds are
 * fused (fma), as nvcc contracts them by default.
 * x_f64 selects T (double or float) for x, y and accumulation.
 * tex_bounds = 1 reproduces texture fetch semantics (dispatch.h:41-50):
 *   a scalar x fetch at index >= n_cols returns 0, and a W-wide x fetch at
 *   vector index >= n_cols / W (floor) returns 0.
 * tex_bounds = 0 bounds each x element individually (index >= n_cols -> 0),
 *   which is the product's documented semantics.
 * Returns 0, or -1 for an invalid (N, H) / slice combination. */
int orc_slell_spmv_kernel_order(const orc_slell *A, unsigned N, unsigned H, int tex_bounds,
                                int x_f64, const void *x, void *y);

/* Same walk, exact-ish: every product accumulated in long double per row, and
 * absrow[r] = sum |a_rk| |x_k| (the forward-error scale used by the tests). */
int orc_slell_spmv_exact(const orc_slell *A, int tex_bounds, int x_f64, const void *x,
                         double *y, double *absrow);

/* FP64 CSR y = A x (OpenMP over rows); absrow optional. */
void orc_csr_spmv_f64(int n_rows, const int *row_ptr, const int *cols, const double *elms,
                      const double *x, double *y, double *absrow);

/* FP64 CSR y = A x for a matrix whose values are float. */
void orc_csr_spmv_f32e(int n_rows, const int *row_ptr, const int *cols, const float *elms,
                       const double *x, double *y);

/* util/cuda/sblas.cu:18-33 copy_indexed: dst[k] = src[idx[k]]. */
void orc_copy_indexed(int f64, void *dst, const void *src, const int *idx, int n);
/* util/cuda/sblas.cu:36-51 add_indexed: dst[idx[k]] += src[k]; duplicates
 * are all applied, in k order (the reference races on them). */
void orc_add_indexed(int f64, void *dst, const void *src, const int *idx, int n);
/* util/cuda/sblas.cu:126-153 dot: sum x_i y_i, accumulated in long double. */
double orc_dot(int f64, const void *x, const void *y, int n);
/* util/cuda/sblas.cu:156-174 ppcg_update_scalars, in T. */
void orc_ppcg_update_scalars(int f64, void *alpha, void *beta, const void *gamma,
                             const void *gammaold, const void *delta);
/* util/cuda/sblas.cu:177-216 ppcg_update_vectors: the eight fused recurrences
 * in T with fma contraction; the three reductions (sum |r|, r.u, w.u) of the
 * updated vectors are returned in long double precision as doubles. */
void orc_ppcg_update_vectors(int f64, double *resnorm, double *gamma, double *delta,
                             const void *alpha, const void *beta, const void *nv,
                             const void *mv, void *p, void *s, void *q, void *z, void *x,
                             void *r, void *u, void *w, int n);

/* Preconditioned CG in FP64 on CSR operands, M = G2 (G1 v) (the pair
 * fastainv_sym returns, fastainv/fastainv.cpp:489-558).  pipelined = 0: the
 * textbook recurrence; 1: the pipelined recurrence the sblas fusions implement
 * (sblas.cu:156-216, Ghysels & Vanroose 2014).  G1/G2 may be NULL (no
 * preconditioner).  Stops when ||b - A x||_2 / ||b||_2 <= tol (recursive
 * residual, then confirmed with a true residual) or after max_it iterations.
 * Returns the iteration count; *relres = final true relative residual. */
int orc_pcg_f64(int pipelined, int n, const int *A_rp, const int *A_ci, const double *A_v,
                const int *G1_rp, const int *G1_ci, const double *G1_v, const int *G2_rp,
                const int *G2_ci, const double *G2_v, const double *b, double *x, double tol,
                int max_it, double *relres);

/* Number of OpenMP threads the oracle's parallel loops use. */
int orc_num_threads(void);

/* FSAI factor rows on A's lower pattern, the construction of the GPU build
 * (ispm-sparse-lib_b200/csrc/fsai.cu): for each listed row i, P = the sorted
 * entries of row i of A up to the diagonal, A[P,P] y = e_last (dense FP64
 * Cholesky), g = y / sqrt(y_last); a local matrix that is not positive
 * definite gives the Jacobi row.  orc_fsai_pattern_size: entries the listed
 * rows hold.  orc_fsai_rows fills out_rp[n_rows_out + 1], out_ci, out_v and
 * returns the Jacobi-row count (-1 if a pattern is empty or exceeds 64
 * entries). */
long long orc_fsai_pattern_size(const int *rp, const int *ci, const int *rows, int n_rows_out);
long long orc_fsai_rows(const int *rp, const int *ci, const double *v, const int *rows,
                        int n_rows_out, int *out_rp, int *out_ci, double *out_v);

#ifdef __cplusplus
}
#endif
#endif
