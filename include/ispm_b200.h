/* ispm_b200.h -- C ABI of the B200-native ispm-sparse-lib hot path.
 *
 * Plain pointers and sizes only: no C++, CUDA or torch types cross this
 * boundary (streams are passed as void *, i.e. a cudaStream_t; NULL is the
 * legacy default stream the reference runs on).  Every entry point returns
 * an ISPM_* status code instead of aborting the process the way the
 * reference's CUDA_CHECK does (util/cuda/check.h:8-15); ispm_last_error()
 * gives the message of the calling thread's last failure.
 *
 * Each declaration names the reference interface it replaces
 * (path:line within the reference project).
 *
 * Pointer conventions: "host" pointers are ordinary process memory, "device"
 * pointers are global memory of the current CUDA device (the reference's
 * devmem<T> / vector<T, device_memory_space_tag>).
 */
#ifndef ISPM_B200_H
#define ISPM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define ISPM_OK 0
#define ISPM_ERR_INVALID 1        /* bad argument or unsupported combination */
#define ISPM_ERR_CUDA 2           /* a CUDA runtime call failed */
#define ISPM_ERR_NOMEM 3          /* host or device allocation failed */
#define ISPM_ERR_ARCH 4           /* device is not sm_100 */
#define ISPM_ERR_BREAKDOWN 5      /* solver breakdown (zero / negative curvature) */
#define ISPM_ERR_NOT_CONVERGED 6  /* iteration limit reached before the target */
#define ISPM_ERR_TIMEOUT 7        /* a bounded device-side wait ran out */
#define ISPM_ERR_TOO_LARGE 8      /* size beyond a documented maximum */

/* element / vector types (ISPM_BF16, ISPM_F16: solver-internal element arrays only) */
#define ISPM_F32 0
#define ISPM_F64 1
#define ISPM_BF16 2
#define ISPM_F16 3

const char *ispm_error_string(int status);
/* Message of the calling thread's most recent failing call ("" if none). */
const char *ispm_last_error(void);
/* Library version string. */
const char *ispm_version(void);

/* ---- device initialisation (util/cuda/initialize.h:4-10,
 *      util/cuda/initialize.cu:17-42) --------------------------------------
 * Checks that the current device is compute capability 10.0 (sm_100) --
 * ISPM_ERR_ARCH otherwise, where the reference aborts -- and sets
 * cudaDeviceMapHost like the reference does.  The reference's 8-byte shared
 * memory bank request has no effect on sm_100 and is not made. */
int ispm_initialize(void);
/* "dddd:bb:dd (name)" of the current device into buf (at most len bytes). */
int ispm_get_device_string(char *buf, int len);

/* ---- sliced-ELLPACK matrices (formats/formats.h:39-102) ---------------- */

/* Plain view of one sliced-ELL matrix: the fields of slell_matrix<E, space>
 * (formats/formats.h:44-55) plus the lengths of its three arrays and the
 * tallest slice.  The arrays are host or device memory depending on where the
 * view came from. */
typedef struct {
  int n_rows;          /* rows after padding to a multiple of 512 */
  int n_cols;
  int n_nz;            /* non-zeros of the source CSR */
  unsigned slice_height;
  unsigned n_slices;
  unsigned hblock;     /* 1, 2 or 4 */
  int var_height;
  int diags;
  int elm_dtype;       /* ISPM_F32 / ISPM_F64 (ISPM_F16: ispm_launch_spmv_split) */
  unsigned min_slice_height; /* shortest / tallest slice (equal unless var_height) */
  unsigned max_slice_height;
  long long n_slice_ptr;
  long long n_cols_arr;
  long long n_elms;
  const unsigned *slice_ptr;
  const unsigned *cols;
  const void *elms;
} ispm_slell_view;

/* slell_params (formats/formats.h:39-42) */
typedef struct {
  unsigned S, H, V, D; /* slice height, hblock width, var height, diagonals */
} ispm_slell_params;

typedef struct ispm_slell ispm_slell;   /* host matrix  (host_memory_space_tag) */
typedef struct ispm_dslell ispm_dslell; /* device matrix (device_memory_space_tag) */

/* csr_to_slell (formats/conversion.h:338-414).  Converts an n_rows x n_cols
 * CSR (row_ptr[n_rows + 1], cols[nnz], elms[nnz] of elm_dtype, host memory)
 * into a host sliced-ELL matrix.  Result layout is bit-identical to the
 * reference's.  The reference pads the caller's CSR to a multiple of 512 rows
 * in place (conversion.h:343); this entry point leaves the caller's arrays
 * untouched and reports the padded row count in the result's n_rows.
 * A fixed slice height must divide the padded row count (the reference reads
 * past the CSR otherwise): ISPM_ERR_INVALID. */
int ispm_csr_to_slell(int elm_dtype, int n_rows, int n_cols, const int *row_ptr,
                      const int *cols, const void *elms, int slice_height, int hblock,
                      int var_height, int use_diags, int min_height, ispm_slell **out);

/* csr_to_slell_guess_format (formats/conversion.h:416-492): picks slice
 * height, hblock width, variable height and diagonal extraction from the first
 * examine_ratio percent of rows, then converts. Rows past n_rows read as empty
 * (the reference reads them unpadded for matrices under ~3,200 rows). */
int ispm_csr_to_slell_guess_format(int elm_dtype, int n_rows, int n_cols, const int *row_ptr,
                                   const int *cols, const void *elms, int examine_ratio,
                                   int min_height, ispm_slell **out);

/* View of a host matrix's arrays; valid until the matrix is freed. */
int ispm_slell_get_view(const ispm_slell *m, ispm_slell_view *view);
/* Mutable host element array (the public slell_matrix::elms member the
 * reference's callers edit before update_device_matrix_coefs). */
void *ispm_slell_elms(ispm_slell *m);
/* slell_matrix::spmv_bytes (formats/formats.h:72-78) with the vector element
 * size honoured (the reference always counts 4 bytes: sizeof(vec_elt_size)). */
unsigned long long ispm_slell_spmv_bytes(const ispm_slell *m, int effective, int vec_elt_size);
void ispm_slell_free(ispm_slell *m);

/* slell_matrix<E, device> copy constructor (formats/formats.h:56-66): upload
 * a host matrix to the current device. */
int ispm_dslell_upload(const ispm_slell *h, ispm_dslell **out);
/* The same for a host matrix whose FP32 elements are all exact binary16
 * values (an FP16 split, ispm_csr_split_f16): the device copy keeps them as
 * FP16 (elm_dtype ISPM_F16), for ispm_launch_spmv_split.  No counterpart in
 * the reference. */
int ispm_dslell_upload_f16(const ispm_slell *h, ispm_dslell **out);
/* Diagnostics of the staged SpMV walk (launch shape N = S, H = 1; no
 * counterpart in the reference): the tile records an upload of m computes
 * (144 ints per 256-row tile; none unless m has diagonal blocks and a fixed
 * slice height in [16, 256]).  *n_ints receives the count; at most cap ints
 * are written to out (which may be NULL with cap 0). */
int ispm_slell_stage_records(const ispm_slell *m, int *out, long long cap, long long *n_ints);
/* The staged walk's wait-timeout record: *code = 0, or the first timeout a
 * staged launch met since the last call (1 a consumer warp's wait for a
 * tile, 2 the copy warp's wait for a free slot); the record is cleared.
 * Synchronous. */
int ispm_spmv_stage_fault(int *code);
/* Re-upload only the element values of a matrix with unchanged structure
 * (plan/plan.h:39-42, implemented as the element-only H2D copy it means). */
int ispm_dslell_update_elms(ispm_dslell *d, const ispm_slell *h);
/* View of a device matrix's arrays (device pointers). */
int ispm_dslell_get_view(const ispm_dslell *d, ispm_slell_view *view);
void ispm_dslell_free(ispm_dslell *d);

/* ---- SpMV launch (cuda/spmv/kernel-iface.h:6-74, cuda/spmv/dispatch.h) -- */

/* spmv_launch_params (kernel-iface.h:6-17).  N = threads cooperating on one
 * slice, S = slice height the launch is specialised for, H = consecutive rows
 * per thread.  use_tex_* are accepted for source compatibility and ignored:
 * sm_100 has no texture references; x goes through the read-only data path. */
typedef struct {
  unsigned N, S, H;
  int use_tex_sliceptr;
  int use_tex_x;
} ispm_launch_params;

/* SPMV_PARAMS_VALID_P (kernel-iface.h:4): N >= S / H && S >= H. */
int ispm_launch_params_valid(const ispm_launch_params *p);

/* launch_spmv_kernel<T, E> (kernel-iface.h:20-74): y = A x on `stream`.
 * x_dtype is T (ISPM_F32 / ISPM_F64), A's elm_dtype is E; (T, E) must be one
 * of the reference's instantiations (float,float), (double,float),
 * (double,double).  x holds n_cols values of T, y n_rows (padded) values of T.
 * Where the reference silently launches nothing for unsupported parameters
 * (dispatch.h:131,143,166,180,202-203), this returns ISPM_ERR_INVALID.
 * Supported: N a power of two in [4, 1024]; H in {1, 2, 4}; S the matrix's
 * slice height (fixed-height matrices) and N * H >= every slice's height. */
int ispm_launch_spmv(int x_dtype, const ispm_launch_params *p, const ispm_slell_view *m,
                     const void *x, void *y, void *stream);

/* Split-operator SpMV (no counterpart in the reference): y = inv_scale *
 * (A_off x) + diag .* x with FP32 x and y, where m holds the off-diagonal
 * part as FP16 elements (elm_dtype ISPM_F16, e.g. the split of
 * ispm_csr_split_f16 converted with ispm_csr_to_slell and its element array
 * stored as binary16) and diag holds m->n_rows FP32 values (0 on padded
 * rows), 16-byte aligned.  This is the product the solver's matrix_f16 inner
 * iterations run; same launch parameters as ispm_launch_spmv.  diag NULL:
 * y = inv_scale * (m x), an FP16-stored factor (the factor_f16 option). */
int ispm_launch_spmv_split(const ispm_launch_params *p, const ispm_slell_view *m,
                           const float *diag, float inv_scale, const float *x, float *y,
                           void *stream);

/* Launch shape the library picks for a matrix without timing anything (the
 * DEFAULT plan's choice; plan/plan.h:74-96 uses N = 512, H = 1 there). */
int ispm_default_launch(int x_dtype, const ispm_slell_view *m, ispm_launch_params *out);

/* ---- autotuning plan (plan/plan.h:9-161) -------------------------------- */
#define ISPM_PLAN_DEFAULT 0
#define ISPM_PLAN_ESTIMATE 1
#define ISPM_PLAN_EXHAUSTIVE 2
#define ISPM_SPMV_NO_TEXTURE_MEMORY 1
#define ISPM_SPMV_PLAN_NO_DEVICE 2

typedef struct ispm_plan ispm_plan;

/* spmv_plan<T, E>(csr_matrix<E>, kind, flags) (plan/plan.h:64-146).
 * DEFAULT/ESTIMATE: guessed format, launch parameters from a B200 heuristic.
 * EXHAUSTIVE: the reference's format grid (S 32..512, V, D, hblock 1/2) widened
 * with hblock 4, and every launch shape timed with CUDA events (median of
 * repeats) instead of one timed launch. */
int ispm_plan_create(int vec_dtype, int elm_dtype, int n_rows, int n_cols, const int *row_ptr,
                     const int *cols, const void *elms, int kind, unsigned flags,
                     ispm_plan **out);
/* spmv_plan::execute_spmv (plan/plan.h:148-161) */
int ispm_plan_execute(ispm_plan *p, const void *x, void *y, void *stream);
/* spmv_plan::upload (plan/plan.h:44-49) */
int ispm_plan_upload(ispm_plan *p);
/* spmv_plan::update_device_matrix_coefs (plan/plan.h:39-42) */
int ispm_plan_update_device_matrix_coefs(ispm_plan *p);
/* spmv_plan::change_host_matrix (plan/plan.h:51-56): re-convert a new CSR
 * with the plan's stored format parameters (host matrix only). */
int ispm_plan_change_host_matrix(ispm_plan *p, int n_rows, int n_cols, const int *row_ptr,
                                 const int *cols, const void *elms);
/* Device-side fast path of update_device_matrix_coefs / change_host_matrix
 * for an unchanged sparsity pattern (plan/plan.h:39-56): new CSR values
 * (device array, FP32 or FP64, in the CSR entry order of row_ptr / cols) are
 * scattered straight into the device sliced-ELL matrix -- no host conversion,
 * no host-to-device copy of the matrix.  The first call computes the entry ->
 * slot map from the (host) pattern and keeps it on the device; later calls
 * with the same nnz reuse it.  The plan's host matrix is not updated. */
int ispm_plan_refresh_values(ispm_plan *p, int n_rows, const int *row_ptr, const int *cols,
                             const void *vals_dev, int val_dtype, void *stream);
/* The map itself (map[k] = element slot of CSR entry k, n_nz entries, host)
 * and the scatter for callers managing device matrices directly. */
int ispm_slell_value_map(const ispm_slell *m, int n_rows, const int *row_ptr, const int *cols,
                         unsigned *map);
int ispm_dslell_refresh_values(ispm_dslell *d, const unsigned *map_dev, const void *vals_dev,
                               int val_dtype, int n_nz, void *stream);
int ispm_plan_get_params(const ispm_plan *p, ispm_slell_params *mparams,
                         ispm_launch_params *params);
/* The plan's matrices (NULL if absent); owned by the plan. */
ispm_slell *ispm_plan_host_matrix(ispm_plan *p);
const ispm_dslell *ispm_plan_device_matrix(const ispm_plan *p);
/* Best time (seconds) an EXHAUSTIVE plan measured, else 0. */
double ispm_plan_tuned_seconds(const ispm_plan *p);
void ispm_plan_free(ispm_plan *p);

/* ---- sblas: BLAS-1 and pipelined-CG fusions (util/cuda/sblas.h:1-56) ----
 * All vector and scalar pointers are device pointers of dtype T.
 * Reductions accumulate in FP64 whatever T is (the reference accumulates in
 * T) and finish inside the same launch (the reference adds a one-block
 * launch).  They use a per-device scratch area allocated on first use, so
 * calls that overlap on the GPU (different streams, or threads) race on it,
 * exactly as the reference's full_launch singleton does. */

/* sblas::copy_indexed (sblas.cu:18-33): dst[k] = src[idx[k]], k < n. */
int ispm_sblas_copy_indexed(int dtype, void *dst, const void *src, const int *idx, int n,
                            void *stream);
/* sblas::add_indexed (sblas.cu:36-51): dst[idx[k]] += src[k].  Uses atomic
 * adds, so repeated indices all count (the reference races on them). */
int ispm_sblas_add_indexed(int dtype, void *dst, const void *src, const int *idx, int n,
                           void *stream);
/* sblas::dot (sblas.cu:126-153): *s = sum x_i y_i. */
int ispm_sblas_dot(int dtype, const void *x, const void *y, void *s, int n, void *stream);
/* ispm_sblas_dot without any device allocation.  No counterpart in the
 * reference: it is for callers that cannot let a library cudaMalloc (a fixed,
 * pre-reserved device memory budget, or loops that must not risk the implicit
 * synchronisation of cudaMalloc / cudaFree).  Same arguments and result as
 * ispm_sblas_dot; its scratch is a static device array inside the library
 * (1024 partial sums + a counter, about 8 KB per GPU, held until exit); the
 * dot's grid is capped at 1024 CTAs, so a device with more than 256 SMs runs
 * it with 1024 CTAs.  The first call on a device looks the array up (cudaGetSymbolAddress) -- make it
 * before any stream capture.  All calls share the array: calls that overlap
 * on the GPU race. */
int ispm_sblas_dot_noalloc(int dtype, const void *x, const void *y, void *s, int n,
                           void *stream);
/* sblas::ppcg_update_scalars (sblas.cu:156-174):
 * beta = gamma / gammaold; alpha = gamma / (delta - beta * gamma / alpha). */
int ispm_sblas_ppcg_update_scalars(int dtype, void *alpha, void *beta, const void *gamma,
                                   const void *gammaold, const void *delta, void *stream);
/* sblas::ppcg_update_vectors (sblas.cu:177-237): z = n + beta z;
 * q = m + beta q; s = w + beta s; p = u + beta p; u -= alpha q; w -= alpha z;
 * r -= alpha s; x += alpha p; then *resnorm = sum |r_i|, *gamma = r.u,
 * *delta = w.u of the updated vectors. */
int ispm_sblas_ppcg_update_vectors(int dtype, void *resnorm, void *gamma, void *delta,
                                   const void *alpha, const void *beta, const void *n,
                                   const void *m, void *p, void *s, void *q, void *z, void *x,
                                   void *r, void *u, void *w, int n_elts, void *stream);

/* ---- approximate inverse (fastainv/fastainv.h:8-30) --------------------- */

typedef struct ispm_csr ispm_csr; /* host CSR owned by the library */
typedef void (*ispm_progress_f)(void *);

typedef struct {
  long long storage_chunks;   /* chunk capacity after the maxneed cap */
  long long chunks_used;
  long long truncated_rows;   /* row updates cut short by exhausted storage */
  long long breakdowns;       /* pivots D_jj == 0 (row scale set to 0) */
} ispm_fastainv_stats;

/* fastainv_sym<double, out_real> (fastainv/fastainv.cpp:395-566).  A is an
 * n x n symmetric CSR in FP64 (host).  Produces Ainv1 (= G) and Ainv2 (= G^T
 * with unsigned scale), so that Ainv2 * Ainv1 ~ A^-1, bit-identical to the
 * reference for out_dtype FP64 (double,double) and FP32 (double,float).
 * progress(v) is called once per row as in the reference (may be NULL).
 * Returns ISPM_ERR_INVALID for n <= 0 (the reference returns false).
 * stats may be NULL; storage exhaustion truncates rows exactly as the
 * reference does (fastainv.cpp:74-78) and is counted in stats. */
int ispm_fastainv_sym(int out_dtype, int n, const int *row_ptr, const int *cols,
                      const double *elms, ispm_progress_f progress, void *v,
                      long long max_elts, double droptol, ispm_csr **ainv1, ispm_csr **ainv2,
                      ispm_fastainv_stats *stats);
/* fastainv_sym with per-row controls (extends fastainv/fastainv.cpp:395-566;
 * the plain entry point above is unchanged).  row_droptol[i] replaces droptol
 * in the drop test of factor row i (fastainv.cpp:304), row_scale[j] > 0
 * multiplies the pivot scale sqrt|D_jj| of factor row j in both outputs
 * (fastainv.cpp:518-519), so M = Ainv2 Ainv1 = sum_j row_scale[j]^2 z_j z_j^T /
 * D_jj.  Either array may be NULL (then droptol / 1).  Used by the learned
 * FSAI, which predicts both per row. */
int ispm_fastainv_sym_ex(int out_dtype, int n, const int *row_ptr, const int *cols,
                         const double *elms, const double *row_droptol, const double *row_scale,
                         long long max_elts, double droptol, ispm_csr **ainv1, ispm_csr **ainv2,
                         ispm_fastainv_stats *stats);
/* Factorized sparse approximate inverse built on the GPU: a parallel
 * replacement for fastainv_sym's serial host build (fastainv.cpp:395-566),
 * equivalent in PCG iterations rather than bit-identical.  G is lower
 * triangular on A's lower pattern, each row solving A[P,P] y = e_i on the
 * device; the pair is returned in fastainv_sym's convention, Ainv1 = G and
 * Ainv2 = G^T, so that Ainv2 Ainv1 = G^T G ~ A^-1.  A: symmetric positive
 * definite host CSR in FP64 with sorted columns, at most 32 entries per row
 * at or left of the diagonal.  *fallbacks (may be NULL) counts rows whose
 * local matrix was not positive definite (built as Jacobi rows). */
int ispm_fsai_sym_gpu(int out_dtype, int n, const int *row_ptr, const int *cols,
                      const double *elms, ispm_csr **ainv1, ispm_csr **ainv2,
                      unsigned *fallbacks);
/* The FP16 split of a square FP64 CSR matrix that the solver's matrix_f16
 * option stores (no counterpart in the reference, whose matrices are FP32 or
 * FP64).  For every row i: off-diagonal values a_ij become
 * h_ij = fp16(a_ij * scale) (round to nearest even, subnormals kept), written
 * as IEEE binary16 bit patterns to off_f16[k] for CSR entry k (0 for the
 * diagonal entry); diag[i] = fp32(a_ii + sum_j (|h_ij| / scale - |a_ij|)),
 * the diagonal moved by the rounding of the row's off-diagonal magnitudes so
 * that the split matrix minus A is the weighted graph Laplacian of the
 * rounding errors (zero row sums for an M-matrix).  scale is the power of
 * two that maps the largest off-diagonal magnitude into [2^13, 2^14).
 * off_f16 has row_ptr[n] entries, diag n. */
/* Reverse Cuthill-McKee ordering of a symmetric n x n pattern (no
 * counterpart in the reference; the solver's opts.reorder uses it):
 * perm[new] = old, n entries.  The renumbered matrix P A P^T keeps each
 * row's neighbours in a narrow band, so SpMV gathers of x become local. */
int ispm_rcm_order(int n, const int *row_ptr, const int *cols, int *perm);
/* max |col - row| over the pattern, or -1 for a malformed CSR. */
long long ispm_csr_bandwidth(int n, const int *row_ptr, const int *cols);
int ispm_csr_split_f16(int n, const int *row_ptr, const int *cols, const double *vals,
                       uint16_t *off_f16, float *diag, float *scale);
int ispm_csr_get_info(const ispm_csr *m, int *n_rows, int *n_cols, int *n_nz, int *dtype);
/* Host views of the CSR arrays; valid until ispm_csr_free. */
int ispm_csr_get_arrays(const ispm_csr *m, const int **row_ptr, const int **cols,
                        const void **elms);
void ispm_csr_free(ispm_csr *m);

/* ---- preconditioned pipelined CG (the loop the reference leaves to its
 *      external solver driver, README.md:5-9, built from the primitives
 *      above: launch_spmv_kernel, sblas::ppcg_update_*, fastainv_sym) ----- */

typedef struct {
  int inner_dtype;      /* ISPM_F64: plain FP64 solve; ISPM_F32: FP32 matrices and
                           vectors, FP64 reductions and FP64 reliable updates */
  double tol;           /* target ||b - A x||_2 / ||b||_2, checked in FP64 */
  int max_iters;        /* total iterations */
  int max_refinements;  /* reliable updates + restarts */
  int check_every;      /* iterations per CUDA-graph chunk between host checks */
  int use_graph;        /* 1: replay iteration chunks as a CUDA graph, the host
                           reading the device flags after each chunk; 2 (the
                           classic iteration of an FP32 inner solve; others
                           as 1): the chunk is the body of the graph's while
                           node, repeated on the device until the flags end
                           the phase, so a phase is one graph launch and one
                           host wait; 0: eager launches */
  double replace_ratio_f32; /* reliable update once the recursive residual fell by
                               this factor since the last one (FP32 inner) */
  double replace_ratio_f64; /* same for FP64 */
  int variant;          /* ISPM_PCG_AUTO (pipelined in FP64, classic in FP32),
                           ISPM_PCG_PIPELINED or ISPM_PCG_CLASSIC */
  int prec;             /* ISPM_PREC_GIVEN: the (g1, g2) pair passed to
                           ispm_solver_create (none if NULL); ISPM_PREC_FSAI_GPU:
                           FSAI factor on A's lower pattern built on the GPU
                           (g1, g2 ignored) */
  int factor_bf16;      /* FP32 inner solve: keep the preconditioner factor's values
                           in BF16 (half the bytes of each factor application; the
                           preconditioner stays SPD, its values lose 16 mantissa
                           bits; A, the reductions and the reliable updates are
                           unchanged) */
  int reorder;          /* ISPM_REORDER_AUTO (default): unless the bandwidth is
                           already under n / 16, renumber the unknowns in
                           reverse Cuthill-McKee order when that shrinks the
                           matrix bandwidth at least 4x (a scattered numbering),
                           so the SpMV gathers become local; b and x stay in the
                           caller's order.  ISPM_REORDER_RCM: always;
                           ISPM_REORDER_NONE: never.  Not with a given factor
                           pair (it is in the caller's order). */
  int matrix_f16;       /* FP32 inner solve: store A for the inner iterations as
                           FP16 off-diagonal values (times a power-of-two scale)
                           plus an FP32 diagonal, the split of
                           ispm_csr_split_f16.  The inner matrix then differs
                           from A by a weighted graph Laplacian of at most 2^-11
                           times A's own off-diagonal weights, so it keeps A's
                           near-null space (row sums) and the FP64 reliable
                           updates still converge; each inner SpMV reads about
                           half the matrix bytes.  replace_ratio_f32 is raised
                           to at least 3e-2 (a reliable update at least every
                           33x fall of the recursive residual).  A and its
                           reliable-update residuals stay FP64. */
  int factor_f16;       /* FP32 inner solve with prec = ISPM_PREC_FSAI_GPU: keep
                           the factor's values in FP16 times one power-of-two
                           scale (the largest magnitude lands in [2^13, 2^14)),
                           11 mantissa bits where BF16 keeps 8; half the bytes
                           of each factor application.  Takes precedence over
                           factor_bf16.  On by default (the 128^3 27-point
                           solve: 59.4 against 61.9 ms with FP32 factors,
                           499 against 501 iterations, on a B200). */
  int refresh;          /* keep what ispm_solver_update_values needs to take new
                           values of A (same sparsity pattern) on the device:
                           the CSR-entry -> element-slot maps of both device
                           copies of A, the renumbering's entry map and, with
                           prec = ISPM_PREC_FSAI_GPU, the factor's device
                           patterns (about 20 bytes per entry of A and 32 per
                           entry of G).  Not with matrix_f16. */
} ispm_solver_opts;

#define ISPM_REORDER_NONE 0
#define ISPM_REORDER_RCM 1
#define ISPM_REORDER_AUTO 2

#define ISPM_PREC_GIVEN 0
#define ISPM_PREC_FSAI_GPU 1

#define ISPM_PCG_AUTO 0
#define ISPM_PCG_PIPELINED 1
#define ISPM_PCG_CLASSIC 2

typedef struct {
  int iterations;       /* iterations over the whole solve */
  int refinements;      /* reliable updates (true-residual replacements) + restarts */
  int converged;
  int status;
  double true_relres;   /* ||b - A x||_2 / ||b||_2 with the FP64 matrix */
  double seconds;       /* host wall time of the solve call */
} ispm_solve_stats;

/* Defaults: FP32 inner with FP64 reliable updates, tol 1e-10, max_iters
 * 100000, max_refinements 500, check_every 16, use_graph 1,
 * replace_ratio_f32 1e-2, replace_ratio_f64 1e-4, variant AUTO, prec GIVEN,
 * factor_bf16 0, reorder AUTO, matrix_f16 0, factor_f16 1, refresh 0. */
void ispm_solver_default_opts(ispm_solver_opts *opts);

typedef struct ispm_solver ispm_solver;

/* A: n x n SPD CSR in FP64 (host).  (g1, g2): the fastainv_sym pair
 * (Ainv1, Ainv2) in FP64 (host), or all NULL for no preconditioner.  The
 * solver keeps device copies only (FP64 A for residuals, A and the factor
 * pair in the inner type). */
int ispm_solver_create(int n, const int *row_ptr, const int *cols, const double *vals,
                       const int *g1_row_ptr, const int *g1_cols, const double *g1_vals,
                       const int *g2_row_ptr, const int *g2_cols, const double *g2_vals,
                       const ispm_solver_opts *opts, ispm_solver **out);
/* Padded row count (the length of the device vectors the solver expects). */
int ispm_solver_rows(const ispm_solver *s);
/* Solve A x = b; b and x are device FP64 vectors of ispm_solver_rows()
 * entries (x is overwritten; the solve starts from zero). */
int ispm_solver_solve(ispm_solver *s, const double *b, double *x, ispm_solve_stats *stats,
                      void *stream);
/* Same with host vectors of n entries: copies b in and x out inside the call. */
int ispm_solver_solve_host(ispm_solver *s, const double *b_host, double *x_host,
                           ispm_solve_stats *stats, void *stream);
/* New values of A for a solver created with opts.refresh = 1: vals holds
 * row_ptr[n] FP64 values in the CSR order (and sparsity pattern) passed to
 * ispm_solver_create, on the device when vals_on_device is nonzero, else on
 * the host.  Both device copies of A are rewritten in place and, with prec =
 * ISPM_PREC_FSAI_GPU, the FSAI factor pair is rebuilt on the device from the
 * new values; no conversion, ordering or pattern work runs on the host, so a
 * time-stepping caller whose matrix keeps its pattern pays this instead of
 * a new ispm_solver_create.  A given factor pair (prec = ISPM_PREC_GIVEN)
 * stays as it was.  The values are not checked (a non-SPD matrix shows as a
 * breakdown in the next solve).  Synchronous.  (The reference's
 * counterpart for one matrix is spmv_plan::refresh_values, plan/plan.h:39-56.) */
int ispm_solver_update_values(ispm_solver *s, const double *vals, int vals_on_device);
/* The device matrices the solver iterates with, for inspection or a
 * caller's own products: which = 0 the inner-precision A, 1 the FP64 A of
 * the reliable updates, 2 G, 3 G^T (in the solver's numbering when it
 * renumbered); *view gets the device view, *params (may be NULL) the launch
 * shape the solver uses.  Valid until ispm_solver_free. */
int ispm_solver_operator(const ispm_solver *s, int which, ispm_slell_view *view,
                         ispm_launch_params *params);
/* The sliced-ELL shape the solver stores an n x n operator in (elm_dtype
 * ISPM_F32 or ISPM_F64): among the reference's guessed format and the fixed
 * heights 32 / 64 / 128 with and without diagonal blocks (and hblock 2),
 * the fewest stored bytes, with 32- and 64-row slices counted 10% / 2%
 * above their bytes (measured on a B200: short slices cost time their
 * bytes do not show).  Host only. */
int ispm_solver_choose_shape(int elm_dtype, int n, const int *row_ptr, const int *cols,
                             const double *vals, ispm_slell_params *out);
/* True relative residual after each outer cycle of the last solve; returns
 * the count (writes at most cap values). */
int ispm_solver_history(const ispm_solver *s, double *out, int cap);
void ispm_solver_free(ispm_solver *s);

/* ---- batched PCG: many independent SPD systems of uneven size, each with
 *      one or more right-hand sides, advanced together (one set of launches
 *      per iteration for all of them).  The reference has no batched path: a
 *      caller with several systems per time step calls its primitives
 *      (cuda/spmv/kernel-iface.h:20-74, util/cuda/sblas.h:1-25) once per
 *      system.  Every (system, right-hand side) pair is a lane; lanes are
 *      padded to whole 1024-row tiles and stacked in one device vector. ---- */

#define ISPM_PREC_NONE 2 /* batched solver: no preconditioner */

typedef struct ispm_batch ispm_batch;

/* System k: n_rows[k] x n_rows[k] SPD CSR in FP64 (host arrays row_ptr[k],
 * cols[k], vals[k]) with n_rhs[k] >= 1 right-hand sides.  opts (NULL: the
 * solver defaults with prec = ISPM_PREC_FSAI_GPU and replace_ratio_f32 =
 * 1e-3): inner_dtype, tol, max_iters (per lane), max_refinements (per lane),
 * check_every (rounded up to an even count), use_graph, replace_ratio_f32 /
 * _f64 (a lane pauses for a reliable update once its recursive residual fell
 * by this factor), prec (ISPM_PREC_FSAI_GPU or ISPM_PREC_NONE).
 * The iteration is classic PCG in the inner type with FP64 lane sums and an
 * FP64 reliable update after every chunk. */
int ispm_batch_create(int n_systems, const int *n_rows, const int *const *row_ptr,
                      const int *const *cols, const double *const *vals, const int *n_rhs,
                      const ispm_solver_opts *opts, ispm_batch **out);
int ispm_batch_lanes(const ispm_batch *b);
/* Length of the stacked device vectors. */
long long ispm_batch_rows(const ispm_batch *b);
/* Lane -> system, right-hand side, first stacked row, format group
 * (any output may be NULL). */
int ispm_batch_lane_info(const ispm_batch *b, int lane, int *system, int *rhs, long long *row0,
                         int *group);
/* Format groups: the sliced-ELL shape of each group's A and its lane count
 * (writes at most cap entries; returns the group count). */
int ispm_batch_groups(const ispm_batch *b, ispm_slell_params *a_fmt, int *lanes, int cap);
/* Solve every lane; b and x are stacked device FP64 vectors of
 * ispm_batch_rows() entries (lane l at its row0; padding rows of b zero).
 * lane_stats (may be NULL): one entry per lane; total (may be NULL):
 * maxima over the lanes, converged = all converged. */
int ispm_batch_solve(ispm_batch *b, const double *b_dev, double *x_dev,
                     ispm_solve_stats *lane_stats, ispm_solve_stats *total, void *stream);
/* Host vectors: b_host[k] / x_host[k] hold system k's n_rhs[k] right-hand
 * sides / solutions of n_rows[k] entries each, one after the other; copied
 * in and out inside the call. */
int ispm_batch_solve_host(ispm_batch *b, const double *const *b_host, double *const *x_host,
                          ispm_solve_stats *lane_stats, ispm_solve_stats *total, void *stream);
/* Kernels the last solve launched (graph replays counted per node). */
int ispm_batch_launches(const ispm_batch *b);
/* Rows of the stacked FSAI factor built as Jacobi rows. */
unsigned ispm_batch_fsai_fallbacks(const ispm_batch *b);
void ispm_batch_free(ispm_batch *b);

/* ---- learned drop tolerances (replaces the tuning search of
 *      fastainv/droptol-tuning.h:4-103 with a per-row prediction) ---------
 * A per-row MLP 32 -> 64 -> 64 -> 2 (ReLU; BF16 weights and inputs, FP32
 * accumulation) predicts, from ispm_row_features, the log2 drop tolerance
 * ratio and the log rescale of each row of the approximate inverse; the
 * caller feeds them to ispm_fastainv_sym_ex.  Trained and run on the GPU. */

/* Features (32 BF16 values per row, device output, row-major) of an FP64
 * CSR held in device memory; nx, ny: grid dimensions of a box stencil
 * (neighbours located by offset, nx, ny >= 3), or 0, 0 (entries in column
 * order). */
int ispm_row_features(int n, const int *row_ptr, const int *cols, const double *vals, int nx,
                      int ny, void *out_bf16, void *stream);

typedef struct ispm_mlp ispm_mlp;
/* Parameter count; layout: W1[64][32], b1[64], W2[64][64], b2[64], W3[2][64],
 * b3[2] (FP32 master copy; the kernels round W1..W3 to BF16). */
int ispm_mlp_n_params(void);
int ispm_mlp_create(const float *init_params, ispm_mlp **out);
int ispm_mlp_get_params(const ispm_mlp *m, float *host_out);
/* Replace the parameters and reset the optimiser state. */
int ispm_mlp_set_params(ispm_mlp *m, const float *host_in);
/* out[2 * r + o] = output o of row r (device; features device BF16). */
int ispm_mlp_forward(const ispm_mlp *m, long long n_rows, const void *feat_bf16, float *out,
                     void *stream);
/* Loss sum_r sum_o w_ro (y_ro - t_ro)^2 / n_rows and its gradient (kept for
 * ispm_mlp_adam_step; copied to grad_out, host, when non-NULL).  target and
 * weight (NULL: all ones) are device [n_rows][2] FP32.  Deterministic. */
int ispm_mlp_loss_grad(ispm_mlp *m, long long n_rows, const void *feat_bf16,
                       const float *target, const float *weight, float *grad_out,
                       double *loss_out, void *stream);
/* One Adam step on the last gradient (plus weight_decay * parameter, an L2
 * term, added to it). */
int ispm_mlp_adam_step(ispm_mlp *m, float lr, float beta1, float beta2, float eps,
                       float weight_decay, void *stream);
void ispm_mlp_free(ispm_mlp *m);

/* ---- drop-tolerance tuner (fastainv/droptol-tuning.h:4-103) ------------ */
typedef struct ispm_droptol_tuner ispm_droptol_tuner;
ispm_droptol_tuner *ispm_droptol_tuner_create(double lo, double hi);
double ispm_droptol_tuner_get_droptol(const ispm_droptol_tuner *t);
double ispm_droptol_tuner_get_best_droptol(const ispm_droptol_tuner *t);
void ispm_droptol_tuner_note_time(ispm_droptol_tuner *t, double time);
void ispm_droptol_tuner_restart(ispm_droptol_tuner *t);
void ispm_droptol_tuner_reset_phase(ispm_droptol_tuner *t);
int ispm_droptol_tuner_iterations(const ispm_droptol_tuner *t);
void ispm_droptol_tuner_free(ispm_droptol_tuner *t);

#ifdef __cplusplus
}
#endif
#endif
