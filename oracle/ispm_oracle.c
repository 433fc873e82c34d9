/* ORACLE / TEST INFRASTRUCTURE ONLY -- see ispm_oracle.h.
 *
 * CPU restatement of the reference's sliced-ELL SpMV kernel
 * (cuda/spmv/kernel.h), its column reduction (cuda/reduce.h), the sblas
 * BLAS-1 / pipelined-CG fusions (util/cuda/sblas.cu), and FP64 CSR / PCG
 * oracles.  Built with -ffp-contract=off so that every fused multiply-add
 * below is the explicit fma()/fmaf() call it is written as. */
#include "ispm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

int orc_num_threads(void)
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

static int is_pow2(unsigned v) { return v && !(v & (v - 1)); }

/* Slice header decode: kernel.h:13-61.  Fills the fields a slice walk needs.
 * slice record layout: [elms_end, (row_end if V), (cols_end if W>1 or D),
 * (diag_ptr if D)] (conversion.h:393-402). */
typedef struct {
  unsigned e0, e1, y0, sz, c0, c1, d0, cb;
} slice_hdr;

static void decode_slice(const orc_slell *A, unsigned b, slice_hdr *h)
{
  const unsigned *sp = A->slice_ptr;
  unsigned W = A->hblock;
  int V = A->var_height, D = A->diags;
  unsigned spe = 1 + (W > 1) + (unsigned)V + 2u * (unsigned)D;
  unsigned p0 = spe * b;
  h->e0 = sp[p0];
  h->e1 = sp[p0 + spe];
  if (V) {
    h->y0 = sp[p0 + 1];
    h->sz = sp[p0 + 1 + spe] - h->y0;
  } else {
    h->y0 = A->slice_height * b;
    h->sz = A->slice_height;
  }
  h->d0 = 0;
  h->cb = 0;
  if (D) {
    h->c0 = sp[p0 + V + 1];
    h->d0 = sp[p0 + V + 2];
    h->c1 = sp[p0 + V + 1 + spe];
  } else if (W > 1) {
    h->c0 = sp[p0 + V + 1];
    h->c1 = sp[p0 + V + 1 + spe];
    unsigned nse = (W * (h->c1 - h->c0) - (h->e1 - h->e0)) / (W - 1);
    h->cb = h->c1;
    h->c1 = h->c0 + nse;
    h->e1 = h->e0 + nse;
  } else {
    h->c0 = h->e0;
    h->c1 = h->e1;
  }
}

/* kernel.h:1-135 walk, instantiated for T = double and T = float. */
#define DEF_KERNEL_ORDER(SUF, T, FMA)                                                       \
  static T xs_##SUF(const T *x, unsigned idx, unsigned n_cols)                              \
  {                                                                                         \
    return idx < n_cols ? x[idx] : (T)0;                                                    \
  }                                                                                         \
  static void xw_##SUF(const T *x, unsigned vidx, unsigned W, unsigned n_cols, int tex,     \
                       T *out)                                                              \
  {                                                                                         \
    for (unsigned w = 0; w < W; w++) {                                                      \
      unsigned e = vidx * W + w;                                                            \
      int ok = tex ? (vidx < n_cols / W) : (e < n_cols);                                    \
      out[w] = ok ? x[e] : (T)0;                                                            \
    }                                                                                       \
  }                                                                                         \
  static T ld_##SUF(const orc_slell *A, unsigned i)                                         \
  {                                                                                         \
    return A->e_f64 ? (T)((const double *)A->elms)[i] : (T)((const float *)A->elms)[i];     \
  }                                                                                         \
  static int spmv_ko_##SUF(const orc_slell *A, unsigned N, unsigned H, int tex, const T *x, \
                           T *y)                                                            \
  {                                                                                         \
    unsigned W = A->hblock;                                                                 \
    T *acc = (T *)malloc(sizeof(T) * N * H);                                                \
    int bad = 0;                                                                            \
    for (unsigned b = 0; b < A->n_slices && !bad; b++) {                                    \
      slice_hdr s;                                                                          \
      decode_slice(A, b, &s);                                                               \
      unsigned sz = s.sz;                                                                   \
      if (!is_pow2(sz) || sz < H || N < sz / H) {                                           \
        bad = 1;                                                                            \
        break;                                                                              \
      }                                                                                     \
      for (unsigned t = 0; t < N; t++) {                                                    \
        T a[4] = {0, 0, 0, 0};                                                              \
        unsigned i = s.e0 + t * H, j = s.c0 + t * H;                                        \
        for (; j < s.c1; i += N * H, j += N * H) /* kernel.h:70-79 */                       \
          for (unsigned h = 0; h < H; h++)                                                  \
            a[h] = FMA(ld_##SUF(A, i + h), xs_##SUF(x, A->cols[j + h], A->n_cols), a[h]);   \
        if (A->diags) { /* kernel.h:80-92 */                                                \
          unsigned adj = ((t * H) & (sz - 1)) - sz;                                         \
          unsigned jj = s.d0 + (j - s.c1) / sz;                                             \
          for (; i < s.e1; i += N * H, jj += N * H / sz) {                                  \
            unsigned ii = A->slice_ptr[jj] + adj;                                           \
            for (unsigned h = 0; h < H; h++)                                                \
              a[h] = FMA(ld_##SUF(A, i + h), xs_##SUF(x, ii + h, A->n_cols), a[h]);         \
          }                                                                                 \
        } else if (W > 1) { /* kernel.h:93-119 */                                           \
          i = s.e1 + ((i - s.e1) & (sz - 1)) + ((i - s.e1) & ~(sz - 1)) * W;                \
          for (; j < s.cb; i += W * N * H, j += N * H)                                      \
            for (unsigned h = 0; h < H; h++) {                                              \
              T wx[4];                                                                      \
              xw_##SUF(x, A->cols[j + h], W, A->n_cols, tex, wx);                           \
              /* t += e0*wx0 + e1*wx1 (+ e2*wx2 + e3*wx3): inner sum contracted */          \
              T sum = ld_##SUF(A, i + h) * wx[0];                                           \
              for (unsigned w = 1; w < W; w++)                                              \
                sum = FMA(ld_##SUF(A, i + h + sz * w), wx[w], sum);                         \
              a[h] = a[h] + sum;                                                            \
            }                                                                               \
        }                                                                                   \
        for (unsigned h = 0; h < H; h++)                                                    \
          acc[t * H + h] = a[h];                                                            \
      }                                                                                     \
      /* reduce.h:80-127: fold the upper half of the threads onto the lower half */         \
      for (unsigned n = N; n > sz / H; n /= 2)                                              \
        for (unsigned t = 0; t < n / 2; t++)                                                \
          for (unsigned h = 0; h < H; h++)                                                  \
            acc[t * H + h] = acc[t * H + h] + acc[(t + n / 2) * H + h];                     \
      for (unsigned t = 0; t < sz / H; t++) /* kernel.h:130-134 */                          \
        for (unsigned h = 0; h < H; h++)                                                    \
          y[s.y0 + t * H + h] = acc[t * H + h];                                             \
    }                                                                                       \
    free(acc);                                                                              \
    return bad ? -1 : 0;                                                                    \
  }

DEF_KERNEL_ORDER(d, double, fma)
DEF_KERNEL_ORDER(f, float, fmaf)

int orc_slell_spmv_kernel_order(const orc_slell *A, unsigned N, unsigned H, int tex_bounds,
                                int x_f64, const void *x, void *y)
{
  if (!is_pow2(N) || !is_pow2(H) || H > 4 || (A->hblock != 1 && A->hblock != 2 && A->hblock != 4))
    return -1;
  if (x_f64)
    return spmv_ko_d(A, N, H, tex_bounds, (const double *)x, (double *)y);
  return spmv_ko_f(A, N, H, tex_bounds, (const float *)x, (float *)y);
}

static double xget(int x_f64, const void *x, unsigned idx)
{
  return x_f64 ? ((const double *)x)[idx] : (double)((const float *)x)[idx];
}

static double eget(const orc_slell *A, unsigned i)
{
  return A->e_f64 ? ((const double *)A->elms)[i] : (double)((const float *)A->elms)[i];
}

int orc_slell_spmv_exact(const orc_slell *A, int tex, int x_f64, const void *x, double *y,
                         double *absrow)
{
  unsigned W = A->hblock;
  for (unsigned b = 0; b < A->n_slices; b++) {
    slice_hdr s;
    decode_slice(A, b, &s);
    unsigned sz = s.sz;
    if (!sz)
      continue;
    unsigned kc = (s.c1 - s.c0) / sz;
    for (unsigned r = 0; r < sz; r++) {
      long double acc = 0, aacc = 0;
      for (unsigned k = 0; k < kc; k++) {
        unsigned c = A->cols[s.c0 + r + k * sz];
        double e = eget(A, s.e0 + r + k * sz);
        double xv = c < (unsigned)A->n_cols ? xget(x_f64, x, c) : 0.0;
        acc += (long double)e * xv;
        aacc += fabsl((long double)e * xv);
      }
      if (A->diags) {
        unsigned nd = (s.e1 - s.e0 - kc * sz) / sz;
        for (unsigned d = 0; d < nd; d++) {
          unsigned c = A->slice_ptr[s.d0 + d] + r - sz;
          double e = eget(A, s.e0 + kc * sz + r + d * sz);
          double xv = c < (unsigned)A->n_cols ? xget(x_f64, x, c) : 0.0;
          acc += (long double)e * xv;
          aacc += fabsl((long double)e * xv);
        }
      } else if (W > 1) {
        unsigned nb = (s.cb - s.c1) / sz;
        for (unsigned bb = 0; bb < nb; bb++) {
          unsigned vc = A->cols[s.c1 + r + bb * sz];
          for (unsigned w = 0; w < W; w++) {
            unsigned c = vc * W + w;
            int ok = tex ? (vc < (unsigned)A->n_cols / W) : (c < (unsigned)A->n_cols);
            double e = eget(A, s.e1 + (bb * W + w) * sz + r);
            double xv = ok ? xget(x_f64, x, c) : 0.0;
            acc += (long double)e * xv;
            aacc += fabsl((long double)e * xv);
          }
        }
      }
      y[s.y0 + r] = (double)acc;
      if (absrow)
        absrow[s.y0 + r] = (double)aacc;
    }
  }
  return 0;
}

void orc_csr_spmv_f64(int n_rows, const int *row_ptr, const int *cols, const double *elms,
                      const double *x, double *y, double *absrow)
{
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n_rows; i++) {
    double acc = 0, aacc = 0;
    for (int k = row_ptr[i]; k < row_ptr[i + 1]; k++) {
      acc += elms[k] * x[cols[k]];
      aacc += fabs(elms[k] * x[cols[k]]);
    }
    y[i] = acc;
    if (absrow)
      absrow[i] = aacc;
  }
}

void orc_csr_spmv_f32e(int n_rows, const int *row_ptr, const int *cols, const float *elms,
                       const double *x, double *y)
{
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n_rows; i++) {
    double acc = 0;
    for (int k = row_ptr[i]; k < row_ptr[i + 1]; k++)
      acc += (double)elms[k] * x[cols[k]];
    y[i] = acc;
  }
}

void orc_copy_indexed(int f64, void *dst, const void *src, const int *idx, int n)
{
  for (int k = 0; k < n; k++) {
    if (f64)
      ((double *)dst)[k] = ((const double *)src)[idx[k]];
    else
      ((float *)dst)[k] = ((const float *)src)[idx[k]];
  }
}

void orc_add_indexed(int f64, void *dst, const void *src, const int *idx, int n)
{
  for (int k = 0; k < n; k++) {
    if (f64)
      ((double *)dst)[idx[k]] += ((const double *)src)[k];
    else
      ((float *)dst)[idx[k]] += ((const float *)src)[k];
  }
}

double orc_dot(int f64, const void *x, const void *y, int n)
{
  long double s = 0;
  for (int i = 0; i < n; i++)
    s += (long double)xget(f64, x, i) * (long double)xget(f64, y, i);
  return (double)s;
}

void orc_ppcg_update_scalars(int f64, void *alpha, void *beta, const void *gamma,
                             const void *gammaold, const void *delta)
{
  if (f64) {
    double g = *(const double *)gamma;
    double b = g / *(const double *)gammaold;
    *(double *)beta = b;
    *(double *)alpha = g / (*(const double *)delta - b * g / *(double *)alpha);
  } else {
    float g = *(const float *)gamma;
    float b = g / *(const float *)gammaold;
    *(float *)beta = b;
    *(float *)alpha = g / (*(const float *)delta - b * g / *(float *)alpha);
  }
}

#define DEF_UPD(SUF, T, FMA, FABS)                                                          \
  static void upd_##SUF(double *resnorm, double *gamma, double *delta, T a, T b,            \
                        const T *nv, const T *mv, T *p, T *s, T *q, T *z, T *x, T *r, T *u, \
                        T *w, int n)                                                        \
  {                                                                                         \
    long double rn = 0, ga = 0, de = 0;                                                     \
    for (int i = 0; i < n; i++) {                                                           \
      T wi = w[i], ui = u[i], zi, qi, si, pi, ri;                                           \
      z[i] = zi = FMA(b, z[i], nv[i]);                                                      \
      q[i] = qi = FMA(b, q[i], mv[i]);                                                      \
      s[i] = si = FMA(b, s[i], wi);                                                         \
      p[i] = pi = FMA(b, p[i], ui);                                                         \
      u[i] = ui = FMA(-a, qi, ui);                                                          \
      w[i] = wi = FMA(-a, zi, wi);                                                          \
      r[i] = ri = FMA(-a, si, r[i]);                                                        \
      x[i] = FMA(a, pi, x[i]);                                                              \
      rn += FABS(ri);                                                                       \
      ga += (long double)ri * ui;                                                           \
      de += (long double)wi * ui;                                                           \
    }                                                                                       \
    *resnorm = (double)rn;                                                                  \
    *gamma = (double)ga;                                                                    \
    *delta = (double)de;                                                                    \
  }
DEF_UPD(d, double, fma, fabs)
DEF_UPD(f, float, fmaf, fabsf)

void orc_ppcg_update_vectors(int f64, double *resnorm, double *gamma, double *delta,
                             const void *alpha, const void *beta, const void *nv,
                             const void *mv, void *p, void *s, void *q, void *z, void *x,
                             void *r, void *u, void *w, int n)
{
  if (f64)
    upd_d(resnorm, gamma, delta, *(const double *)alpha, *(const double *)beta,
          (const double *)nv, (const double *)mv, (double *)p, (double *)s, (double *)q,
          (double *)z, (double *)x, (double *)r, (double *)u, (double *)w, n);
  else
    upd_f(resnorm, gamma, delta, *(const float *)alpha, *(const float *)beta,
          (const float *)nv, (const float *)mv, (float *)p, (float *)s, (float *)q,
          (float *)z, (float *)x, (float *)r, (float *)u, (float *)w, n);
}

/* ---------------- FP64 PCG oracle ---------------- */

typedef struct {
  int n;
  const int *rp, *ci;
  const double *v;
} csr_ref;

static void csr_mv(const csr_ref *A, const double *x, double *y)
{
  orc_csr_spmv_f64(A->n, A->rp, A->ci, A->v, x, y, NULL);
}

static double dotd(const double *a, const double *b, int n)
{
  double s = 0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (int i = 0; i < n; i++)
    s += a[i] * b[i];
  return s;
}

static void prec(const csr_ref *G1, const csr_ref *G2, const double *v, double *out, double *tmp,
                 int n)
{
  if (!G1) {
    memcpy(out, v, sizeof(double) * n);
    return;
  }
  csr_mv(G1, v, tmp);
  csr_mv(G2, tmp, out);
}

static double true_relres(const csr_ref *A, const double *b, const double *x, double *tmp,
                          double bnorm)
{
  int n = A->n;
  csr_mv(A, x, tmp);
  double s = 0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (int i = 0; i < n; i++) {
    double d = b[i] - tmp[i];
    s += d * d;
  }
  return sqrt(s) / bnorm;
}

int orc_pcg_f64(int pipelined, int n, const int *A_rp, const int *A_ci, const double *A_v,
                const int *G1_rp, const int *G1_ci, const double *G1_v, const int *G2_rp,
                const int *G2_ci, const double *G2_v, const double *b, double *x, double tol,
                int max_it, double *relres)
{
  csr_ref A = {n, A_rp, A_ci, A_v};
  csr_ref G1s = {n, G1_rp, G1_ci, G1_v}, G2s = {n, G2_rp, G2_ci, G2_v};
  const csr_ref *G1 = G1_rp ? &G1s : NULL, *G2 = G2_rp ? &G2s : NULL;
  double *r = calloc(n, sizeof(double)), *u = calloc(n, sizeof(double));
  double *w = calloc(n, sizeof(double)), *p = calloc(n, sizeof(double));
  double *q = calloc(n, sizeof(double)), *s = calloc(n, sizeof(double));
  double *z = calloc(n, sizeof(double)), *m = calloc(n, sizeof(double));
  double *nv = calloc(n, sizeof(double)), *tmp = calloc(n, sizeof(double));
  double bnorm = sqrt(dotd(b, b, n));
  if (bnorm == 0)
    bnorm = 1;
  int it = 0;
  csr_mv(&A, x, tmp);
  for (int i = 0; i < n; i++)
    r[i] = b[i] - tmp[i];
  double rel = sqrt(dotd(r, r, n)) / bnorm;
  if (!pipelined) {
    prec(G1, G2, r, z, tmp, n);
    memcpy(p, z, sizeof(double) * n);
    double rz = dotd(r, z, n);
    while (rel > tol && it < max_it) {
      csr_mv(&A, p, q);
      double alpha = rz / dotd(p, q, n);
      for (int i = 0; i < n; i++) {
        x[i] += alpha * p[i];
        r[i] -= alpha * q[i];
      }
      it++;
      rel = sqrt(dotd(r, r, n)) / bnorm;
      if (rel <= tol)
        break;
      prec(G1, G2, r, z, tmp, n);
      double rzn = dotd(r, z, n);
      double beta = rzn / rz;
      rz = rzn;
      for (int i = 0; i < n; i++)
        p[i] = z[i] + beta * p[i];
    }
  } else {
    prec(G1, G2, r, u, tmp, n);
    csr_mv(&A, u, w);
    double gamma = dotd(r, u, n), delta = dotd(w, u, n);
    double gammaold = 0, alpha = 0, beta = 0;
    while (rel > tol && it < max_it) {
      prec(G1, G2, w, m, tmp, n);
      csr_mv(&A, m, nv);
      if (it == 0) {
        beta = 0;
        alpha = gamma / delta;
      } else {
        beta = gamma / gammaold;
        alpha = gamma / (delta - beta * gamma / alpha);
      }
      gammaold = gamma;
      double ga = 0, de = 0, rr = 0;
      for (int i = 0; i < n; i++) {
        z[i] = nv[i] + beta * z[i];
        q[i] = m[i] + beta * q[i];
        s[i] = w[i] + beta * s[i];
        p[i] = u[i] + beta * p[i];
        x[i] += alpha * p[i];
        r[i] -= alpha * s[i];
        u[i] -= alpha * q[i];
        w[i] -= alpha * z[i];
        ga += r[i] * u[i];
        de += w[i] * u[i];
        rr += r[i] * r[i];
      }
      gamma = ga;
      delta = de;
      it++;
      rel = sqrt(rr) / bnorm;
    }
  }
  double tr = true_relres(&A, b, x, tmp, bnorm);
  if (relres)
    *relres = tr;
  free(r); free(u); free(w); free(p); free(q); free(s); free(z); free(m); free(nv); free(tmp);
  return it;
}

/* FSAI rows on A's lower pattern (the construction fsai.cu runs on the GPU):
 * row i solves A[P,P] y = e_last with P = {j <= i : a_ij != 0} (A's sorted
 * row i up to its diagonal), then g = y / sqrt(y_last).  Dense Cholesky per
 * row in FP64; a local matrix that is not positive definite gives the Jacobi
 * row (1/sqrt(a_ii) when a_ii > 0, else 1). */
long long orc_fsai_pattern_size(const int *rp, const int *ci, const int *rows, int n_rows_out)
{
  long long s = 0;
  for (int k = 0; k < n_rows_out; k++) {
    const int i = rows[k];
    for (int e = rp[i]; e < rp[i + 1] && ci[e] <= i; e++)
      s++;
  }
  return s;
}

static double csr_at(const int *rp, const int *ci, const double *v, int r, int c)
{
  int lo = rp[r], hi = rp[r + 1];
  while (lo < hi) {
    int mid = (lo + hi) / 2;
    if (ci[mid] < c)
      lo = mid + 1;
    else
      hi = mid;
  }
  return (lo < rp[r + 1] && ci[lo] == c) ? v[lo] : 0.0;
}

long long orc_fsai_rows(const int *rp, const int *ci, const double *v, const int *rows,
                        int n_rows_out, int *out_rp, int *out_ci, double *out_v)
{
  out_rp[0] = 0;
  for (int k = 0; k < n_rows_out; k++) {
    const int i = rows[k];
    int K = 0;
    for (int e = rp[i]; e < rp[i + 1] && ci[e] <= i; e++)
      K++;
    out_rp[k + 1] = out_rp[k] + K;
  }
  long long jacobi = 0;
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : jacobi, bad)
  for (int k = 0; k < n_rows_out; k++) {
    const int i = rows[k];
    const int o = out_rp[k], K = out_rp[k + 1] - o;
    if (K > 64 || K == 0) {
      bad++;
      continue;
    }
    double L[64][64], y[64];
    int P[64];
    for (int a = 0; a < K; a++)
      P[a] = ci[rp[i] + a];
    for (int a = 0; a < K; a++)
      for (int b = 0; b <= a; b++)
        L[a][b] = csr_at(rp, ci, v, P[a], P[b]);
    int ok = 1;
    for (int c = 0; c < K && ok; c++) {
      double d = L[c][c];
      for (int t = 0; t < c; t++)
        d -= L[c][t] * L[c][t];
      if (!(d > 0.0)) {
        ok = 0;
        break;
      }
      L[c][c] = sqrt(d);
      for (int r = c + 1; r < K; r++) {
        double s = L[r][c];
        for (int t = 0; t < c; t++)
          s -= L[r][t] * L[c][t];
        L[r][c] = s / L[c][c];
      }
    }
    if (!ok) {
      const double aii = csr_at(rp, ci, v, i, i);
      for (int a = 0; a < K; a++) {
        out_ci[o + a] = P[a];
        out_v[o + a] = 0.0;
      }
      out_v[o + K - 1] = aii > 0.0 ? 1.0 / sqrt(aii) : 1.0;
      jacobi++;
      continue;
    }
    /* L L^T y = e_last: y_last = 1 / L_last^2, then back-substitute with L^T */
    for (int a = 0; a < K; a++)
      y[a] = 0.0;
    y[K - 1] = 1.0 / (L[K - 1][K - 1] * L[K - 1][K - 1]);
    for (int r = K - 2; r >= 0; r--) {
      double s = 0.0;
      for (int c = r + 1; c < K; c++)
        s += L[c][r] * y[c];
      y[r] = -s / L[r][r];
    }
    const double sc = 1.0 / sqrt(y[K - 1]);
    for (int a = 0; a < K; a++) {
      out_ci[o + a] = P[a];
      out_v[o + a] = y[a] * sc;
    }
  }
  return bad ? -1 : jacobi;
}
