// Factorized sparse approximate inverse built on the GPU.
//
// The reference builds its approximate inverse on the host, one factor row
// after another (right-looking AINV, fastainv/fastainv.cpp:395-566): every
// row update depends on the rows before it.  Here each row of a lower
// triangular factor G is independent -- the classic FSAI construction:
//
//     P_i = { j <= i : a_ij != 0 }            (the row's lower pattern of A)
//     A[P_i, P_i] y = e_i,   g_i = y / sqrt(y_i)
//
// so that diag(G A G^T) = 1 and M = G^T G ~ A^-1, with G's non-zeros on A's
// lower triangle.  On the 27-point GRF systems this preconditioner needs a
// few per cent more PCG iterations than the AINV factor with droptol 0.01
// while holding ~5% fewer non-zeros, and it is built in milliseconds instead
// of seconds.
//
// One warp per row: lanes gather the |P_i| x |P_i| local matrix (|P_i| <= 32)
// into shared memory, factor it (Cholesky) and back-substitute.  FP64
// throughout.  A local matrix that is not positive definite (indefinite A)
// falls back to the Jacobi row e_i / sqrt(a_ii) when a_ii > 0, else to e_i,
// and is counted.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "cuda_util.cuh"
#include "fsai.h"

namespace ispm {
namespace {

constexpr int kWarpsPerBlock = 4;  // 4 x 32 x 33 doubles = 33.8 KB of shared memory
constexpr int kMaxPattern = 32;

__global__ void __launch_bounds__(kWarpsPerBlock * 32)
    fsai_rows_kernel(int n, const int *__restrict__ a_rp, const int *__restrict__ a_ci,
                     const double *__restrict__ a_v, const int *__restrict__ g_rp,
                     double *__restrict__ g_v, unsigned *fallbacks)
{
  __shared__ double sm[kWarpsPerBlock][kMaxPattern][kMaxPattern + 1];
  __shared__ int pat[kWarpsPerBlock][kMaxPattern];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double(*L)[kMaxPattern + 1] = sm[w];
  const int i = blockIdx.x * kWarpsPerBlock + w;
  if (i >= n)
    return;  // whole warp leaves together
  const int g0 = g_rp[i], K = g_rp[i + 1] - g0;  // pattern = first K entries of row i
  const int a0 = a_rp[i];
  if (lane < K)
    pat[w][lane] = __ldg(a_ci + a0 + lane);
  __syncwarp();
  // Lane l gathers column l of A[P,P]: entries a(p_l, p_k), k < K, by merging
  // the (sorted) row p_l of A with the (sorted) pattern.
  if (lane < K) {
    const int row = pat[w][lane];
    int e = __ldg(a_rp + row);
    const int stop = __ldg(a_rp + row + 1);
    for (int k = 0; k < K; k++) {
      const int want = pat[w][k];
      while (e < stop && __ldg(a_ci + e) < want)
        e++;
      L[k][lane] = (e < stop && __ldg(a_ci + e) == want) ? __ldg(a_v + e) : 0.0;
    }
  }
  __syncwarp();
  // Cholesky, right-looking, lower triangle; lane j owns column j.
  bool ok = true;
  for (int k = 0; k < K; k++) {
    const double d = L[k][k];
    if (!(d > 0.0)) {
      ok = false;
      break;  // uniform: every lane reads the same shared value
    }
    const double lkk = sqrt(d);
    __syncwarp();
    if (lane == k)
      L[k][k] = lkk;
    if (lane > k && lane < K)
      L[lane][k] /= lkk;
    __syncwarp();
    // trailing update of column j = lane (rows i >= j)
    if (lane > k && lane < K) {
      const double ljk = L[lane][k];
      for (int r = lane; r < K; r++)
        L[r][lane] -= L[r][k] * ljk;
    }
    __syncwarp();
  }
  if (!ok) {
    // Jacobi fallback on the diagonal entry (the last pattern slot is i)
    if (lane == 0) {
      const double aii = __ldg(a_v + a0 + K - 1);
      atomicAdd(fallbacks, 1u);
      for (int k = 0; k < K - 1; k++)
        g_v[g0 + k] = 0.0;
      g_v[g0 + K - 1] = aii > 0.0 ? 1.0 / sqrt(aii) : 1.0;
    }
    return;
  }
  // L L^T y = e_{K-1}: y_{K-1} = 1 / L_{K-1,K-1}^2, then back-substitute;
  // g = y / sqrt(y_{K-1}) = y * L_{K-1,K-1}.  Sequential in lane 0 (K <= 32).
  if (lane == 0) {
    double y[kMaxPattern];
    const double lnn = L[K - 1][K - 1];
    y[K - 1] = 1.0 / (lnn * lnn);
    for (int r = K - 2; r >= 0; r--) {
      double s = 0.0;
      for (int c = r + 1; c < K; c++)
        s = fma(L[c][r], y[c], s);
      y[r] = -s / L[r][r];
    }
    for (int k = 0; k < K; k++)
      g_v[g0 + k] = y[k] * lnn;
  }
}

}  // namespace

int fsai_lower_pattern(int n, const int *rp, const int *ci, std::vector<int> &g_rp,
                       std::vector<int> &g_ci)
{
  g_rp.assign(n + 1, 0);
  for (int i = 0; i < n; i++) {
    int cnt = 0, last = -1;
    for (int e = rp[i]; e < rp[i + 1]; e++) {
      if (ci[e] <= last || ci[e] < 0 || ci[e] >= n)
        return fail(ISPM_ERR_INVALID, "row %d columns not strictly increasing in [0, n)", i);
      last = ci[e];
      if (ci[e] <= i)
        cnt++;
    }
    if (cnt == 0 || ci[rp[i] + cnt - 1] != i)
      return fail(ISPM_ERR_INVALID, "row %d has no diagonal entry", i);
    if (cnt > kMaxPattern)
      return fail(ISPM_ERR_TOO_LARGE, "row %d has %d lower entries (at most %d)", i, cnt,
                  kMaxPattern);
    g_rp[i + 1] = g_rp[i] + cnt;
  }
  g_ci.resize(g_rp[n]);
  for (int i = 0; i < n; i++)
    std::copy(ci + rp[i], ci + rp[i] + (g_rp[i + 1] - g_rp[i]), g_ci.begin() + g_rp[i]);
  return ISPM_OK;
}

void fsai_transpose_pattern(int n, const std::vector<int> &g_rp, const std::vector<int> &g_ci,
                            std::vector<int> &t_rp, std::vector<int> &t_ci,
                            std::vector<unsigned> &t_of)
{
  // G^T in CSR; t_of[k] = position in G^T of G's entry k
  t_rp.assign(n + 1, 0);
  for (int c : g_ci)
    t_rp[c + 1]++;
  for (int i = 0; i < n; i++)
    t_rp[i + 1] += t_rp[i];
  t_ci.resize(g_ci.size());
  t_of.resize(g_ci.size());
  std::vector<int> fill(t_rp.begin(), t_rp.end() - 1);
  for (int i = 0; i < n; i++)
    for (int e = g_rp[i]; e < g_rp[i + 1]; e++) {
      const int at = fill[g_ci[e]]++;
      t_ci[at] = i;
      t_of[e] = (unsigned)at;
    }
}

int fsai_build_values(int n, const int *a_rp_d, const int *a_ci_d, const double *a_v_d,
                      const int *g_rp_d, double *g_v_d, unsigned *fallbacks_d, cudaStream_t s)
{
  const int blocks = (n + kWarpsPerBlock - 1) / kWarpsPerBlock;
  fsai_rows_kernel<<<blocks, kWarpsPerBlock * 32, 0, s>>>(n, a_rp_d, a_ci_d, a_v_d, g_rp_d,
                                                          g_v_d, fallbacks_d);
  cudaError_t e = cudaPeekAtLastError();
  return e == cudaSuccess ? ISPM_OK : fail(ISPM_ERR_CUDA, "fsai rows: %s", cudaGetErrorString(e));
}

}  // namespace ispm

using namespace ispm;

namespace {

struct Scoped {
  std::vector<void *> p;
  ~Scoped()
  {
    for (void *q : p)
      cudaFree(q);
  }
  template <class T> int get(T **out, size_t count, const T *init = nullptr)
  {
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(ISPM_ERR_NOMEM, "cudaMalloc: %s", cudaGetErrorString(e));
    }
    p.push_back(q);
    *out = (T *)q;
    if (init && count)
      ISPM_CUDA_TRY(cudaMemcpy(q, init, count * sizeof(T), cudaMemcpyHostToDevice));
    return ISPM_OK;
  }
};

}  // namespace

extern "C" int ispm_fsai_sym_gpu(int out_dtype, int n, const int *row_ptr, const int *cols,
                                 const double *elms, ispm_csr **ainv1, ispm_csr **ainv2,
                                 unsigned *fallbacks)
{
  clear_error();
  if (!ainv1 || !ainv2)
    return fail(ISPM_ERR_INVALID, "output pointers are NULL");
  *ainv1 = *ainv2 = nullptr;
  if (n <= 0 || !row_ptr || (row_ptr[n] && (!cols || !elms)))
    return fail(ISPM_ERR_INVALID, "bad CSR");
  if (out_dtype != ISPM_F32 && out_dtype != ISPM_F64)
    return fail(ISPM_ERR_INVALID, "out_dtype %d", out_dtype);
  std::vector<int> g_rp, g_ci, t_rp, t_ci;
  std::vector<unsigned> t_of;
  if (int e = fsai_lower_pattern(n, row_ptr, cols, g_rp, g_ci))
    return e;
  fsai_transpose_pattern(n, g_rp, g_ci, t_rp, t_ci, t_of);
  const size_t nnz_a = (size_t)row_ptr[n], nnz_g = g_ci.size();
  Scoped mem;
  int *a_rp, *a_ci, *gr;
  double *a_v, *g_v;
  unsigned *fb;
  if (int e = mem.get(&a_rp, (size_t)n + 1, row_ptr))
    return e;
  if (int e = mem.get(&a_ci, nnz_a, cols))
    return e;
  if (int e = mem.get(&a_v, nnz_a, elms))
    return e;
  if (int e = mem.get(&gr, (size_t)n + 1, g_rp.data()))
    return e;
  if (int e = mem.get(&g_v, nnz_g))
    return e;
  if (int e = mem.get(&fb, 1))
    return e;
  ISPM_CUDA_TRY(cudaMemset(fb, 0, sizeof(unsigned)));
  if (int e = fsai_build_values(n, a_rp, a_ci, a_v, gr, g_v, fb, 0))
    return e;
  std::vector<double> gv(nnz_g);
  ISPM_CUDA_TRY(cudaMemcpy(gv.data(), g_v, nnz_g * sizeof(double), cudaMemcpyDeviceToHost));
  unsigned nfb = 0;
  ISPM_CUDA_TRY(cudaMemcpy(&nfb, fb, sizeof(unsigned), cudaMemcpyDeviceToHost));
  if (fallbacks)
    *fallbacks = nfb;
  ispm_csr *g1 = new (std::nothrow) ispm_csr, *g2 = new (std::nothrow) ispm_csr;
  if (!g1 || !g2) {
    delete g1;
    delete g2;
    return fail(ISPM_ERR_NOMEM, "host allocation");
  }
  // Ainv1 = G (lower), Ainv2 = G^T, so Ainv2 Ainv1 = G^T G ~ A^-1 as for fastainv_sym
  for (ispm_csr *g : {g1, g2}) {
    g->m.n_rows = g->m.n_cols = n;
    g->m.n_nz = (int)nnz_g;
    g->m.dtype = out_dtype;
  }
  g1->m.row_ptr = g_rp;
  g1->m.cols = g_ci;
  g2->m.row_ptr = t_rp;
  g2->m.cols = t_ci;
  std::vector<double> tv(nnz_g);
  for (size_t k = 0; k < nnz_g; k++)
    tv[t_of[k]] = gv[k];
  if (out_dtype == ISPM_F64) {
    g1->m.elms_d = std::move(gv);
    g2->m.elms_d = std::move(tv);
  } else {
    g1->m.elms_f.assign(gv.begin(), gv.end());
    g2->m.elms_f.assign(tv.begin(), tv.end());
  }
  *ainv1 = g1;
  *ainv2 = g2;
  return ISPM_OK;
}
