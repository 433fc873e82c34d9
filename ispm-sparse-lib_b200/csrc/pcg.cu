// Preconditioned pipelined CG on sliced-ELL operands with FP64 reliable
// updates.
//
// The reference ships the primitives of this loop -- SpMV
// (cuda/spmv/kernel-iface.h), ppcg_update_scalars / ppcg_update_vectors
// (util/cuda/sblas.cu:156-237) and the FSAI pair from fastainv_sym -- and
// leaves the loop itself to an external driver.  This file is that driver,
// B200-first:
//  * one iteration = three SpMVs (t = G' w, m = H' t, n = A m) and one fused
//    update kernel that also derives alpha / beta on the device, so an
//    iteration never waits on the host; chunks of iterations are captured in
//    a CUDA graph and replayed, and a device "done" flag turns the rest of a
//    chunk into no-ops as soon as the solve needs the host;
//  * reductions (gamma = r.u, delta = w.u, ||r||^2) accumulate in FP64 and
//    finish in the last CTA of the update launch;
//  * inner precision T is FP64 (plain) or FP32 (mixed: FP32 matrices and
//    vectors, FP64 reductions);
//  * reliable updates (residual replacement): whenever the recursive residual
//    has dropped by `replace_ratio` since the last update, or meets the
//    target, the correction accumulated in T is folded into the FP64 iterate,
//    r = b - A x is recomputed with the FP64 matrix, and the pipelined
//    auxiliaries are re-derived from it (u = M r, w = A u, s = A p, q = M s,
//    z = A q) without restarting the Krylov recurrence.  This bounds the
//    drift between the recursive and the true residual that otherwise stalls
//    pipelined CG in FP32 (and limits its attainable accuracy in FP64);
//  * the FSAI pair is stored as G' = P Ainv1 (rows reversed) and H' = Ainv2 P
//    (columns reversed), P the index reversal: M = Ainv2 Ainv1 = H' G', and
//    both factors become banded with stencil-like diagonals that the
//    diagonal-block format captures (Ainv1 itself runs along anti-diagonals).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <vector>

#include "cuda_util.cuh"
#include "fsai.h"
#include "nvtx_range.h"
#include "operator.h"
#include "pcg_state.h"
#include "sblas_impl.h"
#include "spmv_launch.h"

namespace ispm {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 1024;
// Smallest reliable-update ratio with an FP16-stored inner matrix
// (ispm_solver_opts.matrix_f16).
constexpr double kSplitReplaceRatio = 3e-2;

struct Scratch {
  double *part;  // 4 * kMaxBlocks partials
  unsigned *ticket;
};

template <int NV> struct Acc {
  double v[NV];
};

template <int NV> __device__ __forceinline__ Acc<NV> block_sum(Acc<NV> a)
{
  __shared__ double sh[NV][32];
#pragma unroll
  for (int k = 0; k < NV; k++)
    for (int off = 16; off > 0; off >>= 1)
      a.v[k] += __shfl_down_sync(0xffffffffu, a.v[k], off);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; k++)
      sh[k][warp] = a.v[k];
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) {
      a.v[k] = lane < nw ? sh[k][lane] : 0.0;
      for (int off = 16; off > 0; off >>= 1)
        a.v[k] += __shfl_down_sync(0xffffffffu, a.v[k], off);
    }
  }
  __syncthreads();
  return a;
}

// Publish per-block partials; true in the last block, whose thread 0 holds
// the block-ordered totals.
template <int NV> __device__ bool grid_total(Acc<NV> a, Scratch sc, Acc<NV> &tot)
{
  __shared__ bool last;
  a = block_sum<NV>(a);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++)
      sc.part[k * kMaxBlocks + blockIdx.x] = a.v[k];
    __threadfence();
    last = atomicAdd(sc.ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last)
    return false;
  __threadfence();
  Acc<NV> s;
#pragma unroll
  for (int k = 0; k < NV; k++) {
    s.v[k] = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
      s.v[k] += __ldcg(sc.part + k * kMaxBlocks + b);
  }
  tot = block_sum<NV>(s);
  if (threadIdx.x == 0)
    *sc.ticket = 0u;
  return true;
}

#define GRID_STRIDE(i, n) \
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (n); \
       i += (long long)gridDim.x * blockDim.x)

template <class T> struct Vec16;
template <> struct Vec16<float> {
  using type = float4;
  static constexpr int n = 4;
};
template <> struct Vec16<double> {
  using type = double2;
  static constexpr int n = 2;
};

// x += d (FP64 iterate, correction in T), d = 0; then r64 = b - A x needs the
// SpMV, done separately.
template <class T>
__global__ void __launch_bounds__(kThreads)
    fold_correction_kernel(double *__restrict__ x, T *__restrict__ d, long long n)
{
  GRID_STRIDE(i, n)
  {
    x[i] += (double)d[i];
    d[i] = T(0);
  }
}

// r64 = b - Ax, res2 = ||r64||^2
__global__ void __launch_bounds__(kThreads)
    true_residual_kernel(const double *__restrict__ b, const double *__restrict__ ax,
                         double *__restrict__ r, long long n, PcgState *st, Scratch sc)
{
  Acc<1> a{{0.0}};
  GRID_STRIDE(i, n)
  {
    double v = b[i] - ax[i];
    r[i] = v;
    a.v[0] = fma(v, v, a.v[0]);
  }
  Acc<1> tot;
  if (grid_total<1>(a, sc, tot) && threadIdx.x == 0)
    st->res2 = tot.v[0];
}

// r = (T) r64 on the real rows (0 on padding); on a full restart also zero
// the search-direction recurrences.
template <class T>
__global__ void __launch_bounds__(kThreads)
    load_residual_kernel(const double *__restrict__ r64, T *r, T *d, T *p, T *s, T *q, T *z,
                         long long n, long long n_pad, int restart)
{
  GRID_STRIDE(i, n_pad)
  {
    r[i] = i < n ? (T)r64[i] : T(0);
    d[i] = T(0);
    if (restart) {
      p[i] = T(0);
      s[i] = T(0);
      q[i] = T(0);
      z[i] = T(0);
    }
  }
}

// gamma = r.u, delta = w.u, rr = r.r after a (re)start; keeps the previous
// alpha / gamma on a replacement so the recurrence continues.
template <class T>
__global__ void __launch_bounds__(kThreads)
    sync_dots_kernel(const T *__restrict__ r, const T *__restrict__ u, const T *__restrict__ w,
                     long long n, PcgState *st, Scratch sc, double thresh2, double ru2,
                     int max_it, int restart)
{
  Acc<3> a{{0.0, 0.0, 0.0}};
  GRID_STRIDE(i, n)
  {
    double ri = r[i], ui = u[i], wi = w[i];
    a.v[0] = fma(ri, ui, a.v[0]);
    a.v[1] = fma(wi, ui, a.v[1]);
    a.v[2] = fma(ri, ri, a.v[2]);
  }
  Acc<3> tot;
  if (grid_total<3>(a, sc, tot) && threadIdx.x == 0) {
    st->gamma = tot.v[0];
    st->delta = tot.v[1];
    st->rr = tot.v[2];
    st->rr_ref = tot.v[2];
    st->thresh2 = thresh2;
    st->ru2 = ru2;
    if (restart) {
      st->gammaold = 0;
      st->alpha = 0;
      st->beta = 0;
      st->it = 0;
    }
    st->max_it = max_it;
    st->done = tot.v[2] <= thresh2 ? kConverged : kRunning;
  }
}

// One pipelined-CG step (sblas.cu:156-216): scalars from the device state,
// z = n + b z, q = m + b q, s = w + b s, p = u + b p, d += a p, r -= a s,
// u -= a q, w -= a z, then gamma, delta and ||r||^2 of the new vectors.
template <class T>
__global__ void __launch_bounds__(kThreads)
    pcg_step_kernel(const T *__restrict__ nv, const T *__restrict__ mv, T *__restrict__ p,
                    T *__restrict__ s, T *__restrict__ q, T *__restrict__ z, T *__restrict__ d,
                    T *__restrict__ r, T *__restrict__ u, T *__restrict__ w, long long n,
                    PcgState *st, Scratch sc)
{
  if (st->done)
    return;
  const double g = st->gamma, de = st->delta;
  double beta, alpha;
  if (st->it == 0) {
    beta = 0.0;
    alpha = g / de;
  } else {
    beta = g / st->gammaold;
    alpha = g / (de - beta * g / st->alpha);
  }
  if (!(alpha > 0.0) || !isfinite(alpha) || !isfinite(beta)) {
    // Lost positive definiteness in finite precision: stop; the host folds
    // the correction in and restarts from the true residual.
    if (blockIdx.x == 0 && threadIdx.x == 0)
      st->done = kBreakdown;
    return;
  }
  const T a = (T)alpha, b = (T)beta;
  Acc<3> acc{{0.0, 0.0, 0.0}};
  GRID_STRIDE(i, n)
  {
    T wi = w[i], ui = u[i];
    T zi = fma(b, z[i], nv[i]);
    T qi = fma(b, q[i], mv[i]);
    T si = fma(b, s[i], wi);
    T pi = fma(b, p[i], ui);
    ui = fma(-a, qi, ui);
    wi = fma(-a, zi, wi);
    T ri = fma(-a, si, r[i]);
    d[i] = fma(a, pi, d[i]);
    z[i] = zi;
    q[i] = qi;
    s[i] = si;
    p[i] = pi;
    u[i] = ui;
    w[i] = wi;
    r[i] = ri;
    acc.v[0] = fma((double)ri, (double)ui, acc.v[0]);
    acc.v[1] = fma((double)wi, (double)ui, acc.v[1]);
    acc.v[2] = fma((double)ri, (double)ri, acc.v[2]);
  }
  Acc<3> tot;
  if (grid_total<3>(acc, sc, tot) && threadIdx.x == 0) {
    st->gammaold = g;
    st->alpha = alpha;
    st->beta = beta;
    st->gamma = tot.v[0];
    st->delta = tot.v[1];
    st->rr = tot.v[2];
    st->it += 1;
    if (!isfinite(tot.v[2]) || !isfinite(tot.v[0]))
      st->done = kBreakdown;
    else if (tot.v[2] <= st->thresh2)
      st->done = kConverged;
    else if (tot.v[2] < st->ru2 * st->rr_ref)
      st->done = kReplace;
    else if (st->it >= st->max_it)
      st->done = kCap;
  }
}

// ---- classic PCG (one recurrence, r; the dots p.Ap and r.z come fused out
// of the SpMVs that produce Ap and z) ----------------------------------------

// alpha = rz / pq; d += alpha p; r -= alpha q.
// Without a preconditioner (noprec) also rr = ||r||^2 (= r.z) and the stop
// test, finished in the last block.  With one, r.r comes with r.z from the
// G^T SpMV and the stop test runs at the head of the direction step; this
// kernel then has no reduction: alpha = rz_new / pq, and block 0 rolls the
// scalars (rz = rz_new, fresh = 0, it += 1) -- the direction step that read
// the old values has finished, and no block here reads them.
template <class T>
__global__ void __launch_bounds__(kThreads)
    cg_update_kernel(const T *__restrict__ p, const T *__restrict__ q, T *__restrict__ r,
                     T *__restrict__ d, long long n, PcgState *st, Scratch sc, int noprec)
{
  pdl_wait();
  if (st->done)
    return;
  const double alpha = (noprec ? st->rz : st->rz_new) / st->pq;
  if (!(alpha > 0.0) || !isfinite(alpha)) {
    if (blockIdx.x == 0 && threadIdx.x == 0)
      st->done = kBreakdown;
    return;
  }
  const T a = (T)alpha;
  Acc<1> acc{{0.0}};
  // 128-bit words: n is a multiple of 512 and the vectors are cudaMalloc'd
  using V = typename Vec16<T>::type;
  constexpr int K = Vec16<T>::n;
  GRID_STRIDE(i, n / K)
  {
    V pv = reinterpret_cast<const V *>(p)[i], qv = __ldcs(reinterpret_cast<const V *>(q) + i);
    V rv = reinterpret_cast<const V *>(r)[i], dv = reinterpret_cast<const V *>(d)[i];
    T *P = reinterpret_cast<T *>(&pv), *Q = reinterpret_cast<T *>(&qv);
    T *Rr = reinterpret_cast<T *>(&rv), *D = reinterpret_cast<T *>(&dv);
#pragma unroll
    for (int k = 0; k < K; k++) {
      Rr[k] = fma(-a, Q[k], Rr[k]);
      D[k] = fma(a, P[k], D[k]);
      acc.v[0] = fma((double)Rr[k], (double)Rr[k], acc.v[0]);
    }
    reinterpret_cast<V *>(r)[i] = rv;
    reinterpret_cast<V *>(d)[i] = dv;
  }
  pdl_trigger();
  if (!noprec) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      st->alpha = alpha;
      st->rz = st->rz_new;
      st->fresh = 0;
      st->it += 1;
    }
    return;
  }
  Acc<1> tot;
  if (grid_total<1>(acc, sc, tot) && threadIdx.x == 0) {
    st->alpha = alpha;
    st->rr = tot.v[0];
    if (noprec)
      st->rz_new = tot.v[0];
    st->it += 1;
    cg_flags(st, tot.v[0]);
  }
}

// beta = rz_new / rz (0 on a fresh start); p = z + beta p.
// noprec: the last block rolls rz = rz_new (the update's stop test already
// ran).  With a preconditioner: every block first evaluates the stop test on
// rr (from the G^T SpMV) and block 0 records it; the scalars roll in the
// next update kernel, so no cross-block finish is needed here.
// loop: launched inside the body of a graph's while node; block 0 ends the
// loop (condition 0) once the solve needs the host.
template <class T>
__global__ void __launch_bounds__(kThreads)
    cg_direction_kernel(const T *__restrict__ z, T *__restrict__ p, long long n, PcgState *st,
                        Scratch sc, int noprec, cudaGraphConditionalHandle loop, int in_loop)
{
  pdl_wait();
  const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
  if (st->done) {
    if (in_loop && lead)
      cudaGraphSetConditional(loop, 0u);
    return;
  }
  if (!noprec) {
    const double rr = st->rr;
    if (cg_stop(st, rr)) {
      if (lead) {
        cg_flags(st, rr);
        if (in_loop)
          cudaGraphSetConditional(loop, 0u);
      }
      return;
    }
  }
  const bool fresh = st->fresh;
  const double rzn = st->rz_new;
  const double beta = fresh ? 0.0 : rzn / st->rz;
  if (!(rzn > 0.0) || !isfinite(beta)) {
    // M is not positive definite on this residual (or r vanished exactly)
    if (lead) {
      st->done = rzn == 0.0 ? kConverged : kBreakdown;
      if (in_loop)
        cudaGraphSetConditional(loop, 0u);
    }
    return;
  }
  const T b = (T)beta;
  using V = typename Vec16<T>::type;
  constexpr int K = Vec16<T>::n;
  if (fresh) {
    GRID_STRIDE(i, n / K)
    reinterpret_cast<V *>(p)[i] = reinterpret_cast<const V *>(z)[i];
  } else {
    GRID_STRIDE(i, n / K)
    {
      V zv = reinterpret_cast<const V *>(z)[i], pv = reinterpret_cast<const V *>(p)[i];
      T *Z = reinterpret_cast<T *>(&zv), *P = reinterpret_cast<T *>(&pv);
#pragma unroll
      for (int k = 0; k < K; k++)
        P[k] = fma(b, P[k], Z[k]);
      reinterpret_cast<V *>(p)[i] = pv;
    }
  }
  pdl_trigger();
  if (!noprec)
    return;
  Acc<1> none{{0.0}}, tot;
  if (grid_total<1>(none, sc, tot) && threadIdx.x == 0) {
    st->beta = beta;
    st->rz = rzn;
    st->fresh = 0;
  }
}

// r = (T) r64 (0 on padding), d = 0, rr = ||r||^2; arms the phase.
template <class T>
__global__ void __launch_bounds__(kThreads)
    cg_load_kernel(const double *__restrict__ r64, T *r, T *d, long long n, long long n_pad,
                   PcgState *st, Scratch sc, double thresh2, double ru2, int max_it,
                   int restart, int noprec)
{
  Acc<1> acc{{0.0}};
  GRID_STRIDE(i, n_pad)
  {
    T ri = i < n ? (T)r64[i] : T(0);
    r[i] = ri;
    d[i] = T(0);
    acc.v[0] = fma((double)ri, (double)ri, acc.v[0]);
  }
  Acc<1> tot;
  if (grid_total<1>(acc, sc, tot) && threadIdx.x == 0) {
    st->rr = tot.v[0];
    st->rr_ref = tot.v[0];
    st->thresh2 = thresh2;
    st->ru2 = ru2;
    st->max_it = max_it;
    if (noprec)
      st->rz_new = tot.v[0];
    if (restart) {
      st->it = 0;
      st->fresh = 1;
    }
    st->done = tot.v[0] <= thresh2 ? kConverged : kRunning;
  }
}

// Reordered solves: out[i] = in[perm[i]] (b into the solver's order) and
// out[perm[i]] = in[i] (x back), i < n.
__global__ void permute_in_kernel(double *__restrict__ out, const double *__restrict__ in,
                                  const int *__restrict__ perm, long long n)
{
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = in[perm[i]];
}

__global__ void permute_out_kernel(double *__restrict__ out, const double *__restrict__ in,
                                   const int *__restrict__ perm, long long n)
{
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[perm[i]] = in[i];
}

int grid_for(long long n)
{
  long long blocks = (n + kThreads - 1) / kThreads;
  // about one full wave of 256-thread CTAs (8 per SM) for the streaming kernels
  long long cap = std::min<long long>(kMaxBlocks, (long long)device_sm_count() * 8);
  return (int)std::max(1LL, std::min(blocks, cap));
}

struct DevMem {
  std::vector<void *> blocks;
  ~DevMem()
  {
    for (void *p : blocks)
      cudaFree(p);
  }
  template <class T> int get(T **out, size_t count)
  {
    void *p = nullptr;
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T) + 256;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(ISPM_ERR_NOMEM, "solver cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
    }
    blocks.push_back(p);
    e = cudaMemset(p, 0, bytes);
    if (e != cudaSuccess)
      return fail(ISPM_ERR_CUDA, "cudaMemset: %s", cudaGetErrorString(e));
    *out = (T *)p;
    return ISPM_OK;
  }
};

bool is_lower(int n, const int *rp, const int *ci)
{
  for (int i = 0; i < n; i++)
    for (int e = rp[i]; e < rp[i + 1]; e++)
      if (ci[e] > i)
        return false;
  return true;
}

// CSR -> reversed forms used for the factors.
void reverse_rows(int n, const int *rp, const int *ci, const double *v, std::vector<int> &orp,
                  std::vector<int> &oci, std::vector<double> &ov)
{
  orp.assign(n + 1, 0);
  oci.resize(rp[n]);
  ov.resize(rp[n]);
  int at = 0;
  for (int i = 0; i < n; i++) {
    int src = n - 1 - i;
    for (int e = rp[src]; e < rp[src + 1]; e++, at++) {
      oci[at] = ci[e];
      ov[at] = v[e];
    }
    orp[i + 1] = at;
  }
}

void reverse_cols(int n, const int *rp, const int *ci, const double *v, std::vector<int> &orp,
                  std::vector<int> &oci, std::vector<double> &ov)
{
  orp.assign(rp, rp + n + 1);
  oci.resize(rp[n]);
  ov.resize(rp[n]);
  for (int i = 0; i < n; i++) {
    int lo = rp[i], hi = rp[i + 1];
    for (int e = lo; e < hi; e++) {
      oci[lo + (hi - 1 - e)] = n - 1 - ci[e];
      ov[lo + (hi - 1 - e)] = v[e];
    }
  }
}

}  // namespace

struct Solver {
  int n = 0, n_pad = 0;
  ispm_solver_opts opts{};
  int inner = ISPM_F64;  // inner vector / matrix type
  bool have_prec = false;
  Operator A64, Ain, G, Ht;
  DevMem mem;
  PcgState *st = nullptr;
  PcgState *st_host = nullptr;  // pinned mirror
  Scratch sc{};
  unsigned part_capacity = 0;  // partial slots in sc.part
  bool classic = false;        // classic PCG instead of the pipelined recurrence
  unsigned fsai_fallbacks = 0; // GPU FSAI rows built as Jacobi rows
  double *x64 = nullptr, *r64 = nullptr, *t64 = nullptr, *b64 = nullptr;
  double *b_stage = nullptr, *x_stage = nullptr;  // device copies for host-vector solves
  // reordered solves: perm[new] = old, and b / x in the solver's order
  int *perm = nullptr;
  double *b_perm = nullptr, *x_perm = nullptr;
  // opts.refresh: what ispm_solver_update_values needs.  pos_*: CSR entry
  // (solver order) -> element slot of each device copy of A; entry_src: for
  // a renumbered solve, solver-order entry -> caller-order entry; a_v: A's
  // values in solver order (device); fsai: the factor build's device arrays.
  bool refreshable = false;
  long long nnz_a = 0;
  unsigned *pos_ain = nullptr, *pos_a64 = nullptr;
  int *entry_src = nullptr;
  double *a_v = nullptr, *a_raw = nullptr;
  struct FsaiArrays {
    int *a_rp = nullptr, *a_ci = nullptr, *g_rp = nullptr;
    unsigned *t_of = nullptr, *pos_g = nullptr, *pos_t = nullptr, *fb = nullptr;
    double *g_v = nullptr, *gt_v = nullptr;
    long long nnz_g = 0;
    bool f16 = false;
  } fsai;
  bool fsai_kept = false;
  void *vec[11] = {};
  enum { R, U, W, M, NV, P, S, Q, Z, D, TT };
  cudaGraphExec_t graph = nullptr;
  // use_graph 2 (classic iteration): the chunk is the body of the graph's
  // while node, whose condition the direction kernel clears; set while the
  // body is being captured
  cudaGraphConditionalHandle loop = 0;
  bool capturing_loop = false;
  // The solve runs on the solver's own stream (the legacy default stream
  // cannot be captured into a graph), ordered after / before the caller's
  // stream with two events.
  cudaStream_t own = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  std::vector<double> history;
  int replacements = 0, restarts = 0;
  // ISPM_SOLVER_VERBOSE=1: one stderr line per solver phase (diagnostics)
  bool verbose = getenv("ISPM_SOLVER_VERBOSE") && atoi(getenv("ISPM_SOLVER_VERBOSE")) > 0;

  ~Solver()
  {
    if (graph)
      cudaGraphExecDestroy(graph);
    if (st_host)
      cudaFreeHost(st_host);
    if (ev_in)
      cudaEventDestroy(ev_in);
    if (ev_out)
      cudaEventDestroy(ev_out);
    if (own)
      cudaStreamDestroy(own);
  }

  size_t esize() const { return inner == ISPM_F32 ? 4 : 8; }

  int init_stream()
  {
    ISPM_CUDA_TRY(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking));
    ISPM_CUDA_TRY(cudaEventCreateWithFlags(&ev_in, cudaEventDisableTiming));
    ISPM_CUDA_TRY(cudaEventCreateWithFlags(&ev_out, cudaEventDisableTiming));
    return ISPM_OK;
  }

  int launched(const char *what)
  {
    cudaError_t e = cudaPeekAtLastError();
    return e == cudaSuccess ? ISPM_OK : fail(ISPM_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  }

  // out = M in (two SpMVs), or a copy without a preconditioner.
  int prec(const void *in, void *out, cudaStream_t s, const int *skip)
  {
    if (!have_prec) {
      ISPM_CUDA_TRY(cudaMemcpyAsync(out, in, (size_t)n_pad * esize(), cudaMemcpyDeviceToDevice, s));
      return ISPM_OK;
    }
    if (int e = G.apply(inner, in, vec[TT], s, skip))
      return e;
    return Ht.apply(inner, vec[TT], out, s, skip);
  }

  template <class T> int step(cudaStream_t s)
  {
    pcg_step_kernel<T><<<grid_for(n_pad), kThreads, 0, s>>>(
        (const T *)vec[NV], (const T *)vec[M], (T *)vec[P], (T *)vec[S], (T *)vec[Q],
        (T *)vec[Z], (T *)vec[D], (T *)vec[R], (T *)vec[U], (T *)vec[W], n_pad, st, sc);
    return launched("pcg step");
  }

  // One iteration.  Pipelined: m = M w, n = A m, fused update.  Classic:
  // q = A p (+ p.q), d/r update (+ r.r), z = M r (+ r.z), new direction.
  int iteration(cudaStream_t s)
  {
    const int *skip = &st->done;
    if (classic)
      return inner == ISPM_F32 ? cg_iteration<float>(s) : cg_iteration<double>(s);
    if (int e = prec(vec[W], vec[M], s, skip))
      return e;
    if (int e = Ain.apply(inner, vec[M], vec[NV], s, skip))
      return e;
    return inner == ISPM_F32 ? step<float>(s) : step<double>(s);
  }

  SpmvDot dot_into(const void *v, double *out) const
  {
    SpmvDot ep;
    ep.v = v;
    ep.out = out;
    ep.part = sc.part;
    ep.ticket = sc.ticket;
    ep.part_capacity = part_capacity;
    return ep;
  }

  // z = M r with r.z fused into the last SpMV; without a preconditioner
  // z = r and r.z was produced with r.r.
  template <class T> int cg_precondition(cudaStream_t s, const int *skip)
  {
    if (!have_prec)
      return ISPM_OK;
    if (int e = G.apply(inner, vec[R], vec[TT], s, skip, nullptr, true))
      return e;
    SpmvDot ep = dot_into(vec[R], &st->rz_new);
    ep.out2 = &st->rr;  // r.r from the same pass over r (the stop test's input)
    return Ht.apply(inner, vec[TT], vec[Z], s, skip, &ep, true);
  }

  template <class T> int cg_direction(cudaStream_t s)
  {
    const T *z = (const T *)(have_prec ? vec[Z] : vec[R]);
    ISPM_CUDA_TRY(launch_kernel(cg_direction_kernel<T>, dim3(grid_for(n_pad)), dim3(kThreads), 0,
                                s, true, z, (T *)vec[P], (long long)n_pad, st, sc,
                                have_prec ? 0 : 1, capturing_loop ? loop : 0ULL,
                                capturing_loop ? 1 : 0));
    return launched("cg direction");
  }

  template <class T> int cg_iteration(cudaStream_t s)
  {
    const int *skip = &st->done;
    SpmvDot ep = dot_into(vec[P], &st->pq);
    if (int e = Ain.apply(inner, vec[P], vec[Q], s, skip, &ep, true))
      return e;
    ISPM_CUDA_TRY(launch_kernel(cg_update_kernel<T>, dim3(grid_for(n_pad)), dim3(kThreads), 0,
                                s, true, (const T *)vec[P], (const T *)vec[Q], (T *)vec[R],
                                (T *)vec[D], (long long)n_pad, st, sc, have_prec ? 0 : 1));
    if (int e = launched("cg update"))
      return e;
    if (int e = cg_precondition<T>(s, skip))
      return e;
    return cg_direction<T>(s);
  }

  // Classic-CG phase start: r from r64, then z = M r and the new direction
  // (a fresh one on a restart, p = z + beta p after a reliable update).
  template <class T>
  int cg_resync(cudaStream_t s, bool restart, double thresh2, double ru2, int max_it)
  {
    cg_load_kernel<T><<<grid_for(n_pad), kThreads, 0, s>>>(
        r64, (T *)vec[R], (T *)vec[D], n, n_pad, st, sc, thresh2, ru2, max_it, restart,
        have_prec ? 0 : 1);
    if (int e = launched("cg load"))
      return e;
    const int *skip = &st->done;
    if (int e = cg_precondition<T>(s, skip))
      return e;
    return cg_direction<T>(s);
  }

  // The chunk of check_every iterations as a graph; with use_graph 2 (classic
  // iteration) the chunk is the body of a while node that repeats until the
  // direction kernel clears the condition, so a phase is one graph launch
  // and one host wait instead of one per chunk.
  int build_graph(cudaStream_t s)
  {
    if (graph)
      return ISPM_OK;
    cudaGraph_t g;
    cudaError_t e;
    int err = ISPM_OK;
    if (opts.use_graph == 2 && classic) {
      ISPM_CUDA_TRY(cudaGraphCreate(&g, 0));
      e = cudaGraphConditionalHandleCreate(&loop, g, 1u, cudaGraphCondAssignDefault);
      cudaGraphNodeParams np = {};
      np.type = cudaGraphNodeTypeConditional;
      np.conditional.handle = loop;
      np.conditional.type = cudaGraphCondTypeWhile;
      np.conditional.size = 1;
      cudaGraphNode_t node;
      if (e == cudaSuccess)
        e = cudaGraphAddNode(&node, g, nullptr, 0, &np);
      if (e == cudaSuccess)
        e = cudaStreamBeginCaptureToGraph(s, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return fail(ISPM_ERR_CUDA, "graph loop node: %s", cudaGetErrorString(e));
      }
      capturing_loop = true;
      for (int k = 0; k < opts.check_every && !err; k++)
        err = iteration(s);
      capturing_loop = false;
      cudaGraph_t body;
      e = cudaStreamEndCapture(s, &body);
      if (err || e != cudaSuccess)
        cudaGraphDestroy(g);
    } else {
      ISPM_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      for (int k = 0; k < opts.check_every && !err; k++)
        err = iteration(s);
      e = cudaStreamEndCapture(s, &g);
    }
    if (err)
      return err;
    if (e != cudaSuccess)
      return fail(ISPM_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess)
      return fail(ISPM_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    return ISPM_OK;
  }

  // r64 = b - A x64 and its norm (host copy of the state afterwards).
  int true_residual(cudaStream_t s)
  {
    if (int e = A64.apply(ISPM_F64, x64, t64, s, nullptr))
      return e;
    true_residual_kernel<<<grid_for(n), kThreads, 0, s>>>(b64, t64, r64, n, st, sc);
    if (int e = launched("true residual"))
      return e;
    ISPM_CUDA_TRY(cudaMemcpyAsync(st_host, st, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
    ISPM_CUDA_TRY(cudaStreamSynchronize(s));
    return ISPM_OK;
  }

  // Load r from r64 and re-derive the pipelined auxiliaries.  restart: also
  // reset the search directions (first start, or after a breakdown).
  template <class T>
  int resync(cudaStream_t s, bool restart, double thresh2, double ru2, int max_it)
  {
    load_residual_kernel<T><<<grid_for(n_pad), kThreads, 0, s>>>(
        r64, (T *)vec[R], (T *)vec[D], (T *)vec[P], (T *)vec[S], (T *)vec[Q], (T *)vec[Z], n,
        n_pad, restart);
    if (int e = launched("load residual"))
      return e;
    if (int e = prec(vec[R], vec[U], s, nullptr))  // u = M r
      return e;
    if (int e = Ain.apply(inner, vec[U], vec[W], s, nullptr))  // w = A u
      return e;
    if (!restart) {
      if (int e = Ain.apply(inner, vec[P], vec[S], s, nullptr))  // s = A p
        return e;
      if (int e = prec(vec[S], vec[Q], s, nullptr))  // q = M s
        return e;
      if (int e = Ain.apply(inner, vec[Q], vec[Z], s, nullptr))  // z = A q
        return e;
    }
    sync_dots_kernel<T><<<grid_for(n_pad), kThreads, 0, s>>>(
        (const T *)vec[R], (const T *)vec[U], (const T *)vec[W], n_pad, st, sc, thresh2, ru2,
        max_it, restart);
    return launched("sync dots");
  }

  int fold(cudaStream_t s)
  {
    if (inner == ISPM_F32)
      fold_correction_kernel<float><<<grid_for(n), kThreads, 0, s>>>(x64, (float *)vec[D], n);
    else
      fold_correction_kernel<double><<<grid_for(n), kThreads, 0, s>>>(x64, (double *)vec[D], n);
    return launched("fold correction");
  }

  int solve(const double *b, double *x, ispm_solve_stats *stats, cudaStream_t s)
  {
    auto t0 = std::chrono::steady_clock::now();
    history.clear();
    replacements = restarts = 0;
    b64 = const_cast<double *>(b);
    x64 = x;
    ISPM_CUDA_TRY(cudaMemsetAsync(x64, 0, (size_t)n_pad * sizeof(double), s));
    if (int e = true_residual(s))  // r64 = b
      return e;
    const double bnorm = std::sqrt(st_host->res2);
    if (!std::isfinite(bnorm)) {
      // a NaN or infinite right-hand side: no iterate can meet a relative
      // target; stop before iterating (x stays zero)
      ispm_solve_stats out{};
      out.true_relres = bnorm;
      out.converged = 0;
      out.status = ISPM_ERR_INVALID;
      out.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      if (stats)
        *stats = out;
      return fail(ISPM_ERR_INVALID, "the right-hand side holds a NaN or infinite value");
    }
    double rel = bnorm > 0 ? 1.0 : 0.0;
    int total_it = 0, status = ISPM_OK;
    const double target = opts.tol * bnorm;
    // the recursive residual must get a little below the target so that the
    // true residual (which it tracks to within the drift) meets it
    const double thresh2 = 0.25 * target * target;
    double ru = inner == ISPM_F32 ? opts.replace_ratio_f32 : opts.replace_ratio_f64;
    // an FP16-stored inner matrix drifts further from A between reliable
    // updates: keep them at most a 33x fall apart
    if (Ain.diag)
      ru = std::max(ru, kSplitReplaceRatio);
    const double ru2 = ru * ru;
    bool restart = true;
    int since_restart = 0;
    while (rel > opts.tol) {
      if (replacements + restarts >= opts.max_refinements || total_it >= opts.max_iters) {
        status = ISPM_ERR_NOT_CONVERGED;
        break;
      }
      const int budget = opts.max_iters - total_it + (restart ? 0 : since_restart);
      int e;
      if (classic)
        e = inner == ISPM_F32 ? cg_resync<float>(s, restart, thresh2, ru2, budget)
                              : cg_resync<double>(s, restart, thresh2, ru2, budget);
      else
        e = inner == ISPM_F32 ? resync<float>(s, restart, thresh2, ru2, budget)
                              : resync<double>(s, restart, thresh2, ru2, budget);
      if (e)
        return e;
      if (restart)
        since_restart = 0;
      int done = kRunning;
      for (;;) {
        ISPM_CUDA_TRY(cudaMemcpyAsync(st_host, st, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
        ISPM_CUDA_TRY(cudaStreamSynchronize(s));
        if (st_host->done) {
          done = st_host->done;
          break;
        }
        if (opts.use_graph) {
          if (int e2 = build_graph(s))
            return e2;
          ISPM_CUDA_TRY(cudaGraphLaunch(graph, s));
        } else {
          for (int k = 0; k < opts.check_every; k++)
            if (int e3 = iteration(s))
              return e3;
        }
      }
      total_it += st_host->it - since_restart;
      since_restart = st_host->it;
      NvtxRange update_range("ispm reliable update");
      if (int e4 = fold(s))
        return e4;
      if (int e5 = true_residual(s))
        return e5;
      const double new_rel = std::sqrt(st_host->res2) / bnorm;
      history.push_back(new_rel);
      if (verbose)
        fprintf(stderr,
                "[ispm solver] %s phase end: done=%d it=%d total=%d recursive=%.3e "
                "true=%.3e\n",
                inner == ISPM_F32 ? "f32" : "f64", done, st_host->it, total_it,
                std::sqrt(std::max(0.0, st_host->rr)) / bnorm, new_rel);
      if (done == kBreakdown) {
        restarts++;
        restart = true;
        if (!(new_rel < rel) && restarts > 2) {
          rel = new_rel;
          status = ISPM_ERR_BREAKDOWN;
          break;
        }
      } else if (done == kCap) {
        rel = new_rel;
        status = ISPM_ERR_NOT_CONVERGED;
        break;
      } else {
        replacements++;
        restart = false;
      }
      rel = new_rel;
    }
    ispm_solve_stats out{};
    out.iterations = total_it;
    out.refinements = replacements + restarts;
    out.true_relres = rel;
    out.converged = rel <= opts.tol;
    out.status = status;
    out.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (stats)
      *stats = out;
    if (status != ISPM_OK)
      return fail(status, "solve stopped at relative residual %.3e after %d iterations", rel,
                  total_it);
    return ISPM_OK;
  }

  int solve_on(const double *b, double *x, ispm_solve_stats *stats, cudaStream_t user)
  {
    NvtxRange range("ispm solve");
    ISPM_CUDA_TRY(cudaEventRecord(ev_in, user));
    ISPM_CUDA_TRY(cudaStreamWaitEvent(own, ev_in, 0));
    int e;
    if (perm) {
      // solve P A P^T (P x) = P b in the solver's order, then x = P^T (P x)
      permute_in_kernel<<<grid_for(n), kThreads, 0, own>>>(b_perm, b, perm, n);
      e = launched("permute b");
      if (!e)
        e = solve(b_perm, x_perm, stats, own);
      // x in the caller's order whenever solve() ran (a refused non-finite b
      // leaves the zero iterate)
      if (!e || e == ISPM_ERR_NOT_CONVERGED || e == ISPM_ERR_BREAKDOWN ||
          e == ISPM_ERR_INVALID) {
        cudaError_t me = cudaMemsetAsync(x, 0, (size_t)n_pad * sizeof(double), own);
        if (me == cudaSuccess)
          permute_out_kernel<<<grid_for(n), kThreads, 0, own>>>(x, x_perm, perm, n);
        const int e2 = me == cudaSuccess ? launched("permute x")
                                         : fail(ISPM_ERR_CUDA, "memset: %s",
                                                cudaGetErrorString(me));
        if (e2)
          e = e2;
      }
    } else {
      e = solve(b, x, stats, own);
    }
    cudaError_t ce = cudaEventRecord(ev_out, own);
    if (ce == cudaSuccess)
      ce = cudaStreamWaitEvent(user, ev_out, 0);
    if (e)
      return e;
    if (ce != cudaSuccess)
      return fail(ISPM_ERR_CUDA, "stream join: %s", cudaGetErrorString(ce));
    return ISPM_OK;
  }
};

}  // namespace ispm

struct ispm_solver {
  ispm::Solver s;
};

namespace ispm {
namespace {

__global__ void scatter_kernel(double *__restrict__ out, const unsigned *__restrict__ at,
                               const double *__restrict__ in, long long n)
{
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x)
    out[at[k]] = in[k];
}

template <class T> int to_device(DevMem &mem, T **d, const T *h, size_t count)
{
  if (int e = mem.get(d, count))
    return e;
  if (count)
    ISPM_CUDA_TRY(cudaMemcpy(*d, h, count * sizeof(T), cudaMemcpyHostToDevice));
  return ISPM_OK;
}

// FSAI values of G from A's device values a_v (solver order, the pattern of
// f.a_rp / f.a_ci), G^T's by the scatter, both written into the device
// factor matrices through their CSR-entry -> slot maps (legacy stream).
int fsai_values(Solver &S, const Solver::FsaiArrays &f, const double *a_v)
{
  if (int e = fsai_build_values(S.n, f.a_rp, f.a_ci, a_v, f.g_rp, f.g_v, f.fb, 0))
    return e;
  const int blocks = grid_for(f.nnz_g);
  scatter_kernel<<<blocks, kThreads>>>(f.gt_v, f.t_of, f.g_v, f.nnz_g);
  ISPM_CUDA_TRY(cudaPeekAtLastError());
  if (f.f16) {
    // one power-of-two scale for both factors: the largest magnitude lands
    // in [2^13, 2^14), below the binary16 maximum (65504)
    double amax = 0.0;
    if (int e = device_absmax(f.g_v, f.nnz_g, amax))
      return e;
    int ex = 0;
    if (amax > 0.0)
      std::frexp(amax, &ex);
    const double sc = std::ldexp(1.0, amax > 0.0 ? 14 - ex : 0);
    if (!(sc > 0.0) || !std::isfinite(sc) || sc > 0x1p126 || sc < 0x1p-126)
      return fail(ISPM_ERR_INVALID, "FP16 factor: magnitudes out of the FP32 scale range");
    if (int e = refresh_values_f16(S.G.dev, f.pos_g, f.g_v, f.nnz_g, sc, 0))
      return e;
    if (int e = refresh_values_f16(S.Ht.dev, f.pos_t, f.gt_v, f.nnz_g, sc, 0))
      return e;
    S.G.inv_scale = S.Ht.inv_scale = (float)(1.0 / sc);
  } else {
    if (int e = refresh_values(S.G.dev, f.pos_g, f.g_v, ISPM_F64, f.nnz_g, 0))
      return e;
    if (int e = refresh_values(S.Ht.dev, f.pos_t, f.gt_v, ISPM_F64, f.nnz_g, 0))
      return e;
  }
  ISPM_CUDA_TRY(cudaMemcpy(&S.fsai_fallbacks, f.fb, sizeof(unsigned), cudaMemcpyDeviceToHost));
  return ISPM_OK;
}

// The preconditioner pair from a GPU FSAI build: G on A's lower pattern and
// its transpose, each stored in its own sliced-ELL shape; the values are
// computed on the device and scattered into the device matrices through the
// CSR-entry -> slot maps, so no factor value crosses the host.  With
// S.refreshable the device arrays stay (S.mem, S.fsai) for value updates.
int build_fsai_on_device(Solver &S, int n, const int *rp, const int *ci, const double *v)
{
  std::vector<int> g_rp, g_ci, t_rp, t_ci;
  std::vector<unsigned> t_of, pos_g, pos_t;
  if (int e = fsai_lower_pattern(n, rp, ci, g_rp, g_ci))
    return e;
  fsai_transpose_pattern(n, g_rp, g_ci, t_rp, t_ci, t_of);
  const size_t nnz_a = (size_t)rp[n], nnz_g = g_ci.size();
  std::vector<double> zeros(nnz_g, 0.0);  // structure only; values come from the GPU
  const bool f16 = S.inner == ISPM_F32 && S.opts.factor_f16;
  const bool bf16 = S.inner == ISPM_F32 && S.opts.factor_bf16 && !f16;
  if (int e = S.G.upload(S.inner, S.inner, n, g_rp.data(), g_ci.data(), zeros.data(), nullptr,
                         &pos_g, false, bf16, f16))
    return e;
  if (int e = S.Ht.upload(S.inner, S.inner, n, t_rp.data(), t_ci.data(), zeros.data(), nullptr,
                          &pos_t, false, bf16, f16))
    return e;
  if (f16) {
    // FP16 factor values in diagonal blocks with at least eight stored
    // entries a row: eight rows a thread (one 16-byte element load per
    // step).  On the 128^3 27-point GRF system (14 a row) G and G^T took
    // 24.6 against 25.8 us and the solve 57.5 against 58.3 ms, same results
    // bit for bit; on the 192^3 unstructured system (4 a row) the solve took
    // 19.5 against 18.3 ms, so short rows keep four
    for (Operator *o : {&S.G, &S.Ht}) {
      const ispm_slell_view m = o->dev.view();
      const unsigned long long rows = (unsigned long long)m.n_slices * m.slice_height;
      if (m.diags && m.hblock == 1 && !m.var_height && m.slice_height >= 32 &&
          (unsigned long long)m.n_elms >= 8ull * rows) {
        o->lp.H = 8;
        o->lp.N = m.slice_height / 8;
      }
    }
  }
  DevMem tmp;
  DevMem &mem = S.refreshable ? S.mem : tmp;
  Solver::FsaiArrays f;
  f.nnz_g = (long long)nnz_g;
  f.f16 = f16;
  double *a_v_d;
  if (int e = to_device(mem, &f.a_rp, rp, (size_t)n + 1))
    return e;
  if (int e = to_device(mem, &f.a_ci, ci, nnz_a))
    return e;
  if (S.refreshable && S.a_v) {
    a_v_d = S.a_v;  // the solver-order values already on the device
    ISPM_CUDA_TRY(cudaMemcpy(a_v_d, v, nnz_a * sizeof(double), cudaMemcpyHostToDevice));
  } else if (int e = to_device(mem, &a_v_d, v, nnz_a)) {
    return e;
  }
  if (int e = to_device(mem, &f.g_rp, g_rp.data(), g_rp.size()))
    return e;
  if (int e = to_device(mem, &f.t_of, t_of.data(), nnz_g))
    return e;
  if (int e = to_device(mem, &f.pos_g, pos_g.data(), nnz_g))
    return e;
  if (int e = to_device(mem, &f.pos_t, pos_t.data(), nnz_g))
    return e;
  if (int e = mem.get(&f.g_v, nnz_g))
    return e;
  if (int e = mem.get(&f.gt_v, nnz_g))
    return e;
  if (int e = mem.get(&f.fb, 1))
    return e;
  if (int e = fsai_values(S, f, a_v_d))
    return e;
  if (S.refreshable) {
    S.fsai = f;
    S.fsai_kept = true;
  }
  return ISPM_OK;
}

__global__ void gather_values_kernel(double *__restrict__ out, const double *__restrict__ in,
                                     const int *__restrict__ src, long long n)
{
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x)
    out[k] = in[src[k]];
}

// ispm_solver_update_values: new values of A in the caller's CSR order.
int update_values(Solver &S, const double *vals, bool on_device)
{
  NvtxRange range("ispm solver update values");
  const long long nnz = S.nnz_a;
  const double *src = vals;
  if (!on_device) {
    double *dst = S.entry_src ? S.a_raw : S.a_v;
    if (nnz)
      ISPM_CUDA_TRY(cudaMemcpy(dst, vals, (size_t)nnz * sizeof(double), cudaMemcpyHostToDevice));
    src = dst;
  }
  // the solver's order (renumbered solves)
  const double *a_v = src;
  if (S.entry_src) {
    gather_values_kernel<<<grid_for(nnz), kThreads>>>(S.a_v, src, S.entry_src, nnz);
    ISPM_CUDA_TRY(cudaPeekAtLastError());
    a_v = S.a_v;
  }
  if (int e = refresh_values(S.A64.dev, S.pos_a64, a_v, ISPM_F64, nnz, 0))
    return e;
  if (int e = refresh_values(S.Ain.dev, S.pos_ain, a_v, ISPM_F64, nnz, 0))
    return e;
  if (S.fsai_kept)
    if (int e = fsai_values(S, S.fsai, a_v))
      return e;
  ISPM_CUDA_TRY(cudaStreamSynchronize(0));
  // the iteration graph holds launch arguments by value (an FP16 factor's
  // scale among them): capture it again at the next solve
  if (S.graph) {
    cudaGraphExecDestroy(S.graph);
    S.graph = nullptr;
  }
  return ISPM_OK;
}

}  // namespace
}  // namespace ispm

using namespace ispm;

extern "C" {

void ispm_solver_default_opts(ispm_solver_opts *o)
{
  if (!o)
    return;
  o->inner_dtype = ISPM_F32;
  o->tol = 1e-10;
  o->max_iters = 100000;
  o->max_refinements = 500;
  o->check_every = 16;
  o->use_graph = 1;
  o->replace_ratio_f32 = 1e-2;
  o->replace_ratio_f64 = 1e-4;
  o->variant = ISPM_PCG_AUTO;
  o->prec = ISPM_PREC_GIVEN;
  o->factor_bf16 = 0;
  o->reorder = ISPM_REORDER_AUTO;
  o->matrix_f16 = 0;
  o->factor_f16 = 1;
  o->refresh = 0;
}

int ispm_solver_create(int n, const int *row_ptr, const int *cols, const double *vals,
                       const int *g1_rp, const int *g1_ci, const double *g1_v,
                       const int *g2_rp, const int *g2_ci, const double *g2_v,
                       const ispm_solver_opts *opts, ispm_solver **out)
{
  clear_error();
  NvtxRange range("ispm solver create");
  if (!out || n <= 0 || !row_ptr || !cols || !vals)
    return fail(ISPM_ERR_INVALID, "bad arguments");
  *out = nullptr;
  // the reordering and the conversions index with these arrays: reject a
  // malformed CSR before anything walks it
  if (int e = validate_csr(n, n, row_ptr, cols))
    return e;
  if ((g1_rp && !g1_ci) || (g2_rp && !g2_ci))
    return fail(ISPM_ERR_INVALID, "factor row pointers without column indices");
  if (g1_rp)
    if (int e = validate_csr(n, n, g1_rp, g1_ci))
      return e;
  if (g2_rp)
    if (int e = validate_csr(n, n, g2_rp, g2_ci))
      return e;
  std::unique_ptr<ispm_solver> h(new (std::nothrow) ispm_solver);
  if (!h)
    return fail(ISPM_ERR_NOMEM, "host allocation");
  Solver &S = h->s;
  if (opts)
    S.opts = *opts;
  else
    ispm_solver_default_opts(&S.opts);
  if (S.opts.inner_dtype != ISPM_F32 && S.opts.inner_dtype != ISPM_F64)
    return fail(ISPM_ERR_INVALID, "inner_dtype %d", S.opts.inner_dtype);
  if (S.opts.check_every < 1 || S.opts.check_every > 4096)
    return fail(ISPM_ERR_INVALID, "check_every %d", S.opts.check_every);
  if (!(S.opts.replace_ratio_f32 > 0 && S.opts.replace_ratio_f32 < 1) ||
      !(S.opts.replace_ratio_f64 > 0 && S.opts.replace_ratio_f64 < 1))
    return fail(ISPM_ERR_INVALID, "replacement ratios must lie in (0, 1)");
  S.inner = S.opts.inner_dtype;
  if (S.opts.variant == ISPM_PCG_AUTO)
    S.classic = S.inner == ISPM_F32;
  else if (S.opts.variant == ISPM_PCG_CLASSIC || S.opts.variant == ISPM_PCG_PIPELINED)
    S.classic = S.opts.variant == ISPM_PCG_CLASSIC;
  else
    return fail(ISPM_ERR_INVALID, "variant %d", S.opts.variant);
  S.n = n;
  if (S.opts.prec != ISPM_PREC_GIVEN && S.opts.prec != ISPM_PREC_FSAI_GPU)
    return fail(ISPM_ERR_INVALID, "prec %d", S.opts.prec);
  S.have_prec = S.opts.prec == ISPM_PREC_FSAI_GPU || (g1_rp && g2_rp);
  if (S.opts.reorder != ISPM_REORDER_NONE && S.opts.reorder != ISPM_REORDER_RCM &&
      S.opts.reorder != ISPM_REORDER_AUTO)
    return fail(ISPM_ERR_INVALID, "reorder %d", S.opts.reorder);
  const bool given_pair = S.opts.prec == ISPM_PREC_GIVEN && g1_rp && g2_rp;
  if (S.opts.reorder == ISPM_REORDER_RCM && given_pair)
    return fail(ISPM_ERR_INVALID, "reordering needs prec = ISPM_PREC_FSAI_GPU or none (a given "
                                  "factor pair is in the caller's order)");
  if (S.opts.refresh && S.inner == ISPM_F32 && S.opts.matrix_f16)
    return fail(ISPM_ERR_INVALID, "refresh is not available with matrix_f16");
  S.refreshable = S.opts.refresh != 0;
  S.nnz_a = row_ptr[n];
  std::vector<int> perm, inv, prp, pci;
  std::vector<double> pv;
  std::vector<int> entry_src;  // refresh + renumbering: solver entry -> caller entry
  try {
    // automatic mode skips matrices whose band is already under n / 16 (a
    // mesh in its natural order) without computing an ordering
    const bool try_rcm = S.opts.reorder == ISPM_REORDER_RCM ||
                         (S.opts.reorder == ISPM_REORDER_AUTO && !given_pair &&
                          16 * bandwidth(n, row_ptr, cols, nullptr) >= (long long)n);
    if (try_rcm) {
      rcm_order(n, row_ptr, cols, perm);
      inv.assign(n, 0);
      for (int i = 0; i < n; i++)
        inv[perm[i]] = i;
      const long long bw0 = bandwidth(n, row_ptr, cols, nullptr);
      const long long bw1 = bandwidth(n, row_ptr, cols, inv.data());
      // automatic: reorder only a matrix whose numbering is far from banded
      if (S.opts.reorder == ISPM_REORDER_RCM || 4 * bw1 <= bw0) {
        if (S.refreshable) {
          // the same permutation applied to the entry indices (exact in FP64)
          std::vector<double> idx((size_t)S.nnz_a), pidx;
          std::vector<int> rp2, ci2;
          for (long long k = 0; k < S.nnz_a; k++)
            idx[(size_t)k] = (double)k;
          permute_csr(n, row_ptr, cols, idx.data(), perm, inv, rp2, ci2, pidx);
          entry_src.resize(pidx.size());
          for (size_t k = 0; k < pidx.size(); k++)
            entry_src[k] = (int)pidx[k];
        }
        permute_csr(n, row_ptr, cols, vals, perm, inv, prp, pci, pv);
        row_ptr = prp.data();
        cols = pci.data();
        vals = pv.data();
      } else {
        perm.clear();
      }
    }
  } catch (const std::bad_alloc &) {
    return fail(ISPM_ERR_NOMEM, "host allocation while reordering");
  }
  try {
    std::vector<unsigned> pos_ain, pos_a64;
    std::vector<unsigned> *want_ain = S.refreshable ? &pos_ain : nullptr;
    std::vector<unsigned> *want_a64 = S.refreshable ? &pos_a64 : nullptr;
    if (S.inner == ISPM_F32 && S.opts.matrix_f16) {
      if (int e = S.Ain.upload_split_f16(n, row_ptr, cols, vals))
        return e;
    } else if (int e = S.Ain.upload(S.inner, S.inner, n, row_ptr, cols, vals, nullptr,
                                    want_ain)) {
      return e;
    }
    // the FP64 operator of the reliable updates takes the inner matrix's
    // shape, unless the inner matrix is an FP16 split (its shape was chosen
    // for the off-diagonal part alone): then A64 gets its own min-bytes shape
    const bool split = S.inner == ISPM_F32 && S.opts.matrix_f16;
    if (int e = S.A64.upload(ISPM_F64, ISPM_F64, n, row_ptr, cols, vals,
                             split ? nullptr : &S.Ain.fmt, want_a64))
      return e;
    if (S.refreshable) {
      const size_t nnz = (size_t)S.nnz_a;
      if (int e = to_device(S.mem, &S.pos_ain, pos_ain.data(), nnz))
        return e;
      if (int e = to_device(S.mem, &S.pos_a64, pos_a64.data(), nnz))
        return e;
      if (int e = S.mem.get(&S.a_v, nnz))
        return e;
      if (!entry_src.empty()) {
        if (int e = to_device(S.mem, &S.entry_src, entry_src.data(), nnz))
          return e;
        if (int e = S.mem.get(&S.a_raw, nnz))
          return e;
      }
    }
    if (S.opts.prec == ISPM_PREC_FSAI_GPU) {
      if (int e = build_fsai_on_device(S, n, row_ptr, cols, vals))
        return e;
    } else if (S.have_prec && is_lower(n, g1_rp, g1_ci)) {
      // already banded (an FSAI pair G, G^T): store as given
      const bool bf16 = S.inner == ISPM_F32 && S.opts.factor_bf16;
      if (int e = S.G.upload(S.inner, S.inner, n, g1_rp, g1_ci, g1_v, nullptr, nullptr, false,
                             bf16))
        return e;
      if (int e = S.Ht.upload(S.inner, S.inner, n, g2_rp, g2_ci, g2_v, nullptr, nullptr, false,
                              bf16))
        return e;
    } else if (S.have_prec) {
      std::vector<int> rp, ci;
      std::vector<double> v;
      const bool bf16 = S.inner == ISPM_F32 && S.opts.factor_bf16;
      reverse_rows(n, g1_rp, g1_ci, g1_v, rp, ci, v);
      if (int e = S.G.upload(S.inner, S.inner, n, rp.data(), ci.data(), v.data(), nullptr,
                             nullptr, false, bf16))
        return e;
      reverse_cols(n, g2_rp, g2_ci, g2_v, rp, ci, v);
      if (int e = S.Ht.upload(S.inner, S.inner, n, rp.data(), ci.data(), v.data(), nullptr,
                              nullptr, false, bf16))
        return e;
    }
  } catch (const std::bad_alloc &) {
    return fail(ISPM_ERR_NOMEM, "host allocation while building the solver");
  }
  S.n_pad = S.A64.dev.meta.n_rows;
  if (int e = S.init_stream())
    return e;
  const size_t npad = (size_t)S.n_pad + 64;
  if (int e = S.mem.get(&S.st, 1))
    return e;
  if (cudaMallocHost(&S.st_host, sizeof(PcgState)) != cudaSuccess)
    return fail(ISPM_ERR_NOMEM, "pinned host allocation");
  // partial slots: the fixed-grid kernels use 4 * kMaxBlocks, a fused SpMV
  // dot one per CTA of that SpMV
  S.part_capacity = std::max<unsigned>(
      {4u * kMaxBlocks, S.Ain.grid(), S.have_prec ? S.Ht.grid() : 0u});
  // two sums' partials for the fused r.z / r.r epilogue
  if (int e = S.mem.get(&S.sc.part, 2 * (size_t)S.part_capacity))
    return e;
  if (int e = S.mem.get(&S.sc.ticket, 4))
    return e;
  double **d64[] = {&S.r64, &S.t64, &S.b_stage, &S.x_stage};
  for (double **pp : d64)
    if (int e = S.mem.get(pp, npad))
      return e;
  if (!perm.empty()) {
    if (int e = S.mem.get(&S.perm, (size_t)n))
      return e;
    ISPM_CUDA_TRY(cudaMemcpy(S.perm, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    if (int e = S.mem.get(&S.b_perm, npad))
      return e;
    if (int e = S.mem.get(&S.x_perm, npad))
      return e;
  }
  for (int k = 0; k < 11; k++) {
    int e = S.inner == ISPM_F32 ? S.mem.get((float **)&S.vec[k], npad)
                                : S.mem.get((double **)&S.vec[k], npad);
    if (e)
      return e;
  }
  *out = h.release();
  return ISPM_OK;
}

int ispm_solver_rows(const ispm_solver *s) { return s ? s->s.n_pad : 0; }

int ispm_solver_solve(ispm_solver *s, const double *b, double *x, ispm_solve_stats *stats,
                      void *stream)
{
  clear_error();
  if (!s || !b || !x)
    return fail(ISPM_ERR_INVALID, "NULL argument");
  return s->s.solve_on(b, x, stats, (cudaStream_t)stream);
}

int ispm_solver_solve_host(ispm_solver *s, const double *b_host, double *x_host,
                           ispm_solve_stats *stats, void *stream)
{
  clear_error();
  if (!s || !b_host || !x_host)
    return fail(ISPM_ERR_INVALID, "NULL argument");
  Solver &S = s->s;
  cudaStream_t st = (cudaStream_t)stream;
  ISPM_CUDA_TRY(cudaMemcpyAsync(S.b_stage, b_host, (size_t)S.n * 8, cudaMemcpyHostToDevice, st));
  int e = S.solve_on(S.b_stage, S.x_stage, stats, st);
  cudaError_t ce = cudaMemcpyAsync(x_host, S.x_stage, (size_t)S.n * 8, cudaMemcpyDeviceToHost, st);
  if (ce == cudaSuccess)
    ce = cudaStreamSynchronize(st);
  if (e)
    return e;
  if (ce != cudaSuccess)
    return fail(ISPM_ERR_CUDA, "D2H: %s", cudaGetErrorString(ce));
  return ISPM_OK;
}

int ispm_solver_history(const ispm_solver *s, double *out, int cap)
{
  if (!s)
    return 0;
  int n = (int)s->s.history.size();
  for (int k = 0; k < n && k < cap; k++)
    out[k] = s->s.history[k];
  return n;
}

int ispm_solver_choose_shape(int elm_dtype, int n, const int *row_ptr, const int *cols,
                             const double *vals, ispm_slell_params *out)
{
  clear_error();
  if (!out || n <= 0 || !row_ptr || !vals || (elm_dtype != ISPM_F32 && elm_dtype != ISPM_F64))
    return fail(ISPM_ERR_INVALID, "bad arguments");
  if (int e = validate_csr(n, n, row_ptr, cols))
    return e;
  try {
    return choose_operator_shape(elm_dtype, n, row_ptr, cols, vals, *out);
  } catch (const std::bad_alloc &) {
    return fail(ISPM_ERR_NOMEM, "host allocation");
  }
}

int ispm_solver_operator(const ispm_solver *s, int which, ispm_slell_view *view,
                         ispm_launch_params *params)
{
  clear_error();
  if (!s || !view)
    return fail(ISPM_ERR_INVALID, "NULL argument");
  const Solver &S = s->s;
  const Operator *op = which == 0 ? &S.Ain : which == 1 ? &S.A64 : which == 2 ? &S.G
                     : which == 3 ? &S.Ht : nullptr;
  if (!op)
    return fail(ISPM_ERR_INVALID, "operator %d (0 inner A, 1 FP64 A, 2 G, 3 G^T)", which);
  if (which >= 2 && !S.have_prec)
    return fail(ISPM_ERR_INVALID, "the solver has no preconditioner");
  *view = op->dev.view();
  if (params)
    *params = op->lp;
  return ISPM_OK;
}

int ispm_solver_update_values(ispm_solver *s, const double *vals, int vals_on_device)
{
  clear_error();
  if (!s || (!vals && s->s.nnz_a))
    return fail(ISPM_ERR_INVALID, "NULL solver or values");
  if (!s->s.refreshable)
    return fail(ISPM_ERR_INVALID, "the solver was created without opts.refresh");
  return update_values(s->s, vals, vals_on_device != 0);
}

void ispm_solver_free(ispm_solver *s) { delete s; }

}  // extern "C"
