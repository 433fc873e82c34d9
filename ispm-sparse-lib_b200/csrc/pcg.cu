// Preconditioned pipelined CG on sliced-ELL operands, with FP64 iterative
// refinement.
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
//    chunk into no-ops once the recursive residual meets the target;
//  * reductions (gamma = r.u, delta = w.u, ||r||^2) accumulate in FP64 and
//    finish in the last CTA of the update launch;
//  * inner precision T is FP64 (plain) or FP32 (mixed: FP32 matrices and
//    vectors, FP64 reductions); an FP64 outer loop recomputes the true
//    residual b - A x with the FP64 matrix and restarts the inner solve on it
//    until ||b - A x||_2 <= tol ||b||_2;
//  * the FSAI pair is stored as G' = P Ainv1 (rows reversed) and H' = Ainv2 P
//    (columns reversed), P the index reversal: M = Ainv2 Ainv1 = H' G', and
//    both factors become banded with stencil-like diagonals that the
//    diagonal-block format captures (Ainv1 itself runs along anti-diagonals).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "cuda_util.cuh"
#include "sblas_impl.h"
#include "spmv_launch.h"

namespace ispm {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 1024;

// Device-resident solver scalars.
struct PcgState {
  double gamma, gammaold, delta, alpha, beta;
  double rr;       // ||r||^2 of the inner recursive residual
  double rr0;      // ||r||^2 when the inner solve started
  double thresh2;  // inner stop: rr <= thresh2
  double res2;     // ||b - A x||^2 of the last outer residual
  double rscale;   // norm the inner right-hand side was divided by
  int it;          // inner iterations so far
  int max_it;      // inner iteration cap
  int done;        // 0 running, 1 converged, 2 breakdown, 3 iteration cap
  int pad;
};

struct Scratch {
  double *part;     // 4 * kMaxBlocks partials
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

// r64 = b - Ax, res2 = ||r64||^2
__global__ void __launch_bounds__(kThreads)
    outer_residual_kernel(const double *__restrict__ b, const double *__restrict__ ax,
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

// Inner right-hand side r = r64 / ||r64|| in T; zero the inner iterate and
// the recurrence vectors.
template <class T>
__global__ void __launch_bounds__(kThreads)
    scale_rhs_kernel(const double *__restrict__ r64, T *r, T *d, T *p, T *s, T *q, T *z,
                     long long n, long long n_pad, PcgState *st)
{
  const double nrm = sqrt(st->res2);
  const double inv = nrm > 0 ? 1.0 / nrm : 0.0;
  GRID_STRIDE(i, n_pad)
  {
    r[i] = i < n ? (T)(r64[i] * inv) : T(0);
    d[i] = T(0);
    p[i] = T(0);
    s[i] = T(0);
    q[i] = T(0);
    z[i] = T(0);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0)
    st->rscale = nrm;
}

// gamma = r.u, delta = w.u, rr = r.r at the start of an inner solve.
template <class T>
__global__ void __launch_bounds__(kThreads)
    init_dots_kernel(const T *__restrict__ r, const T *__restrict__ u,
                     const T *__restrict__ w, long long n, PcgState *st, Scratch sc,
                     double rel_tol, int max_it)
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
    st->rr0 = tot.v[2];
    st->thresh2 = rel_tol * rel_tol * tot.v[2];
    st->gammaold = 0;
    st->alpha = 0;
    st->beta = 0;
    st->it = 0;
    st->max_it = max_it;
    st->done = tot.v[2] == 0.0 ? 1 : 0;
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
    // Lost positive definiteness in finite precision: stop, the outer loop
    // restarts from the true residual.
    if (blockIdx.x == 0 && threadIdx.x == 0)
      st->done = 2;
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
    if (!(tot.v[2] > st->thresh2))
      st->done = isfinite(tot.v[2]) ? 1 : 2;
    else if (st->it >= st->max_it)
      st->done = 3;
  }
}

// x += rscale * d
template <class T>
__global__ void __launch_bounds__(kThreads)
    apply_correction_kernel(double *__restrict__ x, const T *__restrict__ d, long long n,
                            const PcgState *st)
{
  const double sc = st->rscale;
  GRID_STRIDE(i, n) x[i] = fma(sc, (double)d[i], x[i]);
}

int grid_for(long long n)
{
  long long blocks = (n + kThreads - 1) / kThreads;
  long long cap = std::min<long long>(kMaxBlocks, (long long)device_sm_count() * 4);
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
    cudaError_t e = cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T) + 256);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(ISPM_ERR_NOMEM, "solver cudaMalloc(%zu): %s", count * sizeof(T),
                  cudaGetErrorString(e));
    }
    blocks.push_back(p);
    e = cudaMemset(p, 0, std::max<size_t>(count, 1) * sizeof(T) + 256);
    if (e != cudaSuccess)
      return fail(ISPM_ERR_CUDA, "cudaMemset: %s", cudaGetErrorString(e));
    *out = (T *)p;
    return ISPM_OK;
  }
};

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

struct Operator {
  HostSlell host;
  DeviceSlell dev;
  ispm_launch_params lp{};
  int upload(int vec_dtype, int elm_dtype, int n, const int *rp, const int *ci,
             const double *v)
  {
    ispm_slell_params f;
    std::vector<float> vf;
    const void *vals = v;
    if (elm_dtype == ISPM_F32) {
      vf.resize(rp[n]);
      for (int k = 0; k < rp[n]; k++)
        vf[k] = (float)v[k];
      vals = vf.data();
    }
    if (int st = guess_format(elm_dtype, n, n, rp, ci, vals, 1, 4, f))
      return st;
    if (int st = convert_csr(elm_dtype, n, n, rp, ci, vals, (int)f.S, (int)f.H, f.V != 0,
                             f.D != 0, 4, host))
      return st;
    if (int st = dev.upload(host))
      return st;
    lp = default_launch(vec_dtype, dev.view());
    // drop the host copy: the device matrix is all the solver needs
    HostSlell keep_meta;
    keep_meta.n_rows = host.n_rows;
    host = std::move(keep_meta);
    return ISPM_OK;
  }
  int apply(int vdt, const void *x, void *y, cudaStream_t s, const int *skip) const
  {
    return launch_spmv(vdt, lp, dev.view(), x, y, s, skip);
  }
};

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
  double *x64 = nullptr, *r64 = nullptr, *t64 = nullptr, *b64 = nullptr;
  void *vec[11] = {};  // r u w m n p s q z d t (inner type)
  cudaGraphExec_t graph = nullptr;
  cudaStream_t graph_stream = nullptr;
  std::vector<double> history;

  ~Solver()
  {
    if (graph)
      cudaGraphExecDestroy(graph);
    if (st_host)
      cudaFreeHost(st_host);
  }

  void *V(int k) const { return vec[k]; }
  enum { R, U, W, M, NV, P, S, Q, Z, D, TT };

  int prec_apply(const void *in, void *out, cudaStream_t s, const int *skip)
  {
    if (!have_prec)
      return ISPM_ERR_INVALID;
    if (int e = G.apply(inner, in, vec[TT], s, skip))
      return e;
    return Ht.apply(inner, vec[TT], out, s, skip);
  }

  template <class T> int launch_step(cudaStream_t s)
  {
    const int grid = grid_for(n_pad);
    pcg_step_kernel<T><<<grid, kThreads, 0, s>>>(
        (const T *)vec[NV], (const T *)vec[M], (T *)vec[P], (T *)vec[S], (T *)vec[Q],
        (T *)vec[Z], (T *)vec[D], (T *)vec[R], (T *)vec[U], (T *)vec[W], n_pad, st, sc);
    cudaError_t e = cudaPeekAtLastError();
    return e == cudaSuccess ? ISPM_OK : fail(ISPM_ERR_CUDA, "pcg step: %s", cudaGetErrorString(e));
  }

  // One inner iteration: m = M w, n = A m, fused update.
  int iteration(cudaStream_t s)
  {
    const int *skip = &st->done;
    if (have_prec) {
      if (int e = prec_apply(vec[W], vec[M], s, skip))
        return e;
    } else {
      ISPM_CUDA_TRY(cudaMemcpyAsync(vec[M], vec[W], (size_t)n_pad * esize(), cudaMemcpyDeviceToDevice, s));
    }
    if (int e = Ain.apply(inner, vec[M], vec[NV], s, skip))
      return e;
    return inner == ISPM_F32 ? launch_step<float>(s) : launch_step<double>(s);
  }

  size_t esize() const { return inner == ISPM_F32 ? 4 : 8; }

  int build_graph(cudaStream_t s)
  {
    if (graph && graph_stream == s)
      return ISPM_OK;
    if (graph) {
      cudaGraphExecDestroy(graph);
      graph = nullptr;
    }
    cudaGraph_t g;
    ISPM_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    int err = ISPM_OK;
    for (int k = 0; k < opts.check_every && !err; k++)
      err = iteration(s);
    cudaError_t e = cudaStreamEndCapture(s, &g);
    if (err)
      return err;
    if (e != cudaSuccess)
      return fail(ISPM_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess)
      return fail(ISPM_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    graph_stream = s;
    return ISPM_OK;
  }

  template <class T> int start_inner(cudaStream_t s, double rel_tol, int max_it)
  {
    const int grid = grid_for(n_pad);
    scale_rhs_kernel<T><<<grid, kThreads, 0, s>>>(r64, (T *)vec[R], (T *)vec[D], (T *)vec[P],
                                                  (T *)vec[S], (T *)vec[Q], (T *)vec[Z], n,
                                                  n_pad, st);
    // u = M r, w = A u
    if (have_prec) {
      if (int e = prec_apply(vec[R], vec[U], s, nullptr))
        return e;
    } else {
      ISPM_CUDA_TRY(cudaMemcpyAsync(vec[U], vec[R], (size_t)n_pad * sizeof(T), cudaMemcpyDeviceToDevice, s));
    }
    if (int e = Ain.apply(inner, vec[U], vec[W], s, nullptr))
      return e;
    init_dots_kernel<T><<<grid, kThreads, 0, s>>>((const T *)vec[R], (const T *)vec[U],
                                                  (const T *)vec[W], n_pad, st, sc, rel_tol,
                                                  max_it);
    cudaError_t e = cudaPeekAtLastError();
    return e == cudaSuccess ? ISPM_OK : fail(ISPM_ERR_CUDA, "inner start: %s", cudaGetErrorString(e));
  }

  int outer_residual(cudaStream_t s)
  {
    if (int e = A64.apply(ISPM_F64, x64, t64, s, nullptr))
      return e;
    outer_residual_kernel<<<grid_for(n), kThreads, 0, s>>>(b64, t64, r64, n, st, sc);
    ISPM_CUDA_TRY(cudaPeekAtLastError());
    ISPM_CUDA_TRY(cudaMemcpyAsync(st_host, st, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
    ISPM_CUDA_TRY(cudaStreamSynchronize(s));
    return ISPM_OK;
  }

  int solve(const double *b, double *x, ispm_solve_stats *stats, cudaStream_t s)
  {
    auto t0 = std::chrono::steady_clock::now();
    history.clear();
    b64 = const_cast<double *>(b);
    x64 = x;
    ispm_solve_stats out{};
    // ||b|| from the first outer residual with the caller's initial guess
    // replaced by zero
    ISPM_CUDA_TRY(cudaMemsetAsync(x64, 0, (size_t)n * sizeof(double), s));
    if (int e = outer_residual(s))
      return e;
    const double bnorm = std::sqrt(st_host->res2);
    double rel = 1.0;
    int total_it = 0, cycles = 0, status = ISPM_OK;
    if (bnorm == 0.0) {
      rel = 0.0;
    }
    const double eta_min = inner == ISPM_F32 ? opts.inner_tol_f32 : 0.0;
    while (rel > opts.tol) {
      if (cycles >= opts.max_refinements || total_it >= opts.max_iters) {
        status = ISPM_ERR_NOT_CONVERGED;
        break;
      }
      // inner target: the outer goal (with margin), never tighter than FP32 allows
      const double need = 0.5 * opts.tol / rel;
      const double eta = std::max(need, eta_min);
      const int budget = opts.max_iters - total_it;
      int e = inner == ISPM_F32 ? start_inner<float>(s, eta, budget)
                                : start_inner<double>(s, eta, budget);
      if (e)
        return e;
      if (opts.use_graph)
        if (int e2 = build_graph(s))
          return e2;
      for (;;) {
        if (opts.use_graph) {
          ISPM_CUDA_TRY(cudaGraphLaunch(graph, s));
        } else {
          for (int k = 0; k < opts.check_every; k++)
            if (int e3 = iteration(s))
              return e3;
        }
        ISPM_CUDA_TRY(cudaMemcpyAsync(st_host, st, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
        ISPM_CUDA_TRY(cudaStreamSynchronize(s));
        if (st_host->done)
          break;
      }
      total_it += st_host->it;
      cycles++;
      if (inner == ISPM_F32)
        apply_correction_kernel<float><<<grid_for(n), kThreads, 0, s>>>(x64, (const float *)vec[D], n, st);
      else
        apply_correction_kernel<double><<<grid_for(n), kThreads, 0, s>>>(x64, (const double *)vec[D], n, st);
      ISPM_CUDA_TRY(cudaPeekAtLastError());
      const int inner_done = st_host->done;
      if (int e4 = outer_residual(s))
        return e4;
      double new_rel = std::sqrt(st_host->res2) / bnorm;
      history.push_back(new_rel);
      if (inner_done == 2 && !(new_rel < rel)) {
        rel = new_rel;
        status = ISPM_ERR_BREAKDOWN;
        break;
      }
      rel = new_rel;
    }
    out.iterations = total_it;
    out.refinements = cycles;
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
};

}  // namespace ispm

struct ispm_solver {
  ispm::Solver s;
};

using namespace ispm;

extern "C" {

void ispm_solver_default_opts(ispm_solver_opts *o)
{
  if (!o)
    return;
  o->inner_dtype = ISPM_F32;
  o->tol = 1e-10;
  o->max_iters = 100000;
  o->max_refinements = 50;
  o->check_every = 16;
  o->inner_tol_f32 = 1e-5;
  o->use_graph = 1;
}

int ispm_solver_create(int n, const int *row_ptr, const int *cols, const double *vals,
                       const int *g1_rp, const int *g1_ci, const double *g1_v,
                       const int *g2_rp, const int *g2_ci, const double *g2_v,
                       const ispm_solver_opts *opts, ispm_solver **out)
{
  clear_error();
  if (!out || n <= 0 || !row_ptr || !cols || !vals)
    return fail(ISPM_ERR_INVALID, "bad arguments");
  *out = nullptr;
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
  S.inner = S.opts.inner_dtype;
  S.n = n;
  S.have_prec = g1_rp && g2_rp;
  try {
    if (int e = S.A64.upload(ISPM_F64, ISPM_F64, n, row_ptr, cols, vals))
      return e;
    if (int e = S.Ain.upload(S.inner, S.inner, n, row_ptr, cols, vals))
      return e;
    if (S.have_prec) {
      std::vector<int> rp, ci;
      std::vector<double> v;
      reverse_rows(n, g1_rp, g1_ci, g1_v, rp, ci, v);
      if (int e = S.G.upload(S.inner, S.inner, n, rp.data(), ci.data(), v.data()))
        return e;
      reverse_cols(n, g2_rp, g2_ci, g2_v, rp, ci, v);
      if (int e = S.Ht.upload(S.inner, S.inner, n, rp.data(), ci.data(), v.data()))
        return e;
    }
  } catch (const std::bad_alloc &) {
    return fail(ISPM_ERR_NOMEM, "host allocation while building the solver");
  }
  S.n_pad = S.A64.dev.meta.n_rows;
  const size_t npad = (size_t)S.n_pad + 64;
  if (int e = S.mem.get(&S.st, 1))
    return e;
  if (cudaMallocHost(&S.st_host, sizeof(PcgState)) != cudaSuccess)
    return fail(ISPM_ERR_NOMEM, "pinned host allocation");
  if (int e = S.mem.get(&S.sc.part, 4 * kMaxBlocks))
    return e;
  if (int e = S.mem.get(&S.sc.ticket, 4))
    return e;
  if (int e = S.mem.get(&S.r64, npad))
    return e;
  if (int e = S.mem.get(&S.t64, npad))
    return e;
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
  return s->s.solve(b, x, stats, (cudaStream_t)stream);
}

int ispm_solver_solve_host(ispm_solver *s, const double *b_host, double *x_host,
                           ispm_solve_stats *stats, void *stream)
{
  clear_error();
  if (!s || !b_host || !x_host)
    return fail(ISPM_ERR_INVALID, "NULL argument");
  Solver &S = s->s;
  cudaStream_t st = (cudaStream_t)stream;
  double *b = nullptr, *x = nullptr;
  if (int e = S.mem.get(&b, S.n_pad + 64))
    return e;
  if (int e = S.mem.get(&x, S.n_pad + 64))
    return e;
  ISPM_CUDA_TRY(cudaMemcpyAsync(b, b_host, (size_t)S.n * 8, cudaMemcpyHostToDevice, st));
  int e = S.solve(b, x, stats, st);
  cudaError_t ce = cudaMemcpyAsync(x_host, x, (size_t)S.n * 8, cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  // release the two staging vectors
  for (int k = 0; k < 2; k++) {
    cudaFree(S.mem.blocks.back());
    S.mem.blocks.pop_back();
  }
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

void ispm_solver_free(ispm_solver *s) { delete s; }

}  // extern "C"
