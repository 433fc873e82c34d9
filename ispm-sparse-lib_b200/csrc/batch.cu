// Batched preconditioned CG: many independent SPD systems of uneven size,
// each with one or more right-hand sides, advanced together by one set of
// kernels.
//
// The reference solves one system per call through its primitives
// (launch_spmv_kernel, sblas, fastainv_sym); a caller with several systems
// per time step (the U/V/W/p solves) runs them one after another, each
// iteration a handful of small launches.  Here every (system, right-hand
// side) pair is a lane, and all lanes share each launch:
//  * the lanes' matrices are stacked into block-diagonal operators, each
//    lane padded with identity rows to whole 1024-row tiles, so every CTA of
//    the SpMVs and vector kernels belongs to exactly one lane;
//  * systems are grouped by the sliced-ELL shape that suits them (chosen per
//    system, min stored bytes on a band of its rows), one stacked operator
//    per group, so 7-point and 27-point systems each get their own format;
//  * one iteration is the classic-PCG step of the single-system solver with
//    per-lane scalars:
//      q = A p                 (SpMV; lane sums of p.q)
//      alpha = rz / pq; d += alpha p; r -= alpha q   (lane sums of r.r)
//      z = G^T (G r)           (two SpMVs; lane sums of r.z)
//      beta = rz_new / rz; p = z + beta p            (lane stop test)
//    Lane sums are finished by the lane's last CTA to arrive (a per-lane
//    ticket), adding the lane's per-CTA partials in CTA order: deterministic,
//    no extra launch;
//  * CTAs of lanes that stopped return at once, so finished lanes cost
//    nothing while the others go on;
//  * iterations run as a CUDA graph of `check_every` steps (even, so the
//    double-buffered r.z slot is the same at every chunk start); the last
//    step of a chunk ends after the r / d update, and every unfinished lane
//    then takes an FP64 reliable update (fold the inner-precision correction
//    into the FP64 iterate, r = b - A x with the FP64 operator, z = M r, and
//    the direction step the chunk left out) -- lanes whose true residual
//    meets the tolerance finish instead;
//  * the FSAI factor of every group's stack is built on the GPU (fsai.cu).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "cuda_util.cuh"
#include "fsai.h"
#include "nvtx_range.h"
#include "operator.h"

namespace ispm {
namespace {

constexpr int kTile = 1024;    // rows per tile; lanes are padded to whole tiles
constexpr int kThreads = 256;  // vector kernels: one CTA per tile, 4 rows per thread
constexpr int kSampleRows = 8192;  // rows of a system the format choice looks at

enum LaneState { kRun = 0, kStopConv = 1, kBreak = 2, kCap = 3, kFinished = 4, kFailed = 5 };

// Device lane tables.  ib holds five int arrays of n_lanes entries back to
// back (state, skip, fin, fresh, it) so the host moves them in one copy.
struct LaneArgs {
  const int *tile_lane;   // lane of each tile
  const int *lane_tile0;  // first tile of each lane
  const int *lane_ntile;  // tiles of each lane
  int *state;             // LaneState
  int *skip;              // state != kRun: the in-iteration SpMVs skip the lane
  int *fin;               // finished or failed: the reliable-update SpMV skips it
  int *fresh;             // the next direction starts anew (beta = 0)
  int *it;                // iterations of each lane
  double *rz;             // [2][n_lanes] r.z of the current direction, by parity
  double *rz_cur;         // latest r.z of each lane
  double *rz_prev;        // rz_cur as the reliable update found it
  double *thresh2;        // recursive stop: ||r||^2 <= thresh2
  double *ru2ref;         // pause for a reliable update once ||r||^2 < ru2ref
  double *pq, *rzn, *rr, *res;  // lane sums
  unsigned *t_rr, *t_res;       // tickets of the vector kernels' lane sums
  double *part_rr, *part_res;   // per-tile partials of those sums
  int max_it;
  int n_lanes;
};

template <class T> struct V4 {
  T v[4];
};

template <class T> __device__ __forceinline__ V4<T> ld4(const T *p)
{
  V4<T> r;
  if constexpr (sizeof(T) == 4) {
    const float4 a = *reinterpret_cast<const float4 *>(p);
    r.v[0] = a.x, r.v[1] = a.y, r.v[2] = a.z, r.v[3] = a.w;
  } else {
    const double2 a = reinterpret_cast<const double2 *>(p)[0];
    const double2 b = reinterpret_cast<const double2 *>(p)[1];
    r.v[0] = a.x, r.v[1] = a.y, r.v[2] = b.x, r.v[3] = b.y;
  }
  return r;
}

template <class T> __device__ __forceinline__ void st4(T *p, const V4<T> &r)
{
  if constexpr (sizeof(T) == 4) {
    *reinterpret_cast<float4 *>(p) = make_float4(r.v[0], r.v[1], r.v[2], r.v[3]);
  } else {
    reinterpret_cast<double2 *>(p)[0] = make_double2(r.v[0], r.v[1]);
    reinterpret_cast<double2 *>(p)[1] = make_double2(r.v[2], r.v[3]);
  }
}

// Lane sum over the lane's tiles (one CTA per tile): every CTA publishes its
// partial, the lane's last CTA to arrive adds them in tile order and stores
// out[L] (or NaN when !valid); returns true in that CTA's thread 0.
__device__ __forceinline__ bool lane_finish(double v, double *part, unsigned *ticket,
                                            double *out, int L, int t0, int nt, bool valid)
{
  __shared__ bool last;
  v = block_sum_f64(v);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = v;
    __threadfence();
    last = atomicAdd(ticket + L, 1u) == (unsigned)nt - 1u;
  }
  __syncthreads();
  if (!last)
    return false;
  __threadfence();
  double s = 0.0;
  for (int k = threadIdx.x; k < nt; k += blockDim.x)
    s += __ldcg(part + t0 + k);
  s = block_sum_f64(s);
  if (threadIdx.x == 0) {
    out[L] = valid ? s : __longlong_as_double(0x7ff8000000000000LL);
    ticket[L] = 0u;
  }
  return threadIdx.x == 0;
}

// d += alpha p, r -= alpha q (alpha = rz / pq of the tile's lane); lane sums
// of r.r.  A non-positive or non-finite alpha leaves r, d alone and reports
// r.r = NaN (breakdown, seen by the direction step).
template <class T>
__global__ void __launch_bounds__(kThreads)
    b_update_kernel(const T *__restrict__ p, const T *__restrict__ q, T *__restrict__ r,
                    T *__restrict__ d, LaneArgs la, int par)
{
  const int t = blockIdx.x;
  const int L = la.tile_lane[t];
  if (la.state[L] != kRun)
    return;
  const double alpha = la.rz[par * la.n_lanes + L] / la.pq[L];
  const bool ok = alpha > 0.0 && isfinite(alpha);
  double acc = 0.0;
  if (ok) {
    const T a = (T)alpha;
    const long long i = (long long)t * kTile + 4 * threadIdx.x;
    const V4<T> pv = ld4(p + i), qv = ld4(q + i);
    V4<T> rv = ld4(r + i), dv = ld4(d + i);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      rv.v[k] = fma(-a, qv.v[k], rv.v[k]);
      dv.v[k] = fma(a, pv.v[k], dv.v[k]);
      acc = fma((double)rv.v[k], (double)rv.v[k], acc);
    }
    st4(r + i, rv);
    st4(d + i, dv);
  }
  if (lane_finish(acc, la.part_rr, la.t_rr, la.rr, L, la.lane_tile0[L], la.lane_ntile[L], ok) &&
      ok)
    la.it[L] += 1;
}

// p = z + beta p with beta = rzn / rz_old of the tile's lane.
// mode 0 (inside the iteration graph): first the lane stop test on r.r
//   (converged, or fell by the replacement ratio since the last reliable
//   update; breakdown; iteration cap); rz_old from the parity slot, the new
//   value goes to the other slot.
// mode 1 (after a reliable update): rz_old = rz_prev, beta = 0 for a fresh
//   lane; both slots take the new value.
// Only the lane's first tile writes lane scalars; every tile of a lane takes
// the same branch (same inputs), and a tile that sees the state its lane's
// first tile just changed skips exactly as that branch would.
template <class T>
__global__ void __launch_bounds__(kThreads)
    b_direction_kernel(const T *__restrict__ z, T *__restrict__ p, LaneArgs la,
                       const double *__restrict__ rz_lane, int par, int mode)
{
  const int t = blockIdx.x;
  const int L = la.tile_lane[t];
  if (la.state[L] != kRun)
    return;
  const bool lead = t == la.lane_tile0[L] && threadIdx.x == 0;
  if (mode == 0) {
    const double rr = la.rr[L];
    const bool brk = !isfinite(rr);
    const bool stop = !brk && (!(rr > la.thresh2[L]) || rr < la.ru2ref[L]);
    const bool cap = la.it[L] >= la.max_it;
    if (brk || stop || cap) {
      if (lead) {
        la.state[L] = brk ? kBreak : stop ? kStopConv : kCap;
        la.skip[L] = 1;
      }
      return;
    }
  }
  const double rzn = rz_lane[L];
  const bool fresh = mode == 1 && la.fresh[L];
  const double rzo = mode == 0 ? la.rz[par * la.n_lanes + L] : la.rz_prev[L];
  const double beta = fresh ? 0.0 : rzn / rzo;
  if (!(rzn > 0.0) || !isfinite(beta)) {
    if (lead) {
      la.state[L] = rzn == 0.0 ? kStopConv : kBreak;
      la.skip[L] = 1;
    }
    return;
  }
  const T b = (T)beta;
  const long long i = (long long)t * kTile + 4 * threadIdx.x;
  const V4<T> zv = ld4(z + i);
  V4<T> pv;
  if (fresh) {
    pv = zv;
  } else {
    pv = ld4(p + i);
#pragma unroll
    for (int k = 0; k < 4; k++)
      pv.v[k] = fma(b, pv.v[k], zv.v[k]);
  }
  st4(p + i, pv);
  if (lead) {
    la.rz_cur[L] = rzn;
    if (mode == 0) {
      la.rz[(1 - par) * la.n_lanes + L] = rzn;
    } else {
      la.rz[L] = rzn;
      la.rz[la.n_lanes + L] = rzn;
    }
  }
}

// Reliable update, part 1: x += d, d = 0 for every unfinished lane.
template <class T>
__global__ void __launch_bounds__(kThreads)
    b_fold_kernel(double *__restrict__ x, T *__restrict__ d, LaneArgs la)
{
  const int t = blockIdx.x;
  if (la.fin[la.tile_lane[t]])
    return;
  const long long i = (long long)t * kTile + 4 * threadIdx.x;
  const V4<T> dv = ld4(d + i);
  V4<T> zero;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    x[i + k] += (double)dv.v[k];
    zero.v[k] = T(0);
  }
  st4(d + i, zero);
}

// Reliable update, part 2: r64 = b - A x (ax == NULL: x = 0), r = (T) r64,
// lane sums of ||r64||^2.
template <class T>
__global__ void __launch_bounds__(kThreads)
    b_residual_kernel(const double *__restrict__ b, const double *__restrict__ ax,
                      double *__restrict__ r64, T *__restrict__ r, LaneArgs la)
{
  const int t = blockIdx.x;
  const int L = la.tile_lane[t];
  if (la.fin[L])
    return;
  const long long i = (long long)t * kTile + 4 * threadIdx.x;
  double acc = 0.0;
  V4<T> rv;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const double v = ax ? b[i + k] - ax[i + k] : b[i + k];
    r64[i + k] = v;
    rv.v[k] = (T)v;
    acc = fma(v, v, acc);
  }
  st4(r + i, rv);
  lane_finish(acc, la.part_res, la.t_res, la.res, L, la.lane_tile0[L], la.lane_ntile[L], true);
}

__global__ void b_scatter_kernel(double *__restrict__ out, const unsigned *__restrict__ at,
                                 const double *__restrict__ in, long long n)
{
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x)
    out[at[k]] = in[k];
}

struct Mem {
  std::vector<void *> blocks;
  ~Mem()
  {
    for (void *p : blocks)
      cudaFree(p);
  }
  template <class T> int get(T **out, size_t count)
  {
    void *p = nullptr;
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(ISPM_ERR_NOMEM, "batch cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
    }
    blocks.push_back(p);
    e = cudaMemset(p, 0, bytes);
    if (e != cudaSuccess)
      return fail(ISPM_ERR_CUDA, "cudaMemset: %s", cudaGetErrorString(e));
    *out = (T *)p;
    return ISPM_OK;
  }
  template <class T> int put(T **out, const T *h, size_t count)
  {
    if (int e = get(out, count))
      return e;
    if (count)
      ISPM_CUDA_TRY(cudaMemcpy(*out, h, count * sizeof(T), cudaMemcpyHostToDevice));
    return ISPM_OK;
  }
};

// Rows [r0, r1) of a CSR as a CSR of its own (columns unchanged).
void band(const int *rp, const int *ci, const double *v, int r0, int r1, std::vector<int> &brp,
          std::vector<int> &bci, std::vector<double> &bv)
{
  brp.resize(r1 - r0 + 1);
  for (int i = r0; i <= r1; i++)
    brp[i - r0] = rp[i] - rp[r0];
  bci.assign(ci + rp[r0], ci + rp[r1]);
  if (v)
    bv.assign(v + rp[r0], v + rp[r1]);
  else
    bv.assign(bci.size(), 1.0);
}

// Shape for a system's operator, chosen on a band of rows from its middle
// (its first rows are a boundary plane, atypical for a stencil).
int band_format(int elm_dtype, int n, const int *rp, const int *ci, const double *v,
                ispm_slell_params &out)
{
  const int m = std::min(n, kSampleRows);
  const int r0 = (n - m) / 2;
  std::vector<int> brp, bci;
  std::vector<double> bv;
  band(rp, ci, v, r0, r0 + m, brp, bci, bv);
  return choose_format(elm_dtype, m, n, brp.data(), bci.data(), bv.data(), true, out);
}

bool same_shape(const ispm_slell_params &a, const ispm_slell_params &b)
{
  return a.S == b.S && a.H == b.H && a.V == b.V && a.D == b.D;
}

}  // namespace

struct Lane {
  int system, rhs, group;
  long long row0;  // first row in the stacked vectors
  int n;           // rows of the system
  int tile0, ntile;
};

struct Group {
  ispm_slell_params fmt{}, g_fmt{}, h_fmt{};
  long long row0 = 0, rows = 0;  // the group's lanes in the stacked vectors
  int tile0 = 0, tiles = 0;
  int lane0 = 0, lanes = 0;
  // the group's systems, each once, in the stacked matrices
  std::vector<int> systems, sys_tile0;
  int mat_tiles = 0;
  // virtual tiles (matrix tile, lane tile): system by system, tile by tile,
  // the system's lanes one after another
  int2 *vt = nullptr;
  unsigned n_vt = 0;
  Operator A64, Ain, G, Ht;
};

struct Batch {
  ispm_solver_opts opts{};
  int inner = ISPM_F32;
  bool have_prec = true;
  std::vector<Lane> lanes;
  std::vector<Group> groups;
  std::vector<int> sys_rows, sys_rhs;
  std::vector<long long> sys_lane0;  // first lane of each system
  long long n_stack = 0;
  int n_tiles = 0, n_lanes = 0;
  unsigned fsai_fallbacks = 0;
  Mem mem;
  LaneArgs la{};
  int *ib = nullptr;  // state | skip | fin | fresh | it
  int *tile_lane = nullptr;
  int *a_beg = nullptr, *a_cnt = nullptr, *h_beg = nullptr, *h_cnt = nullptr;
  double *part_a = nullptr, *part_h = nullptr;
  unsigned *t_pq = nullptr, *t_rz = nullptr;
  void *vec[6] = {};
  enum { P, Q, R, D, Z, TT };
  double *r64 = nullptr, *t64 = nullptr, *b_stage = nullptr, *x_stage = nullptr;
  // pinned host mirrors
  int *ib_h = nullptr;
  double *res_h = nullptr, *rr_h = nullptr, *thr_h = nullptr, *ref_h = nullptr;
  double *hb = nullptr, *hx = nullptr;  // staging for host-vector solves
  std::vector<double> bnorm, rel;
  std::vector<int> refinements, restarts, status;
  cudaGraphExec_t graph = nullptr;
  cudaStream_t own = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  int chunk = 16;
  int graph_nodes = 0;  // kernels in one replay of the chunk graph
  int launches = 0;  // kernels launched by the last solve (graph nodes counted)
  bool completed = false;  // the last solve ran to its end (lane results are valid)
  bool verbose = getenv("ISPM_SOLVER_VERBOSE") && atoi(getenv("ISPM_SOLVER_VERBOSE")) > 0;

  ~Batch()
  {
    if (graph)
      cudaGraphExecDestroy(graph);
    for (void *p : {(void *)ib_h, (void *)res_h, (void *)rr_h, (void *)thr_h, (void *)ref_h,
                    (void *)hb, (void *)hx})
      if (p)
        cudaFreeHost(p);
    if (ev_in)
      cudaEventDestroy(ev_in);
    if (ev_out)
      cudaEventDestroy(ev_out);
    if (own)
      cudaStreamDestroy(own);
  }

  size_t esize() const { return inner == ISPM_F32 ? 4 : 8; }
  void *vp(int k, long long row0) const { return (char *)vec[k] + row0 * (long long)esize(); }

  int launched(const char *what)
  {
    launches++;
    cudaError_t e = cudaPeekAtLastError();
    return e == cudaSuccess ? ISPM_OK : fail(ISPM_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  }

  SpmvLanes lanes_for(const Group &g, const int *done) const
  {
    SpmvLanes ln;
    ln.tile_lane = tile_lane;
    ln.tile_base = (unsigned)g.tile0;
    ln.done = done;
    ln.vt = g.vt;
    ln.n_vt = g.n_vt;
    ln.lane_tile0 = la.lane_tile0;
    return ln;
  }

  // q = A p (lane sums of p.q), every group.
  int spmv_a(cudaStream_t s)
  {
    for (const Group &g : groups) {
      SpmvLanes ln = lanes_for(g, la.skip);
      ln.v = vp(P, g.row0);
      ln.out = la.pq;
      ln.part = part_a;
      ln.ticket = t_pq;
      ln.cta_beg = a_beg;
      ln.cta_cnt = a_cnt;
      if (int e = g.Ain.apply_lanes(inner, vp(P, g.row0), vp(Q, g.row0), s, ln))
        return e;
      launches++;
    }
    return ISPM_OK;
  }

  // z = G^T (G r) (lane sums of r.z); nothing without a preconditioner.
  int precondition(cudaStream_t s)
  {
    if (!have_prec)
      return ISPM_OK;
    for (const Group &g : groups) {
      SpmvLanes ln = lanes_for(g, la.skip);
      if (int e = g.G.apply_lanes(inner, vp(R, g.row0), vp(TT, g.row0), s, ln))
        return e;
      ln.v = vp(R, g.row0);
      ln.out = la.rzn;
      ln.part = part_h;
      ln.ticket = t_rz;
      ln.cta_beg = h_beg;
      ln.cta_cnt = h_cnt;
      if (int e = g.Ht.apply_lanes(inner, vp(TT, g.row0), vp(Z, g.row0), s, ln))
        return e;
      launches += 2;
    }
    return ISPM_OK;
  }

  // One iteration; `last` (the chunk's final step) stops after the r / d
  // update: the reliable update that follows computes z from the true
  // residual and takes the direction step.
  template <class T> int iteration_t(cudaStream_t s, int par, bool last)
  {
    if (int e = spmv_a(s))
      return e;
    b_update_kernel<T><<<n_tiles, kThreads, 0, s>>>((const T *)vec[P], (const T *)vec[Q],
                                                    (T *)vec[R], (T *)vec[D], la, par);
    if (int e = launched("batch update"))
      return e;
    if (last)
      return ISPM_OK;
    if (int e = precondition(s))
      return e;
    const T *z = (const T *)(have_prec ? vec[Z] : vec[R]);
    b_direction_kernel<T><<<n_tiles, kThreads, 0, s>>>(z, (T *)vec[P], la,
                                                       have_prec ? la.rzn : la.rr, par, 0);
    return launched("batch direction");
  }

  int iteration(cudaStream_t s, int par, bool last)
  {
    return inner == ISPM_F32 ? iteration_t<float>(s, par, last)
                             : iteration_t<double>(s, par, last);
  }

  int run_chunk(cudaStream_t s)
  {
    if (!opts.use_graph) {
      for (int k = 0; k < chunk; k++)
        if (int e = iteration(s, k & 1, k == chunk - 1))
          return e;
      return ISPM_OK;
    }
    if (!graph) {
      cudaGraph_t g;
      const int before = launches;
      ISPM_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      int err = ISPM_OK;
      for (int k = 0; k < chunk && !err; k++)
        err = iteration(s, k & 1, k == chunk - 1);
      cudaError_t e = cudaStreamEndCapture(s, &g);
      graph_nodes = launches - before;
      launches = before;  // counted when replayed
      if (err)
        return err;
      if (e != cudaSuccess)
        return fail(ISPM_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
      e = cudaGraphInstantiate(&graph, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess)
        return fail(ISPM_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    }
    ISPM_CUDA_TRY(cudaGraphLaunch(graph, s));
    launches += graph_nodes;
    return ISPM_OK;
  }

  // Reliable update for every unfinished lane: x += d, r = b - A x (FP64),
  // lane sums of ||r||^2; the lane tables and sums come back to the host.
  template <class T> int true_residual_t(const double *b, double *x, cudaStream_t s, bool zero_x)
  {
    if (!zero_x) {
      b_fold_kernel<T><<<n_tiles, kThreads, 0, s>>>(x, (T *)vec[D], la);
      if (int e = launched("batch fold"))
        return e;
      for (const Group &g : groups) {
        SpmvLanes ln = lanes_for(g, la.fin);
        if (int e = g.A64.apply_lanes(ISPM_F64, x + g.row0, t64 + g.row0, s, ln))
          return e;
        launches++;
      }
    }
    b_residual_kernel<T><<<n_tiles, kThreads, 0, s>>>(b, zero_x ? nullptr : t64, r64,
                                                      (T *)vec[R], la);
    if (int e = launched("batch residual"))
      return e;
    ISPM_CUDA_TRY(cudaMemcpyAsync(ib_h, ib, 5 * sizeof(int) * n_lanes, cudaMemcpyDeviceToHost, s));
    ISPM_CUDA_TRY(cudaMemcpyAsync(res_h, la.res, sizeof(double) * n_lanes, cudaMemcpyDeviceToHost,
                                  s));
    ISPM_CUDA_TRY(cudaMemcpyAsync(rr_h, la.rr, sizeof(double) * n_lanes, cudaMemcpyDeviceToHost, s));
    ISPM_CUDA_TRY(cudaStreamSynchronize(s));
    return ISPM_OK;
  }

  int true_residual(const double *b, double *x, cudaStream_t s, bool zero_x)
  {
    return inner == ISPM_F32 ? true_residual_t<float>(b, x, s, zero_x)
                             : true_residual_t<double>(b, x, s, zero_x);
  }

  // After the host reset the lane tables: z = M r and the new direction.
  template <class T> int restart_t(cudaStream_t s)
  {
    ISPM_CUDA_TRY(cudaMemcpyAsync(ib, ib_h, 4 * sizeof(int) * n_lanes, cudaMemcpyHostToDevice, s));
    ISPM_CUDA_TRY(
        cudaMemcpyAsync(la.ru2ref, ref_h, sizeof(double) * n_lanes, cudaMemcpyHostToDevice, s));
    if (int e = precondition(s))
      return e;
    ISPM_CUDA_TRY(cudaMemcpyAsync(la.rz_prev, la.rz_cur, sizeof(double) * n_lanes,
                                  cudaMemcpyDeviceToDevice, s));
    const T *z = (const T *)(have_prec ? vec[Z] : vec[R]);
    b_direction_kernel<T><<<n_tiles, kThreads, 0, s>>>(z, (T *)vec[P], la,
                                                       have_prec ? la.rzn : la.res, 0, 1);
    if (int e = launched("batch direction"))
      return e;
    ISPM_CUDA_TRY(cudaMemsetAsync(la.fresh, 0, sizeof(int) * n_lanes, s));
    return ISPM_OK;
  }

  int restart(cudaStream_t s)
  {
    return inner == ISPM_F32 ? restart_t<float>(s) : restart_t<double>(s);
  }

  int solve(const double *b, double *x, ispm_solve_stats *lane_stats, ispm_solve_stats *total,
            cudaStream_t s)
  {
    auto t0 = std::chrono::steady_clock::now();
    launches = 0;
    completed = false;
    const int n = n_lanes;
    int *state = ib_h, *skip = ib_h + n, *fin = ib_h + 2 * n, *fresh = ib_h + 3 * n,
        *its = ib_h + 4 * n;
    bnorm.assign(n, 0.0);
    rel.assign(n, 0.0);
    refinements.assign(n, 0);
    restarts.assign(n, 0);
    status.assign(n, ISPM_OK);
    for (int L = 0; L < n; L++)
      state[L] = kRun, skip[L] = 0, fin[L] = 0, fresh[L] = 1, its[L] = 0;
    ISPM_CUDA_TRY(cudaMemcpyAsync(ib, ib_h, 5 * sizeof(int) * n, cudaMemcpyHostToDevice, s));
    ISPM_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(double) * n_stack, s));
    ISPM_CUDA_TRY(cudaMemsetAsync(vec[D], 0, esize() * n_stack, s));
    if (int e = true_residual(b, x, s, true))  // r = b
      return e;
    int active = 0;
    const double ru = inner == ISPM_F32 ? opts.replace_ratio_f32 : opts.replace_ratio_f64;
    for (int L = 0; L < n; L++) {
      bnorm[L] = std::sqrt(res_h[L]);
      const double target = opts.tol * bnorm[L];
      thr_h[L] = 0.25 * target * target;
      ref_h[L] = ru * ru * res_h[L];
      if (bnorm[L] == 0.0) {  // x = 0 solves it
        state[L] = kFinished, skip[L] = 1, fin[L] = 1;
      } else if (!std::isfinite(bnorm[L])) {  // NaN / Inf in b: the lane cannot converge
        state[L] = kFailed, skip[L] = 1, fin[L] = 1;
        status[L] = ISPM_ERR_INVALID;
        rel[L] = bnorm[L];
      } else {
        rel[L] = 1.0;
        active++;
      }
    }
    ISPM_CUDA_TRY(
        cudaMemcpyAsync(la.thresh2, thr_h, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    int rounds = 0;
    while (active > 0) {
      if (int e = restart(s))
        return e;
      if (int e = run_chunk(s))
        return e;
      if (int e = true_residual(b, x, s, false))
        return e;
      rounds++;
      active = 0;
      for (int L = 0; L < n; L++) {
        if (fin[L])
          continue;
        const double r = std::sqrt(res_h[L]) / bnorm[L];
        const int st = state[L];
        const double before = rel[L];
        rel[L] = r;
        if (r <= opts.tol) {
          state[L] = kFinished, fin[L] = 1, skip[L] = 1;
          continue;
        }
        bool failed = false;
        if (st == kCap || its[L] >= opts.max_iters) {
          status[L] = ISPM_ERR_NOT_CONVERGED;
          failed = true;
        } else if (refinements[L] + restarts[L] >= opts.max_refinements) {
          status[L] = ISPM_ERR_NOT_CONVERGED;
          failed = true;
        } else if (st == kBreak) {
          restarts[L]++;
          fresh[L] = 1;
          if (!(r < before) && restarts[L] > 2) {
            status[L] = ISPM_ERR_BREAKDOWN;
            failed = true;
          }
        } else {
          refinements[L]++;
          // the recursive residual ran far below the true one (the inner
          // precision's drift): the old direction no longer fits, restart
          if (!(res_h[L] <= 4.0 * rr_h[L]))
            fresh[L] = 1;
        }
        if (failed) {
          state[L] = kFailed, fin[L] = 1, skip[L] = 1;
          continue;
        }
        ref_h[L] = ru * ru * res_h[L];
        state[L] = kRun, skip[L] = 0;
        active++;
      }
      if (verbose)
        fprintf(stderr, "[ispm batch] round %d: %d of %d lanes continue\n", rounds, active, n);
    }
    int worst = ISPM_OK, max_it = 0, max_ref = 0, all_conv = 1;
    double max_rel = 0.0;
    for (int L = 0; L < n; L++) {
      const bool conv = rel[L] <= opts.tol;
      if (lane_stats) {
        ispm_solve_stats &o = lane_stats[L];
        o.iterations = its[L];
        o.refinements = refinements[L] + restarts[L];
        o.converged = conv;
        o.status = conv ? ISPM_OK : (status[L] ? status[L] : ISPM_ERR_NOT_CONVERGED);
        o.true_relres = rel[L];
        o.seconds = 0.0;
      }
      if (!conv && !worst)
        worst = status[L] ? status[L] : ISPM_ERR_NOT_CONVERGED;
      all_conv &= conv;
      max_it = std::max(max_it, its[L]);
      max_ref = std::max(max_ref, refinements[L] + restarts[L]);
      max_rel = std::max(max_rel, rel[L]);
    }
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (lane_stats)
      for (int L = 0; L < n; L++)
        lane_stats[L].seconds = secs;
    if (total) {
      total->iterations = max_it;
      total->refinements = max_ref;
      total->converged = all_conv;
      total->status = worst;
      total->true_relres = max_rel;
      total->seconds = secs;
    }
    completed = true;
    if (worst)
      return fail(worst, "batched solve: some lanes stopped above the tolerance (worst %.3e)",
                  max_rel);
    return ISPM_OK;
  }

  int solve_on(const double *b, double *x, ispm_solve_stats *lane_stats, ispm_solve_stats *total,
               cudaStream_t user)
  {
    NvtxRange range("ispm batch solve");
    ISPM_CUDA_TRY(cudaEventRecord(ev_in, user));
    ISPM_CUDA_TRY(cudaStreamWaitEvent(own, ev_in, 0));
    int e = solve(b, x, lane_stats, total, own);
    cudaError_t ce = cudaEventRecord(ev_out, own);
    if (ce == cudaSuccess)
      ce = cudaStreamWaitEvent(user, ev_out, 0);
    if (e)
      return e;
    if (ce != cudaSuccess)
      return fail(ISPM_ERR_CUDA, "stream join: %s", cudaGetErrorString(ce));
    return ISPM_OK;
  }

  int build(int n_systems, const int *n_rows, const int *const *rp, const int *const *ci,
            const double *const *v, const int *n_rhs);
  int build_group(Group &g, const int *const *rp, const int *const *ci, const double *const *v);
};

// Stack the group's lanes into one block-diagonal CSR (identity rows pad
// every lane to whole tiles) and upload its operators; the FSAI factor of
// the stack is computed on the device.
int Batch::build_group(Group &g, const int *const *rp, const int *const *ci,
                       const double *const *v)
{
  // the matrix stack holds each system once, tile-padded; the virtual
  // tiles map every lane tile onto its system's matrix tile
  long long rows = 0, nnz = 0;
  std::vector<int2> vt;
  g.sys_tile0.clear();
  for (int k : g.systems) {
    const int n_k = sys_rows[k], nt = (n_k + kTile - 1) / kTile;
    g.sys_tile0.push_back((int)(rows / kTile));
    rows += (long long)nt * kTile;
    nnz += rp[k][n_k] + ((long long)nt * kTile - n_k);
  }
  if (rows > 0x7fffffffLL || nnz > 0x7fffffffLL)
    return fail(ISPM_ERR_TOO_LARGE, "a group of %lld rows / %lld entries exceeds the int32 "
                "CSR range", rows, nnz);
  g.mat_tiles = (int)(rows / kTile);
  for (size_t s_i = 0; s_i < g.systems.size(); s_i++) {
    const int k = g.systems[s_i];
    const int nt = (sys_rows[k] + kTile - 1) / kTile;
    for (int t = 0; t < nt; t++)
      for (int L = (int)sys_lane0[k]; L < (int)sys_lane0[k] + sys_rhs[k]; L++)
        vt.push_back(make_int2(g.sys_tile0[s_i] + t, lanes[L].tile0 + t));
  }
  g.n_vt = (unsigned)vt.size();
  if (g.n_vt != (unsigned)g.tiles)
    return fail(ISPM_ERR_INVALID, "virtual tiles do not cover the group's lanes");
  if (int e = mem.put(&g.vt, vt.data(), vt.size()))
    return e;
  std::vector<int> srp((size_t)rows + 1), sci((size_t)nnz);
  std::vector<double> sv((size_t)nnz);
  long long at = 0, row = 0;
  srp[0] = 0;
  for (int k : g.systems) {
    const int *r = rp[k], *c = ci[k];
    const double *x = v[k];
    const int n_k = sys_rows[k], nt = (n_k + kTile - 1) / kTile;
    const int off = (int)row;
    for (int i = 0; i < n_k; i++, row++) {
      for (int e = r[i]; e < r[i + 1]; e++, at++) {
        sci[at] = c[e] + off;
        sv[at] = x[e];
      }
      srp[row + 1] = (int)at;
    }
    for (int i = n_k; i < nt * kTile; i++, row++) {  // identity padding
      sci[at] = off + i;
      sv[at] = 1.0;
      at++;
      srp[row + 1] = (int)at;
    }
  }
  const int n = (int)rows;
  if (int e = g.Ain.upload(inner, inner, n, srp.data(), sci.data(), sv.data(), &g.fmt))
    return e;
  if (int e = g.A64.upload(ISPM_F64, ISPM_F64, n, srp.data(), sci.data(), sv.data(), &g.fmt))
    return e;
  if ((long long)g.Ain.dev.meta.n_rows != rows || (long long)g.A64.dev.meta.n_rows != rows)
    return fail(ISPM_ERR_INVALID, "stacked operator padded beyond its tiles");
  // lane-segmented launches walk x through registers (the staged shape is
  // for single systems)
  g.Ain.lp = register_walk_launch(inner, g.Ain.dev.view());
  g.A64.lp = register_walk_launch(ISPM_F64, g.A64.dev.view());
  if (!have_prec)
    return ISPM_OK;
  std::vector<int> g_rp, g_ci, t_rp, t_ci;
  std::vector<unsigned> t_of, pos_g, pos_t;
  if (int e = fsai_lower_pattern(n, srp.data(), sci.data(), g_rp, g_ci))
    return e;
  fsai_transpose_pattern(n, g_rp, g_ci, t_rp, t_ci, t_of);
  const size_t nnz_g = g_ci.size();
  std::vector<double> zeros(nnz_g, 0.0);  // structure only; values come from the GPU
  if (int e = g.G.upload(inner, inner, n, g_rp.data(), g_ci.data(), zeros.data(), &g.g_fmt,
                         &pos_g))
    return e;
  if (int e = g.Ht.upload(inner, inner, n, t_rp.data(), t_ci.data(), zeros.data(), &g.h_fmt,
                          &pos_t))
    return e;
  g.G.lp = register_walk_launch(inner, g.G.dev.view());
  g.Ht.lp = register_walk_launch(inner, g.Ht.dev.view());
  Mem tmp;
  int *a_rp_d, *a_ci_d, *g_rp_d;
  double *a_v_d, *g_v_d, *gt_v_d;
  unsigned *t_of_d, *pos_g_d, *pos_t_d, *fb_d;
  if (int e = tmp.put(&a_rp_d, srp.data(), srp.size()))
    return e;
  if (int e = tmp.put(&a_ci_d, sci.data(), sci.size()))
    return e;
  if (int e = tmp.put(&a_v_d, sv.data(), sv.size()))
    return e;
  if (int e = tmp.put(&g_rp_d, g_rp.data(), g_rp.size()))
    return e;
  if (int e = tmp.put(&t_of_d, t_of.data(), nnz_g))
    return e;
  if (int e = tmp.put(&pos_g_d, pos_g.data(), nnz_g))
    return e;
  if (int e = tmp.put(&pos_t_d, pos_t.data(), nnz_g))
    return e;
  if (int e = tmp.get(&g_v_d, nnz_g))
    return e;
  if (int e = tmp.get(&gt_v_d, nnz_g))
    return e;
  if (int e = tmp.get(&fb_d, 1))
    return e;
  if (int e = fsai_build_values(n, a_rp_d, a_ci_d, a_v_d, g_rp_d, g_v_d, fb_d, 0))
    return e;
  const int blocks = (int)std::min<long long>(((long long)nnz_g + 255) / 256, 148LL * 16);
  b_scatter_kernel<<<std::max(blocks, 1), 256>>>(gt_v_d, t_of_d, g_v_d, (long long)nnz_g);
  ISPM_CUDA_TRY(cudaPeekAtLastError());
  if (int e = refresh_values(g.G.dev, pos_g_d, g_v_d, ISPM_F64, (long long)nnz_g, 0))
    return e;
  if (int e = refresh_values(g.Ht.dev, pos_t_d, gt_v_d, ISPM_F64, (long long)nnz_g, 0))
    return e;
  unsigned fb = 0;
  ISPM_CUDA_TRY(cudaMemcpy(&fb, fb_d, sizeof(unsigned), cudaMemcpyDeviceToHost));
  fsai_fallbacks += fb;
  return ISPM_OK;
}

int Batch::build(int n_systems, const int *n_rows, const int *const *rp, const int *const *ci,
                 const double *const *v, const int *n_rhs)
{
  sys_rows.assign(n_rows, n_rows + n_systems);
  sys_rhs.assign(n_rhs, n_rhs + n_systems);
  // per-system shapes (A, and the FSAI factor pair) on a band of rows
  struct Shape {
    ispm_slell_params a, g, h;
  };
  std::vector<Shape> shape(n_systems);
  for (int k = 0; k < n_systems; k++) {
    Shape &sh = shape[k];
    const int n = n_rows[k];
    if (int e = band_format(inner, n, rp[k], ci[k], v[k], sh.a))
      return e;
    sh.g = sh.h = sh.a;
    if (have_prec) {
      std::vector<int> g_rp, g_ci, t_rp, t_ci;
      std::vector<unsigned> t_of;
      if (int e = fsai_lower_pattern(n, rp[k], ci[k], g_rp, g_ci))
        return e;
      fsai_transpose_pattern(n, g_rp, g_ci, t_rp, t_ci, t_of);
      if (int e = band_format(inner, n, g_rp.data(), g_ci.data(), nullptr, sh.g))
        return e;
      if (int e = band_format(inner, n, t_rp.data(), t_ci.data(), nullptr, sh.h))
        return e;
    }
  }
  // groups: systems whose A takes the same shape, in order of first
  // appearance (every group costs one launch per SpMV of an iteration); the
  // factor pair of a group takes the shapes of its system with the most
  // stored entries (summed over right-hand sides)
  std::vector<int> sys_group(n_systems);
  std::vector<long long> heaviest;
  for (int k = 0; k < n_systems; k++) {
    int gi = -1;
    for (int j = 0; j < (int)groups.size() && gi < 0; j++)
      if (same_shape(groups[j].fmt, shape[k].a))
        gi = j;
    if (gi < 0) {
      gi = (int)groups.size();
      groups.emplace_back();
      groups.back().fmt = shape[k].a;
      heaviest.push_back(-1);
    }
    sys_group[k] = gi;
    const long long w = (long long)rp[k][n_rows[k]] * n_rhs[k];
    if (w > heaviest[gi]) {
      heaviest[gi] = w;
      groups[gi].g_fmt = shape[k].g;
      groups[gi].h_fmt = shape[k].h;
    }
  }
  // lanes: grouped, then by system, then by right-hand side
  sys_lane0.assign(n_systems, 0);
  long long row = 0;
  int tile = 0;
  for (int gi = 0; gi < (int)groups.size(); gi++) {
    Group &g = groups[gi];
    g.row0 = row;
    g.tile0 = tile;
    g.lane0 = (int)lanes.size();
    for (int k = 0; k < n_systems; k++) {
      if (sys_group[k] != gi)
        continue;
      g.systems.push_back(k);
      sys_lane0[k] = (long long)lanes.size();
      for (int j = 0; j < n_rhs[k]; j++) {
        Lane ln;
        ln.system = k;
        ln.rhs = j;
        ln.group = gi;
        ln.row0 = row;
        ln.n = n_rows[k];
        ln.tile0 = tile;
        ln.ntile = (n_rows[k] + kTile - 1) / kTile;
        lanes.push_back(ln);
        row += (long long)ln.ntile * kTile;
        tile += ln.ntile;
      }
    }
    g.lanes = (int)lanes.size() - g.lane0;
    g.rows = row - g.row0;
    g.tiles = tile - g.tile0;
  }
  n_stack = row;
  n_tiles = tile;
  n_lanes = (int)lanes.size();
  for (Group &g : groups)
    if (int e = build_group(g, rp, ci, v))
      return e;
  // lane tables
  std::vector<int> tl(n_tiles), lt0(n_lanes), lnt(n_lanes), ab(n_lanes), ac(n_lanes),
      hb_(n_lanes), hc(n_lanes);
  unsigned cap_a = 1, cap_h = 1;
  for (int L = 0; L < n_lanes; L++) {
    const Lane &ln = lanes[L];
    const Group &g = groups[ln.group];
    for (int t = ln.tile0; t < ln.tile0 + ln.ntile; t++)
      tl[t] = L;
    lt0[L] = ln.tile0;
    lnt[L] = ln.ntile;
    // a lane's partial slots: its tiles' CTAs, in tile order, after the
    // group's earlier lanes (a launch covers the group's lane tiles)
    const unsigned per_a = kTile / g.Ain.cta_rows();
    ab[L] = (ln.tile0 - g.tile0) * (int)per_a;
    ac[L] = ln.ntile * (int)per_a;
    cap_a = std::max(cap_a, (unsigned)g.tiles * per_a);
    if (have_prec) {
      const unsigned per_h = kTile / g.Ht.cta_rows();
      hb_[L] = (ln.tile0 - g.tile0) * (int)per_h;
      hc[L] = ln.ntile * (int)per_h;
      cap_h = std::max(cap_h, (unsigned)g.tiles * per_h);
    }
  }
  for (const Group &g : groups) {
    // every CTA of a lane-segmented launch lies in one tile, and the
    // matrix stack is exactly its tiles' CTAs
    for (const Operator *op : {&g.Ain, &g.A64, &g.G, &g.Ht}) {
      if (op == &g.G && !have_prec)
        break;
      const unsigned cr = op->cta_rows();
      if (kTile % cr || op->grid() != (unsigned)g.mat_tiles * (kTile / cr))
        return fail(ISPM_ERR_INVALID, "a stacked operator's CTAs do not tile its systems");
    }
  }
  const size_t nl = (size_t)n_lanes;
  if (int e = mem.put(&tile_lane, tl.data(), tl.size()))
    return e;
  int *lt0_d, *lnt_d;
  if (int e = mem.put(&lt0_d, lt0.data(), nl))
    return e;
  if (int e = mem.put(&lnt_d, lnt.data(), nl))
    return e;
  if (int e = mem.put(&a_beg, ab.data(), nl))
    return e;
  if (int e = mem.put(&a_cnt, ac.data(), nl))
    return e;
  if (int e = mem.put(&h_beg, hb_.data(), nl))
    return e;
  if (int e = mem.put(&h_cnt, hc.data(), nl))
    return e;
  if (int e = mem.get(&ib, 5 * nl))
    return e;
  if (int e = mem.get(&part_a, cap_a))
    return e;
  if (int e = mem.get(&part_h, cap_h))
    return e;
  if (int e = mem.get(&t_pq, nl))
    return e;
  if (int e = mem.get(&t_rz, nl))
    return e;
  la.tile_lane = tile_lane;
  la.lane_tile0 = lt0_d;
  la.lane_ntile = lnt_d;
  la.state = ib;
  la.skip = ib + nl;
  la.fin = ib + 2 * nl;
  la.fresh = ib + 3 * nl;
  la.it = ib + 4 * nl;
  double **lane_d[] = {&la.rz_cur, &la.rz_prev, &la.thresh2, &la.ru2ref,
                       &la.pq,     &la.rzn,     &la.rr,      &la.res};
  for (double **pp : lane_d)
    if (int e = mem.get(pp, nl))
      return e;
  if (int e = mem.get(&la.rz, 2 * nl))
    return e;
  if (int e = mem.get(&la.t_rr, nl))
    return e;
  if (int e = mem.get(&la.t_res, nl))
    return e;
  if (int e = mem.get(&la.part_rr, (size_t)n_tiles))
    return e;
  if (int e = mem.get(&la.part_res, (size_t)n_tiles))
    return e;
  la.max_it = opts.max_iters;
  la.n_lanes = n_lanes;
  for (int k = 0; k < 6; k++) {
    int e = inner == ISPM_F32 ? mem.get((float **)&vec[k], (size_t)n_stack)
                              : mem.get((double **)&vec[k], (size_t)n_stack);
    if (e)
      return e;
  }
  double **d64[] = {&r64, &t64, &b_stage, &x_stage};
  for (double **pp : d64)
    if (int e = mem.get(pp, (size_t)n_stack))
      return e;
  if (cudaMallocHost(&ib_h, 5 * sizeof(int) * nl) != cudaSuccess ||
      cudaMallocHost(&res_h, sizeof(double) * nl) != cudaSuccess ||
      cudaMallocHost(&rr_h, sizeof(double) * nl) != cudaSuccess ||
      cudaMallocHost(&thr_h, sizeof(double) * nl) != cudaSuccess ||
      cudaMallocHost(&ref_h, sizeof(double) * nl) != cudaSuccess ||
      cudaMallocHost(&hb, sizeof(double) * n_stack) != cudaSuccess ||
      cudaMallocHost(&hx, sizeof(double) * n_stack) != cudaSuccess) {
    cudaGetLastError();
    return fail(ISPM_ERR_NOMEM, "pinned host allocation");
  }
  memset(hb, 0, sizeof(double) * n_stack);
  ISPM_CUDA_TRY(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking));
  ISPM_CUDA_TRY(cudaEventCreateWithFlags(&ev_in, cudaEventDisableTiming));
  ISPM_CUDA_TRY(cudaEventCreateWithFlags(&ev_out, cudaEventDisableTiming));
  ISPM_CUDA_TRY(cudaDeviceSynchronize());
  return ISPM_OK;
}

}  // namespace ispm

struct ispm_batch {
  ispm::Batch b;
};

using namespace ispm;

extern "C" {

int ispm_batch_create(int n_systems, const int *n_rows, const int *const *row_ptr,
                      const int *const *cols, const double *const *vals, const int *n_rhs,
                      const ispm_solver_opts *opts, ispm_batch **out)
{
  clear_error();
  NvtxRange range("ispm batch create");
  if (!out || n_systems <= 0 || !n_rows || !row_ptr || !cols || !vals || !n_rhs)
    return fail(ISPM_ERR_INVALID, "bad arguments");
  *out = nullptr;
  for (int k = 0; k < n_systems; k++) {
    if (n_rows[k] <= 0 || n_rhs[k] <= 0 || !row_ptr[k] || !cols[k] || !vals[k])
      return fail(ISPM_ERR_INVALID, "system %d: bad arguments", k);
    if (int e = validate_csr(n_rows[k], n_rows[k], row_ptr[k], cols[k])) {
      const std::string why = ispm_last_error();
      return fail(e, "system %d: %s", k, why.c_str());
    }
  }
  std::unique_ptr<ispm_batch> h(new (std::nothrow) ispm_batch);
  if (!h)
    return fail(ISPM_ERR_NOMEM, "host allocation");
  Batch &B = h->b;
  if (opts)
    B.opts = *opts;
  else {
    ispm_solver_default_opts(&B.opts);
    B.opts.prec = ISPM_PREC_FSAI_GPU;
    // lanes advance in lockstep chunks, so a lane pauses only when needed
    B.opts.replace_ratio_f32 = 1e-3;
  }
  if (!(B.opts.replace_ratio_f32 > 0 && B.opts.replace_ratio_f32 < 1) ||
      !(B.opts.replace_ratio_f64 > 0 && B.opts.replace_ratio_f64 < 1))
    return fail(ISPM_ERR_INVALID, "replacement ratios must lie in (0, 1)");
  if (B.opts.inner_dtype != ISPM_F32 && B.opts.inner_dtype != ISPM_F64)
    return fail(ISPM_ERR_INVALID, "inner_dtype %d", B.opts.inner_dtype);
  if (B.opts.check_every < 1 || B.opts.check_every > 4096)
    return fail(ISPM_ERR_INVALID, "check_every %d", B.opts.check_every);
  if (B.opts.prec != ISPM_PREC_FSAI_GPU && B.opts.prec != ISPM_PREC_NONE)
    return fail(ISPM_ERR_INVALID, "batched prec %d (ISPM_PREC_FSAI_GPU or ISPM_PREC_NONE)",
                B.opts.prec);
  if (B.opts.max_iters < 1 || !(B.opts.tol > 0))
    return fail(ISPM_ERR_INVALID, "max_iters / tol");
  B.inner = B.opts.inner_dtype;
  B.have_prec = B.opts.prec == ISPM_PREC_FSAI_GPU;
  B.chunk = (B.opts.check_every + 1) & ~1;  // even: parity slot 0 at every chunk start
  try {
    if (int e = B.build(n_systems, n_rows, row_ptr, cols, vals, n_rhs))
      return e;
  } catch (const std::bad_alloc &) {
    return fail(ISPM_ERR_NOMEM, "host allocation while building the batch");
  }
  *out = h.release();
  return ISPM_OK;
}

int ispm_batch_lanes(const ispm_batch *b) { return b ? b->b.n_lanes : 0; }

long long ispm_batch_rows(const ispm_batch *b) { return b ? b->b.n_stack : 0; }

int ispm_batch_lane_info(const ispm_batch *b, int lane, int *system, int *rhs, long long *row0,
                         int *group)
{
  clear_error();
  if (!b || lane < 0 || lane >= b->b.n_lanes)
    return fail(ISPM_ERR_INVALID, "lane %d", lane);
  const Lane &ln = b->b.lanes[lane];
  if (system)
    *system = ln.system;
  if (rhs)
    *rhs = ln.rhs;
  if (row0)
    *row0 = ln.row0;
  if (group)
    *group = ln.group;
  return ISPM_OK;
}

int ispm_batch_groups(const ispm_batch *b, ispm_slell_params *a_fmt, int *lanes, int cap)
{
  if (!b)
    return 0;
  const int n = (int)b->b.groups.size();
  for (int g = 0; g < n && g < cap; g++) {
    if (a_fmt)
      a_fmt[g] = b->b.groups[g].fmt;
    if (lanes)
      lanes[g] = b->b.groups[g].lanes;
  }
  return n;
}

int ispm_batch_solve(ispm_batch *b, const double *b_dev, double *x_dev,
                     ispm_solve_stats *lane_stats, ispm_solve_stats *total, void *stream)
{
  clear_error();
  if (!b || !b_dev || !x_dev)
    return fail(ISPM_ERR_INVALID, "NULL argument");
  return b->b.solve_on(b_dev, x_dev, lane_stats, total, (cudaStream_t)stream);
}

int ispm_batch_solve_host(ispm_batch *b, const double *const *b_host, double *const *x_host,
                          ispm_solve_stats *lane_stats, ispm_solve_stats *total, void *stream)
{
  clear_error();
  if (!b || !b_host || !x_host)
    return fail(ISPM_ERR_INVALID, "NULL argument");
  Batch &B = b->b;
  for (const Lane &ln : B.lanes)  // pack (padding rows of hb stay zero)
    memcpy(B.hb + ln.row0, b_host[ln.system] + (size_t)ln.rhs * ln.n, sizeof(double) * ln.n);
  cudaStream_t st = (cudaStream_t)stream;
  ISPM_CUDA_TRY(cudaMemcpyAsync(B.b_stage, B.hb, sizeof(double) * B.n_stack,
                                cudaMemcpyHostToDevice, st));
  int e = B.solve_on(B.b_stage, B.x_stage, lane_stats, total, st);
  // a completed solve hands back every lane's x, also when some lanes
  // stopped (not converged, breakdown, a NaN / Inf right-hand side)
  if (e && !B.completed)
    return e;
  ISPM_CUDA_TRY(cudaMemcpyAsync(B.hx, B.x_stage, sizeof(double) * B.n_stack,
                                cudaMemcpyDeviceToHost, st));
  ISPM_CUDA_TRY(cudaStreamSynchronize(st));
  for (const Lane &ln : B.lanes)
    memcpy(x_host[ln.system] + (size_t)ln.rhs * ln.n, B.hx + ln.row0, sizeof(double) * ln.n);
  return e;
}

int ispm_batch_launches(const ispm_batch *b) { return b ? b->b.launches : 0; }

unsigned ispm_batch_fsai_fallbacks(const ispm_batch *b) { return b ? b->b.fsai_fallbacks : 0; }

void ispm_batch_free(ispm_batch *b) { delete b; }

}  // extern "C"
