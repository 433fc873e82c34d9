// Sliced-ELLPACK SpMV for sm_100a: y = A x.
//
// Same matrix layout and launch-parameter meaning as the reference kernel
// (cuda/spmv/kernel.h:1-135): a slice's entries are column-major (entry
// (r, k) at slice_start + r + k * slice_height); N threads cooperate on one
// slice, each covering H consecutive rows, so N * H / slice_height threads
// share a row and their partial sums are reduced at the end.  What changes
// for B200:
//  * several slices per CTA when N is small (the reference runs one slice per
//    block), so narrow launches still fill the SM;
//  * matrix words are fetched with 128-bit streaming loads (ld.global.cs)
//    that do not displace x from L1/L2; x is gathered through the read-only
//    path with explicit bounds (the reference relied on texture fetches
//    returning 0 out of range: diagonal-block entries of boundary rows point
//    one past either end of x);
//  * the cross-thread reduction is warp shuffles (xor butterfly, uniform
//    across the warp so slices of different heights may share one) with a
//    shared-memory step only when a slice spans several warps;
//  * hblock columns gather W consecutive x values with one vector load;
//  * a split operator (FP16 off-diagonal elements and an FP32 diagonal
//    vector, the solver's matrix_f16 option) scales the stored sum by a power
//    of two and adds the diagonal term in the store epilogue.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <type_traits>

#include "cuda_util.cuh"
#include "spmv_launch.h"

namespace ispm {
namespace {

template <class T, class E> struct SpmvArgs {
  const unsigned *__restrict__ sp;
  const unsigned *__restrict__ cols;
  const E *__restrict__ elms;
  const T *__restrict__ x;
  T *__restrict__ y;
  unsigned n_slices;
  unsigned slice_height;
  unsigned n_cols;
  unsigned tps;       // threads per slice (reference N), power of two
  unsigned log2_tps;
  int x_vec_ok;       // x aligned for W-wide vector loads
  int x_al16;         // x 16-byte aligned (diagonal-window vector loads)
  const int *skip;    // optional device flag: nonzero -> the launch does nothing
  SpmvDot ep;         // optional fused epilogue: *ep.out = sum_i y_i v_i (FP64)
  SpmvLanes ln;       // lane-segmented launches only
  int pdl;            // launched as a programmatic dependent of the previous kernel
  const float *dg;    // split operators (E = __half): FP32 diagonal, one per row
  float inv_scale;    // split operators: 1 / the power-of-two element scale
  int st_slots;       // staged walk: ring slots, bytes per slot, x area offset in a slot
  int st_slot_bytes;
  int st_x_off;
};

// Finish a fused dot product: every block publishes its partial, the last
// block to arrive adds them in block order (deterministic) and stores it.
__device__ __forceinline__ void finish_dot(double v, const SpmvDot &ep)
{
  __shared__ bool last;
  v = block_sum_f64(v);
  if (threadIdx.x == 0) {
    ep.part[blockIdx.x] = v;
    __threadfence();
    last = atomicAdd(ep.ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last)
    return;
  __threadfence();
  double s = 0.0;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
    s += __ldcg(ep.part + b);
  s = block_sum_f64(s);
  if (threadIdx.x == 0) {
    *ep.out = s;
    *ep.ticket = 0u;
  }
}

// Same for two sums at once (partials of the second at part[part_capacity + b]).
__device__ __forceinline__ void finish_dot2(double v, double w, const SpmvDot &ep)
{
  __shared__ bool last;
  v = block_sum_f64(v);
  w = block_sum_f64(w);
  if (threadIdx.x == 0) {
    ep.part[blockIdx.x] = v;
    ep.part[ep.part_capacity + blockIdx.x] = w;
    __threadfence();
    last = atomicAdd(ep.ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last)
    return;
  __threadfence();
  double s = 0.0, s2 = 0.0;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
    s += __ldcg(ep.part + b);
    s2 += __ldcg(ep.part + ep.part_capacity + b);
  }
  s = block_sum_f64(s);
  s2 = block_sum_f64(s2);
  if (threadIdx.x == 0) {
    *ep.out = s;
    *ep.out2 = s2;
    *ep.ticket = 0u;
  }
}

// Lane-segmented finish: the lane's last CTA to arrive adds the lane's
// partials in CTA order (deterministic) and stores the lane's sum.
__device__ __forceinline__ void finish_lane_dot(double v, const SpmvLanes &ln, int lane,
                                                unsigned slot)
{
  __shared__ bool last;
  v = block_sum_f64(v);
  if (threadIdx.x == 0) {
    ln.part[slot] = v;
    __threadfence();
    last = atomicAdd(ln.ticket + lane, 1u) == (unsigned)__ldg(ln.cta_cnt + lane) - 1u;
  }
  __syncthreads();
  if (!last)
    return;
  __threadfence();
  const int beg = __ldg(ln.cta_beg + lane), cnt = __ldg(ln.cta_cnt + lane);
  double s = 0.0;
  for (int c = threadIdx.x; c < cnt; c += blockDim.x)
    s += __ldcg(ln.part + beg + c);
  s = block_sum_f64(s);
  if (threadIdx.x == 0) {
    ln.out[lane] = s;
    ln.ticket[lane] = 0u;
  }
}

// Gather x[c*W .. c*W+W-1] into xw, zero beyond n_cols.
template <class T, int W>
__device__ __forceinline__ void gather_w(const T *__restrict__ x, unsigned c, unsigned n_cols,
                                         bool vec_ok, T (&xw)[W])
{
  const unsigned base = c * W;
  if (vec_ok && base + W <= n_cols) {
    if constexpr (W == 2 && sizeof(T) == 4) {
      float2 v = __ldg(reinterpret_cast<const float2 *>(x + base));
      xw[0] = v.x;
      xw[1] = v.y;
      return;
    } else if constexpr (W == 4 && sizeof(T) == 4) {
      float4 v = __ldg(reinterpret_cast<const float4 *>(x + base));
      xw[0] = v.x;
      xw[1] = v.y;
      xw[2] = v.z;
      xw[3] = v.w;
      return;
    } else if constexpr (W == 2 && sizeof(T) == 8) {
      double2 v = __ldg(reinterpret_cast<const double2 *>(x + base));
      xw[0] = v.x;
      xw[1] = v.y;
      return;
    } else if constexpr (W == 4 && sizeof(T) == 8) {
      double2 a = __ldg(reinterpret_cast<const double2 *>(x + base));
      double2 b = __ldg(reinterpret_cast<const double2 *>(x + base + 2));
      xw[0] = a.x;
      xw[1] = a.y;
      xw[2] = b.x;
      xw[3] = b.y;
      return;
    }
  }
#pragma unroll
  for (int w = 0; w < W; w++)
    xw[w] = ld_x_guard(x, base + w, n_cols);
}

// x[base .. base+H-1] for one diagonal, zero outside [0, n).  Within a slice
// base = diag_pos + row - slice_height with row a multiple of H, so
// base mod H is the same for every thread of the slice: when H values of T
// fill 16 bytes, the window is one aligned 128-bit load (two when base is
// not H-aligned) instead of H scalar loads that each touch the whole warp's
// span of cache lines.
template <class T, int H>
__device__ __forceinline__ void load_window(const T *__restrict__ x, unsigned base, unsigned n,
                                            bool vec_ok, T (&xv)[H])
{
  if constexpr (H * sizeof(T) == 16) {
    using V = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
    const unsigned sh = base & (H - 1);
    const unsigned a0 = base - sh;
    if (vec_ok && a0 < n && n - a0 >= (sh ? 2u * H : (unsigned)H)) {
      T w[2 * H];
      V v0 = __ldg(reinterpret_cast<const V *>(x + a0));
      *reinterpret_cast<V *>(w) = v0;
      if (sh) {
        V v1 = __ldg(reinterpret_cast<const V *>(x + a0 + H));
        *reinterpret_cast<V *>(w + H) = v1;
      } else {
#pragma unroll
        for (int k = H; k < 2 * H; k++)
          w[k] = T(0);
      }
#pragma unroll
      for (int h = 0; h < H; h++) {
        T r = w[h];
#pragma unroll
        for (int k = 1; k < H; k++)
          r = sh == (unsigned)k ? w[h + k] : r;
        xv[h] = r;
      }
      return;
    }
  } else if constexpr (H == 8 && sizeof(T) == 4) {
    // eight FP32 rows a thread (16-bit elements: one 128-bit element load):
    // two aligned 128-bit loads, three when base is not 4-aligned
    const unsigned sh = base & 3u;
    const unsigned a0 = base - sh;
    if (vec_ok && a0 < n && n - a0 >= (sh ? 12u : 8u)) {
      T w[12];
      *reinterpret_cast<float4 *>(w) = __ldg(reinterpret_cast<const float4 *>(x + a0));
      *reinterpret_cast<float4 *>(w + 4) = __ldg(reinterpret_cast<const float4 *>(x + a0 + 4));
      if (sh) {
        *reinterpret_cast<float4 *>(w + 8) = __ldg(reinterpret_cast<const float4 *>(x + a0 + 8));
      } else {
#pragma unroll
        for (int k = 8; k < 12; k++)
          w[k] = T(0);
      }
#pragma unroll
      for (int h = 0; h < 8; h++) {
        T r = w[h];
#pragma unroll
        for (int k = 1; k < 4; k++)
          r = sh == (unsigned)k ? w[h + k] : r;
        xv[h] = r;
      }
      return;
    }
  }
#pragma unroll
  for (int h = 0; h < H; h++)
    xv[h] = ld_x_guard(x, base + h, n);
}

template <class T, class E, int H, int W, bool VAR, bool DIAG, bool LANES>
__device__ __forceinline__ void spmv_body(const SpmvArgs<T, E> &a)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  pdl_wait();             // inputs of a programmatic launch are final from here
  if (a.skip && *a.skip)  // uniform: a converged solver's graph replays as no-ops
    return;
  constexpr unsigned spe = 1 + (W > 1) + (VAR ? 1 : 0) + (DIAG ? 2 : 0);
  const unsigned tps = a.tps;
  const unsigned t = threadIdx.x & (tps - 1);
  const unsigned slice_in_cta = threadIdx.x >> a.log2_tps;
  const unsigned spb = blockDim.x >> a.log2_tps;
  unsigned cta = blockIdx.x;
  const T *__restrict__ xp = a.x;
  T *__restrict__ yp = a.y;
  long long shift = 0;
  int lane = 0;
  unsigned slot = 0;
  if constexpr (LANES) {
    // fixed slice height: the CTA's rows lie in one tile; the virtual tile
    // names the matrix tile it reads and the lane tile it serves
    static_assert(!VAR, "lane-segmented launches use a fixed slice height");
    const unsigned per = 1024u / (spb * a.slice_height);
    const unsigned vt = blockIdx.x / per, q = blockIdx.x - vt * per;
    const int2 e = __ldg(a.ln.vt + vt);
    lane = __ldg(a.ln.tile_lane + e.y);
    if (__ldg(a.ln.done + lane))
      return;
    cta = (unsigned)e.x * per + q;
    shift = ((long long)e.y - (long long)a.ln.tile_base - (long long)e.x) * 1024;
    xp += shift;
    yp += shift;
    if (a.ln.out)
      slot = (unsigned)__ldg(a.ln.cta_beg + lane) +
             (unsigned)(e.y - __ldg(a.ln.lane_tile0 + lane)) * per + q;
  }
  const unsigned b = cta * spb + slice_in_cta;
  const bool active = b < a.n_slices;

  // Slice header (kernel.h:13-61); inactive slices walk nothing.
  unsigned e0 = 0, e1 = 0, c0 = 0, c1 = 0, cb = 0, d0 = 0, y0 = 0;
  unsigned sz = VAR ? tps * H : a.slice_height;
  if (active) {
    const unsigned *rec = a.sp + (size_t)spe * b;
    e0 = __ldg(rec);
    e1 = __ldg(rec + spe);
    if (VAR) {
      y0 = __ldg(rec + 1);
      sz = __ldg(rec + 1 + spe) - y0;
    } else {
      y0 = b * a.slice_height;
    }
    if constexpr (DIAG) {
      c0 = __ldg(rec + (VAR ? 2 : 1));
      d0 = __ldg(rec + (VAR ? 3 : 2));
      c1 = __ldg(rec + (VAR ? 2 : 1) + spe);
    } else if constexpr (W > 1) {
      c0 = __ldg(rec + (VAR ? 2 : 1));
      c1 = __ldg(rec + (VAR ? 2 : 1) + spe);
      const unsigned nse = (W * (c1 - c0) - (e1 - e0)) / (W - 1);
      cb = c1;
      c1 = c0 + nse;
      e1 = e0 + nse;
    } else {
      c0 = e0;
      c1 = e1;
    }
  }

  // lanes of one system read its matrix tile one after another: keep it in
  // L2 (default policy); a single system streams it past (evict-first)
  auto ld_m = [](const auto *q) {
    if constexpr (LANES)
      return ld_keep<H>(q);
    else
      return ld_stream<H>(q);
  };
  const unsigned step = tps * H;
  T acc[H];
#pragma unroll
  for (int h = 0; h < H; h++)
    acc[h] = T(0);

  unsigned i = e0 + t * H, j = c0 + t * H;
  // ELL part with explicit columns (kernel.h:70-79).
#pragma unroll 4
  for (; j < c1; i += step, j += step) {
    Vec<H, unsigned> cc = ld_m(a.cols + j);
    Vec<H, E> ee = ld_m(a.elms + i);
#pragma unroll
    for (int h = 0; h < H; h++)
      acc[h] = fma(T(ee.v[h]), ld_x_guard(xp, cc.v[h], a.n_cols), acc[h]);
  }
  if constexpr (DIAG) {
    // Diagonal blocks (kernel.h:80-92): column index = diag_pos + row - sz.
    const unsigned adj = ((t * H) & (sz - 1)) - sz;
    unsigned jj = d0 + (j - c1) / sz;
    const unsigned jstep = step / sz;
    const bool vec_ok = a.x_al16;
#pragma unroll 4
    for (; i < e1; i += step, jj += jstep) {
      const unsigned base = __ldg(a.sp + jj) + adj;
      Vec<H, E> ee = ld_m(a.elms + i);
      T xv[H];
      load_window<T, H>(xp, base, a.n_cols, vec_ok, xv);
#pragma unroll
      for (int h = 0; h < H; h++)
        acc[h] = fma(T(ee.v[h]), xv[h], acc[h]);
    }
  } else if constexpr (W > 1) {
    // hblock columns (kernel.h:93-119): W values per stored column index.
    i = e1 + ((i - e1) & (sz - 1)) + ((i - e1) & ~(sz - 1)) * W;
    const bool vec_ok = a.x_vec_ok;
#pragma unroll 2
    for (; j < cb; i += W * step, j += step) {
      Vec<H, unsigned> cc = ld_m(a.cols + j);
      Vec<H, E> ew[W];
#pragma unroll
      for (int w = 0; w < W; w++)
        ew[w] = ld_m(a.elms + i + w * sz);
#pragma unroll
      for (int h = 0; h < H; h++) {
        T xw[W];
        gather_w<T, W>(xp, cc.v[h], a.n_cols, vec_ok, xw);
#pragma unroll
        for (int w = 0; w < W; w++)
          acc[h] = fma(T(ew[w].v[h]), xw[w], acc[h]);
      }
    }
  }

  pdl_trigger();  // the successor may be scheduled; it waits for this grid's end
  // Reduce the partial sums of the threads sharing a row (reduce.h:80-127).
  const unsigned R = sz / H;  // row groups in this slice
  const unsigned wspan = tps < 32 ? tps : 32;
  for (unsigned off = 1; off < wspan; off <<= 1) {
#pragma unroll
    for (int h = 0; h < H; h++) {
      T v = __shfl_xor_sync(0xffffffffu, acc[h], off);
      if (off >= R)
        acc[h] += v;
    }
  }
  if (tps > 32) {
    T *red = reinterpret_cast<T *>(smem_raw);
#pragma unroll
    for (int h = 0; h < H; h++)
      red[threadIdx.x * H + h] = acc[h];
    __syncthreads();
    if (t < R) {
      const unsigned stride = R > 32 ? R : 32;
      const unsigned base = slice_in_cta * tps;
#pragma unroll
      for (int h = 0; h < H; h++) {
        T s = T(0);
        for (unsigned k = t; k < tps; k += stride)
          s += red[(base + k) * H + h];
        acc[h] = s;
      }
    }
  }
  if constexpr (std::is_same<E, __half>::value) {
    // FP16 elements: y = inv_scale * (stored sum), plus diag * x for a
    // split operator
    if (active && t < R) {
      if (a.dg) {
        const Vec<H, float> dv = ld_stream<H>(a.dg + y0 + t * H);
#pragma unroll
        for (int h = 0; h < H; h++)
          acc[h] = fma(dv.v[h], ld_x_guard(xp, y0 + t * H + h, a.n_cols), acc[h] * a.inv_scale);
      } else {
#pragma unroll
        for (int h = 0; h < H; h++)
          acc[h] *= a.inv_scale;
      }
    }
  }
  if (active && t < R)
    st_vec<H, T>(yp + y0 + t * H, acc);
  if (LANES ? a.ln.out != nullptr : a.ep.out != nullptr) {
    // fused y.v for the solver (the dot the next recurrence step needs)
    double dv = 0.0, dw = 0.0;
    const bool two = !LANES && a.ep.out2 != nullptr;
    if (active && t < R) {
      const T *v = static_cast<const T *>(LANES ? a.ln.v : a.ep.v) + shift + y0 + t * H;
#pragma unroll
      for (int h = 0; h < H; h++) {
        dv = fma((double)acc[h], (double)v[h], dv);
        if (two)
          dw = fma((double)v[h], (double)v[h], dw);
      }
    }
    if constexpr (LANES)
      finish_lane_dot(dv, a.ln, lane, slot);
    else if (two)
      finish_dot2(dv, dw, a.ep);
    else
      finish_dot(dv, a.ep);
  }
}

template <class T, class E, int H, int W, bool VAR, bool DIAG>
__global__ void __launch_bounds__(1024) slell_spmv_kernel(SpmvArgs<T, E> a)
{
  spmv_body<T, E, H, W, VAR, DIAG, false>(a);
}

// Lane-segmented instances: bounded to two 1024-thread CTAs' registers per
// SM (the virtual-tile set-up costs registers the single-system instances do
// not have).
template <class T, class E, int H, int W, bool DIAG>
__global__ void __launch_bounds__(1024, 2) slell_spmv_lanes_kernel(SpmvArgs<T, E> a)
{
  spmv_body<T, E, H, W, false, DIAG, true>(a);
}

#include "spmv_staged.cuh"


template <class T, class E, int H, int W, bool VAR, bool DIAG, bool LANES = false>
int launch_one(const SpmvArgs<T, E> &args, unsigned tps, cudaStream_t stream)
{
  // A fused dot ends every CTA with a block reduction, a fence and an
  // arrival on the counter: 1024-thread CTAs do that a quarter as often
  // (the C2 mixed solve measured 58.2 against 59.5 ms, same iterations).
  const unsigned block = (!LANES && args.ep.out) ? (tps >= 1024 ? tps : 1024)
                                                 : (tps >= 256 ? tps : 256);
  const unsigned spb = block / tps;
  // lane-segmented: every virtual tile takes 1024 / (spb * S) CTAs
  const unsigned grid = LANES ? args.ln.n_vt * (1024u / (spb * args.slice_height))
                              : (args.n_slices + spb - 1) / spb;
  const size_t smem = tps > 32 ? (size_t)block * H * sizeof(T) : 0;
  cudaError_t e;
  if constexpr (LANES)
    e = launch_kernel(slell_spmv_lanes_kernel<T, E, H, W, DIAG>, dim3(grid), dim3(block), smem,
                      stream, args.pdl != 0, args);
  else
    e = launch_kernel(slell_spmv_kernel<T, E, H, W, VAR, DIAG>, dim3(grid), dim3(block), smem,
                      stream, args.pdl != 0, args);
  if (e == cudaSuccess)
    e = cudaPeekAtLastError();
  if (e != cudaSuccess)
    return fail(ISPM_ERR_CUDA, "SpMV launch: %s", cudaGetErrorString(e));
  return ISPM_OK;
}

template <class T, class E, int H>
int launch_h(const SpmvArgs<T, E> &args, const ispm_slell_view &m, unsigned tps,
             cudaStream_t s, bool lanes)
{
  const bool V = m.var_height != 0, D = m.diags != 0;
  if (lanes) {
    if constexpr (std::is_same<T, E>::value) {
      if (V)
        return fail(ISPM_ERR_INVALID, "lane-segmented SpMV needs a fixed slice height");
      switch (m.hblock) {
      case 1:
        return D ? launch_one<T, E, H, 1, false, true, true>(args, tps, s)
                 : launch_one<T, E, H, 1, false, false, true>(args, tps, s);
      case 2: return launch_one<T, E, H, 2, false, false, true>(args, tps, s);
      case 4: return launch_one<T, E, H, 4, false, false, true>(args, tps, s);
      }
      return fail(ISPM_ERR_INVALID, "hblock %u", m.hblock);
    } else {
      return fail(ISPM_ERR_INVALID, "lane-segmented SpMV needs equal vector and element types");
    }
  }
  switch (m.hblock) {
  case 1:
    if (V)
      return D ? launch_one<T, E, H, 1, true, true>(args, tps, s)
               : launch_one<T, E, H, 1, true, false>(args, tps, s);
    return D ? launch_one<T, E, H, 1, false, true>(args, tps, s)
             : launch_one<T, E, H, 1, false, false>(args, tps, s);
  case 2:
    return V ? launch_one<T, E, H, 2, true, false>(args, tps, s)
             : launch_one<T, E, H, 2, false, false>(args, tps, s);
  case 4:
    return V ? launch_one<T, E, H, 4, true, false>(args, tps, s)
             : launch_one<T, E, H, 4, false, false>(args, tps, s);
  }
  return fail(ISPM_ERR_INVALID, "hblock %u", m.hblock);
}

template <class T, class E>
int launch_te(const ispm_launch_params &p, const ispm_slell_view &m, const void *x, void *y,
              cudaStream_t s, const int *skip, const SpmvDot *ep, const SpmvLanes *ln = nullptr,
              bool pdl = false, const SpmvSplit *split = nullptr)
{
  SpmvArgs<T, E> a;
  a.pdl = pdl ? 1 : 0;
  a.dg = nullptr;
  a.inv_scale = 1.f;
  a.st_slots = a.st_slot_bytes = a.st_x_off = 0;
  if constexpr (std::is_same<E, __half>::value) {
    if (!split || (split->diag && !aligned(split->diag, 16)))
      return fail(ISPM_ERR_INVALID,
                  "FP16 elements need their scale (and a 16-byte aligned split diagonal)");
    a.dg = split->diag;
    a.inv_scale = split->inv_scale;
  }
  a.skip = skip;
  a.ep = ep ? *ep : SpmvDot{};
  a.ln = ln ? *ln : SpmvLanes{};
  if (ep && ep->out) {
    const unsigned block = p.N >= 256 ? p.N : 256;
    const unsigned grid = (m.n_slices + block / p.N - 1) / (block / p.N);
    if (grid > ep->part_capacity)
      return fail(ISPM_ERR_INVALID, "fused dot needs %u partial slots, has %u", grid,
                  ep->part_capacity);
  }
  a.sp = m.slice_ptr;
  a.cols = m.cols;
  a.elms = static_cast<const E *>(m.elms);
  a.x = static_cast<const T *>(x);
  a.y = static_cast<T *>(y);
  a.n_slices = m.n_slices;
  a.slice_height = m.slice_height;
  a.n_cols = (unsigned)m.n_cols;
  a.tps = p.N;
  a.log2_tps = (unsigned)ilog2(p.N);
  a.x_vec_ok = aligned(x, (size_t)m.hblock * sizeof(T));
  a.x_al16 = aligned(x, 16);
  if (!aligned(m.elms, p.H * sizeof(E)) || !aligned(m.cols, p.H * sizeof(unsigned)) ||
      !aligned(y, p.H * sizeof(T)))
    return fail(ISPM_ERR_INVALID, "matrix arrays or y not aligned to H=%u elements", p.H);
  if constexpr (std::is_same<T, float>::value) {
    StageInfo si;
    if (!ln && staged_shape(ISPM_F32, p, m, x, si, a.st_slots, a.st_slot_bytes, a.st_x_off))
      return launch_staged<E>(a, si, s);
  }
  switch (p.H) {
  case 1: return launch_h<T, E, 1>(a, m, p.N, s, ln != nullptr);
  case 2: return launch_h<T, E, 2>(a, m, p.N, s, ln != nullptr);
  case 4: return launch_h<T, E, 4>(a, m, p.N, s, ln != nullptr);
  case 8:
    // eight rows a thread: FP32 vectors, one column per stored index
    if constexpr (std::is_same<T, float>::value) {
      if (ln || m.hblock != 1)
        return fail(ISPM_ERR_INVALID, "H = 8 needs hblock 1 and a single system");
      const bool V = m.var_height != 0, D = m.diags != 0;
      if (V)
        return D ? launch_one<T, E, 8, 1, true, true>(a, p.N, s)
                 : launch_one<T, E, 8, 1, true, false>(a, p.N, s);
      return D ? launch_one<T, E, 8, 1, false, true>(a, p.N, s)
               : launch_one<T, E, 8, 1, false, false>(a, p.N, s);
    }
    return fail(ISPM_ERR_INVALID, "H = 8 needs FP32 vectors");
  }
  return fail(ISPM_ERR_INVALID, "H %u", p.H);
}

}  // namespace

int check_launch(int x_dtype, const ispm_launch_params &p, const ispm_slell_view &m)
{
  const int e = m.elm_dtype;
  if (!((x_dtype == ISPM_F32 && e == ISPM_F32) || (x_dtype == ISPM_F64 && e == ISPM_F32) ||
        (x_dtype == ISPM_F64 && e == ISPM_F64) || (x_dtype == ISPM_F32 && e == ISPM_BF16) ||
        (x_dtype == ISPM_F32 && e == ISPM_F16)))
    return fail(ISPM_ERR_INVALID, "(T, E) = (%s, %s) is not an instantiated pair",
                x_dtype == ISPM_F64 ? "double" : "float",
                e == ISPM_F64   ? "double"
                : e == ISPM_F32 ? "float"
                : e == ISPM_F16 ? "half"
                                : "bfloat16");
  if (!is_pow2(p.N) || p.N < 4 || p.N > 1024)
    return fail(ISPM_ERR_INVALID, "N = %u (power of two in [4, 1024])", p.N);
  if (p.H != 1 && p.H != 2 && p.H != 4 && p.H != 8)
    return fail(ISPM_ERR_INVALID, "H = %u (1, 2, 4, or 8 with FP32 vectors)", p.H);
  if (p.H == 8 && (x_dtype != ISPM_F32 || m.hblock != 1))
    return fail(ISPM_ERR_INVALID, "H = 8 needs FP32 vectors and hblock 1");
  if (!(p.N >= p.S / p.H && p.S >= p.H))
    return fail(ISPM_ERR_INVALID, "launch params fail N >= S/H && S >= H");
  if (m.hblock != 1 && m.hblock != 2 && m.hblock != 4)
    return fail(ISPM_ERR_INVALID, "hblock %u", m.hblock);
  if (m.diags && m.hblock > 1)
    return fail(ISPM_ERR_INVALID, "diagonal blocks with hblock > 1");
  if (m.n_slices == 0)
    return ISPM_OK;
  if (!m.var_height) {
    if (p.S != m.slice_height)
      return fail(ISPM_ERR_INVALID, "S = %u but the matrix slice height is %u", p.S,
                  m.slice_height);
    if (!is_pow2(m.slice_height))
      return fail(ISPM_ERR_INVALID, "slice height %u is not a power of two", m.slice_height);
  } else {
    if (!is_pow2(m.min_slice_height) || !is_pow2(m.max_slice_height))
      return fail(ISPM_ERR_INVALID, "variable slice heights must be powers of two");
    if (m.min_slice_height < p.H)
      return fail(ISPM_ERR_INVALID, "H = %u exceeds the shortest slice (%u rows)", p.H,
                  m.min_slice_height);
    if ((unsigned long long)p.N * p.H < m.max_slice_height)
      return fail(ISPM_ERR_INVALID, "N*H = %u below the tallest slice (%u rows)", p.N * p.H,
                  m.max_slice_height);
  }
  return ISPM_OK;
}

unsigned spmv_cta_rows(const ispm_launch_params &p, const ispm_slell_view &m)
{
  const unsigned block = p.N >= 256 ? p.N : 256;
  return block / p.N * m.slice_height;
}

int launch_spmv_lanes(int x_dtype, const ispm_launch_params &p, const ispm_slell_view &m,
                      const void *x, void *y, cudaStream_t s, const SpmvLanes &lanes)
{
  int st = check_launch(x_dtype, p, m);
  if (st)
    return st;
  if (m.n_slices == 0)
    return ISPM_OK;
  if (!x || !y || !m.slice_ptr || (m.n_elms && (!m.elms)) || (m.n_cols_arr && !m.cols) ||
      !lanes.tile_lane || !lanes.done || !lanes.vt)
    return fail(ISPM_ERR_INVALID, "NULL pointer");
  if (lanes.out && (!lanes.v || !lanes.part || !lanes.ticket || !lanes.cta_beg ||
                    !lanes.cta_cnt || !lanes.lane_tile0))
    return fail(ISPM_ERR_INVALID, "lane dot without its buffers");
  if (m.var_height || 1024u % spmv_cta_rows(p, m) != 0)
    return fail(ISPM_ERR_INVALID, "a CTA of this launch does not fit one 1024-row tile");
  if (x_dtype != m.elm_dtype)
    return fail(ISPM_ERR_INVALID, "lane-segmented SpMV needs equal vector and element types");
  if (x_dtype == ISPM_F32)
    return launch_te<float, float>(p, m, x, y, s, nullptr, nullptr, &lanes);
  return launch_te<double, double>(p, m, x, y, s, nullptr, nullptr, &lanes);
}

unsigned spmv_grid(const ispm_launch_params &p, const ispm_slell_view &m)
{
  const unsigned block = p.N >= 256 ? p.N : 256;
  const unsigned spb = block / p.N;
  return (m.n_slices + spb - 1) / spb;
}

int launch_spmv(int x_dtype, const ispm_launch_params &p, const ispm_slell_view &m,
                const void *x, void *y, cudaStream_t s, const int *skip, const SpmvDot *ep,
                bool pdl, const SpmvSplit *split)
{
  if (split && m.elm_dtype != ISPM_F16)
    return fail(ISPM_ERR_INVALID, "a split diagonal goes with FP16 elements");
  int st = check_launch(x_dtype, p, m);
  if (st)
    return st;
  if (m.n_slices == 0) {
    if (ep && ep->out) {
      cudaError_t e = cudaMemsetAsync(ep->out, 0, sizeof(double), s);
      if (e != cudaSuccess)
        return fail(ISPM_ERR_CUDA, "memset: %s", cudaGetErrorString(e));
    }
    return ISPM_OK;
  }
  if (!x || !y || !m.slice_ptr || (m.n_elms && (!m.elms)) || (m.n_cols_arr && !m.cols))
    return fail(ISPM_ERR_INVALID, "NULL pointer");
  if (x_dtype == ISPM_F32 && m.elm_dtype == ISPM_BF16)
    return launch_te<float, __nv_bfloat16>(p, m, x, y, s, skip, ep, nullptr, pdl);
  if (x_dtype == ISPM_F32 && m.elm_dtype == ISPM_F16)
    return launch_te<float, __half>(p, m, x, y, s, skip, ep, nullptr, pdl, split);
  if (x_dtype == ISPM_F32)
    return launch_te<float, float>(p, m, x, y, s, skip, ep, nullptr, pdl);
  if (m.elm_dtype == ISPM_F32)
    return launch_te<double, float>(p, m, x, y, s, skip, ep, nullptr, pdl);
  return launch_te<double, double>(p, m, x, y, s, skip, ep, nullptr, pdl);
}

}  // namespace ispm

extern "C" {

int ispm_launch_params_valid(const ispm_launch_params *p)
{
  return p && p->H && p->N >= p->S / p->H && p->S >= p->H;
}

int ispm_launch_spmv(int x_dtype, const ispm_launch_params *p, const ispm_slell_view *m,
                     const void *x, void *y, void *stream)
{
  ispm::clear_error();
  if (!p || !m)
    return ispm::fail(ISPM_ERR_INVALID, "NULL params or matrix");
  return ispm::launch_spmv(x_dtype, *p, *m, x, y, (cudaStream_t)stream);
}

int ispm_launch_spmv_split(const ispm_launch_params *p, const ispm_slell_view *m,
                           const float *diag, float inv_scale, const float *x, float *y,
                           void *stream)
{
  ispm::clear_error();
  if (!p || !m)
    return ispm::fail(ISPM_ERR_INVALID, "NULL params or matrix");
  if (m->elm_dtype != ISPM_F16)
    return ispm::fail(ISPM_ERR_INVALID, "the split product takes FP16 elements");
  ispm::SpmvSplit sp{diag, inv_scale};
  return ispm::launch_spmv(ISPM_F32, *p, *m, x, y, (cudaStream_t)stream, nullptr, nullptr,
                           false, &sp);
}

int ispm_spmv_stage_fault(int *code)
{
  ispm::clear_error();
  if (!code)
    return ispm::fail(ISPM_ERR_INVALID, "NULL code");
  unsigned v = 0;
  const unsigned zero = 0;
  ISPM_CUDA_TRY(cudaMemcpyFromSymbol(&v, ispm::g_stage_fault, sizeof v));
  ISPM_CUDA_TRY(cudaMemcpyToSymbol(ispm::g_stage_fault, &zero, sizeof zero));
  *code = (int)v;
  return ISPM_OK;
}

}  // extern "C"
