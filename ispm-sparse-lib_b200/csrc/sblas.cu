// BLAS-1 and pipelined-CG vector fusions (util/cuda/sblas.cu).
//
// Differences from the reference, all B200-motivated:
//  * reductions accumulate in FP64 whatever the vector type, and the
//    cross-block finish happens in the same launch: every CTA publishes its
//    partial, the last CTA to arrive (atomic ticket) adds the partials in
//    block order, so results are deterministic for a given size, and a dot
//    or an update is one launch instead of two;
//  * grid sizes follow the SM count, vectors move in 128-bit words when
//    every pointer is 16-byte aligned;
//  * the recurrences are written as explicit fma() calls, the contraction
//    nvcc applies to the reference's expressions by default.
#include <cuda_runtime.h>

#include <mutex>

#include "cuda_util.cuh"
#include "sblas_impl.h"

namespace ispm {

namespace {

constexpr int kThreads = 256;

struct ScratchSlot {
  double *part = nullptr;
  unsigned *ticket = nullptr;
};

std::mutex g_scratch_mu;
ScratchSlot g_scratch[64];

}  // namespace

int sblas_scratch(double **part, unsigned **ticket)
{
  int dev = 0;
  ISPM_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64)
    return fail(ISPM_ERR_INVALID, "device ordinal %d", dev);
  std::lock_guard<std::mutex> g(g_scratch_mu);
  ScratchSlot &s = g_scratch[dev];
  if (!s.part) {
    void *p = nullptr;
    size_t bytes = sizeof(double) * 3 * kSblasMaxBlocks + 256;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(ISPM_ERR_NOMEM, "sblas scratch: %s", cudaGetErrorString(e));
    }
    e = cudaMemset(p, 0, bytes);
    if (e != cudaSuccess) {
      cudaFree(p);
      return fail(ISPM_ERR_CUDA, "sblas scratch memset: %s", cudaGetErrorString(e));
    }
    s.part = (double *)p;
    s.ticket = (unsigned *)((char *)p + sizeof(double) * 3 * kSblasMaxBlocks);
  }
  *part = s.part;
  *ticket = s.ticket;
  return ISPM_OK;
}

int sblas_grid(long long n, int vec)
{
  long long units = (n + vec - 1) / vec;
  long long blocks = (units + kThreads - 1) / kThreads;
  long long cap = (long long)device_sm_count() * 4;
  if (cap > kSblasMaxBlocks)
    cap = kSblasMaxBlocks;
  if (blocks > cap)
    blocks = cap;
  return blocks < 1 ? 1 : (int)blocks;
}

namespace {

template <int NV> struct Acc {
  double v[NV];
};

// Block-wide sum of NV doubles; the result is valid in thread 0.
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

// Publish this block's NV partials; returns true in the last block to
// arrive, whose thread 0 then holds the block-ordered totals in `tot`.
template <int NV>
__device__ __forceinline__ bool finish_grid(Acc<NV> a, double *part, unsigned *ticket,
                                            Acc<NV> &tot)
{
  __shared__ bool last;
  a = block_sum<NV>(a);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++)
      part[k * kSblasMaxBlocks + blockIdx.x] = a.v[k];
    __threadfence();
    unsigned arrived = atomicAdd(ticket, 1u);
    last = arrived == gridDim.x - 1;
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
      s.v[k] += __ldcg(part + k * kSblasMaxBlocks + b);
  }
  tot = block_sum<NV>(s);
  if (threadIdx.x == 0)
    *ticket = 0u;
  return true;
}

template <class T> struct V16;
template <> struct V16<float> {
  using type = float4;
  static constexpr int n = 4;
};
template <> struct V16<double> {
  using type = double2;
  static constexpr int n = 2;
};

template <class T> __device__ __forceinline__ T get(const typename V16<T>::type &v, int k)
{
  return reinterpret_cast<const T *>(&v)[k];
}

template <class T>
__global__ void __launch_bounds__(kThreads)
    dot_kernel(const T *__restrict__ x, const T *__restrict__ y, T *out, long long n, int vec,
               double *part, unsigned *ticket)
{
  Acc<1> a{{0.0}};
  const long long stride = (long long)gridDim.x * blockDim.x;
  long long i0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long done = 0;
  if (vec) {
    using VT = typename V16<T>::type;
    constexpr int W = V16<T>::n;
    const long long nv = n / W;
    const VT *xv = reinterpret_cast<const VT *>(x), *yv = reinterpret_cast<const VT *>(y);
    for (long long i = i0; i < nv; i += stride) {
      VT p = __ldcs(xv + i), q = __ldcs(yv + i);
#pragma unroll
      for (int k = 0; k < W; k++)
        a.v[0] = fma((double)get<T>(p, k), (double)get<T>(q, k), a.v[0]);
    }
    done = nv * W;
  }
  for (long long i = done + i0; i < n; i += stride)
    a.v[0] = fma((double)x[i], (double)y[i], a.v[0]);
  Acc<1> tot;
  if (finish_grid<1>(a, part, ticket, tot) && threadIdx.x == 0)
    *out = (T)tot.v[0];
}

template <class T>
__global__ void scalars_kernel(T *alpha, T *beta, const T *gamma, const T *gammaold,
                               const T *delta)
{
  // sblas.cu:156-165
  T g = *gamma;
  T b = g / *gammaold;
  *beta = b;
  *alpha = g / (*delta - b * g / *alpha);
}

template <class T>
__device__ __forceinline__ void ppcg_elem(T a, T b, T nv, T mv, T &p, T &s, T &q, T &z, T &x,
                                          T &r, T &u, T &w, Acc<3> &acc)
{
  // sblas.cu:193-203 with nvcc's default contraction spelled out
  T zi = fma(b, z, nv);
  T qi = fma(b, q, mv);
  T si = fma(b, s, w);
  T pi = fma(b, p, u);
  T ui = fma(-a, qi, u);
  T wi = fma(-a, zi, w);
  T ri = fma(-a, si, r);
  x = fma(a, pi, x);
  z = zi;
  q = qi;
  s = si;
  p = pi;
  u = ui;
  w = wi;
  r = ri;
  acc.v[0] += fabs((double)ri);
  acc.v[1] = fma((double)ri, (double)ui, acc.v[1]);
  acc.v[2] = fma((double)wi, (double)ui, acc.v[2]);
}

template <class T>
__global__ void __launch_bounds__(kThreads) ppcg_vectors_kernel(PpcgVecArgs<T> g)
{
  const T a = *g.alpha, b = *g.beta;
  Acc<3> acc{{0.0, 0.0, 0.0}};
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long i0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long done = 0;
  if (g.vec) {
    using VT = typename V16<T>::type;
    constexpr int W = V16<T>::n;
    const long long nv = g.n_elts / W;
    for (long long i = i0; i < nv; i += stride) {
      VT nn = __ldcs(reinterpret_cast<const VT *>(g.n) + i);
      VT mm = __ldcs(reinterpret_cast<const VT *>(g.m) + i);
      VT pp = reinterpret_cast<const VT *>(g.p)[i], ss = reinterpret_cast<const VT *>(g.s)[i];
      VT qq = reinterpret_cast<const VT *>(g.q)[i], zz = reinterpret_cast<const VT *>(g.z)[i];
      VT xx = reinterpret_cast<const VT *>(g.x)[i], rr = reinterpret_cast<const VT *>(g.r)[i];
      VT uu = reinterpret_cast<const VT *>(g.u)[i], ww = reinterpret_cast<const VT *>(g.w)[i];
      T *P = reinterpret_cast<T *>(&pp), *S = reinterpret_cast<T *>(&ss);
      T *Q = reinterpret_cast<T *>(&qq), *Z = reinterpret_cast<T *>(&zz);
      T *X = reinterpret_cast<T *>(&xx), *Rr = reinterpret_cast<T *>(&rr);
      T *U = reinterpret_cast<T *>(&uu), *Wv = reinterpret_cast<T *>(&ww);
#pragma unroll
      for (int k = 0; k < W; k++)
        ppcg_elem<T>(a, b, get<T>(nn, k), get<T>(mm, k), P[k], S[k], Q[k], Z[k], X[k], Rr[k],
                     U[k], Wv[k], acc);
      reinterpret_cast<VT *>(g.p)[i] = pp;
      reinterpret_cast<VT *>(g.s)[i] = ss;
      reinterpret_cast<VT *>(g.q)[i] = qq;
      reinterpret_cast<VT *>(g.z)[i] = zz;
      reinterpret_cast<VT *>(g.x)[i] = xx;
      reinterpret_cast<VT *>(g.r)[i] = rr;
      reinterpret_cast<VT *>(g.u)[i] = uu;
      reinterpret_cast<VT *>(g.w)[i] = ww;
    }
    done = nv * W;
  }
  for (long long i = done + i0; i < g.n_elts; i += stride)
    ppcg_elem<T>(a, b, g.n[i], g.m[i], g.p[i], g.s[i], g.q[i], g.z[i], g.x[i], g.r[i], g.u[i],
                 g.w[i], acc);
  Acc<3> tot;
  if (finish_grid<3>(acc, g.part, g.ticket, tot) && threadIdx.x == 0) {
    *g.resnorm = (T)tot.v[0];
    *g.gamma = (T)tot.v[1];
    *g.delta = (T)tot.v[2];
  }
}

template <class T>
__global__ void copy_indexed_kernel(T *dst, const T *src, const int *idx, int n)
{
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n)
    dst[k] = src[idx[k]];
}

template <class T>
__global__ void add_indexed_kernel(T *dst, const T *src, const int *idx, int n)
{
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n)
    atomicAdd(dst + idx[k], src[k]);
}

}  // namespace

template <class T>
int dot_launch(const T *x, const T *y, T *s, long long n, double *part, unsigned *ticket,
               cudaStream_t st)
{
  const int vec = aligned(x, 16) && aligned(y, 16);
  const int grid = sblas_grid(n, vec ? 16 / (int)sizeof(T) : 1);
  dot_kernel<T><<<grid, kThreads, 0, st>>>(x, y, s, n, vec, part, ticket);
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess)
    return fail(ISPM_ERR_CUDA, "dot launch: %s", cudaGetErrorString(e));
  return ISPM_OK;
}

template <class T> int ppcg_vectors_launch(PpcgVecArgs<T> g, cudaStream_t st)
{
  g.vec = aligned(g.n, 16) && aligned(g.m, 16) && aligned(g.p, 16) && aligned(g.s, 16) &&
          aligned(g.q, 16) && aligned(g.z, 16) && aligned(g.x, 16) && aligned(g.r, 16) &&
          aligned(g.u, 16) && aligned(g.w, 16);
  const int grid = sblas_grid(g.n_elts, g.vec ? 16 / (int)sizeof(T) : 1);
  ppcg_vectors_kernel<T><<<grid, kThreads, 0, st>>>(g);
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess)
    return fail(ISPM_ERR_CUDA, "ppcg_update_vectors launch: %s", cudaGetErrorString(e));
  return ISPM_OK;
}

template int dot_launch<float>(const float *, const float *, float *, long long, double *,
                               unsigned *, cudaStream_t);
template int dot_launch<double>(const double *, const double *, double *, long long, double *,
                                unsigned *, cudaStream_t);
template int ppcg_vectors_launch<float>(PpcgVecArgs<float>, cudaStream_t);
template int ppcg_vectors_launch<double>(PpcgVecArgs<double>, cudaStream_t);

}  // namespace ispm

using namespace ispm;

namespace {

int check_dtype(int dtype)
{
  if (dtype != ISPM_F32 && dtype != ISPM_F64)
    return fail(ISPM_ERR_INVALID, "dtype %d", dtype);
  return ISPM_OK;
}

int launch_status(const char *what)
{
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess)
    return fail(ISPM_ERR_CUDA, "%s launch: %s", what, cudaGetErrorString(e));
  return ISPM_OK;
}

}  // namespace

extern "C" {

int ispm_sblas_copy_indexed(int dtype, void *dst, const void *src, const int *idx, int n,
                            void *stream)
{
  clear_error();
  if (int st = check_dtype(dtype))
    return st;
  if (n < 0 || (n && (!dst || !src || !idx)))
    return fail(ISPM_ERR_INVALID, "bad arguments");
  if (!n)
    return ISPM_OK;
  const int blocks = (n + kThreads - 1) / kThreads;
  if (dtype == ISPM_F32)
    copy_indexed_kernel<float><<<blocks, kThreads, 0, (cudaStream_t)stream>>>(
        (float *)dst, (const float *)src, idx, n);
  else
    copy_indexed_kernel<double><<<blocks, kThreads, 0, (cudaStream_t)stream>>>(
        (double *)dst, (const double *)src, idx, n);
  return launch_status("copy_indexed");
}

int ispm_sblas_add_indexed(int dtype, void *dst, const void *src, const int *idx, int n,
                           void *stream)
{
  clear_error();
  if (int st = check_dtype(dtype))
    return st;
  if (n < 0 || (n && (!dst || !src || !idx)))
    return fail(ISPM_ERR_INVALID, "bad arguments");
  if (!n)
    return ISPM_OK;
  const int blocks = (n + kThreads - 1) / kThreads;
  if (dtype == ISPM_F32)
    add_indexed_kernel<float><<<blocks, kThreads, 0, (cudaStream_t)stream>>>(
        (float *)dst, (const float *)src, idx, n);
  else
    add_indexed_kernel<double><<<blocks, kThreads, 0, (cudaStream_t)stream>>>(
        (double *)dst, (const double *)src, idx, n);
  return launch_status("add_indexed");
}

int ispm_sblas_dot(int dtype, const void *x, const void *y, void *s, int n, void *stream)
{
  clear_error();
  if (int st = check_dtype(dtype))
    return st;
  if (n < 0 || !s || (n && (!x || !y)))
    return fail(ISPM_ERR_INVALID, "bad arguments");
  double *part;
  unsigned *ticket;
  if (int st = sblas_scratch(&part, &ticket))
    return st;
  if (dtype == ISPM_F32)
    return dot_launch<float>((const float *)x, (const float *)y, (float *)s, n, part, ticket,
                             (cudaStream_t)stream);
  return dot_launch<double>((const double *)x, (const double *)y, (double *)s, n, part, ticket,
                            (cudaStream_t)stream);
}

int ispm_sblas_ppcg_update_scalars(int dtype, void *alpha, void *beta, const void *gamma,
                                   const void *gammaold, const void *delta, void *stream)
{
  clear_error();
  if (int st = check_dtype(dtype))
    return st;
  if (!alpha || !beta || !gamma || !gammaold || !delta)
    return fail(ISPM_ERR_INVALID, "NULL scalar");
  if (dtype == ISPM_F32)
    scalars_kernel<float><<<1, 1, 0, (cudaStream_t)stream>>>(
        (float *)alpha, (float *)beta, (const float *)gamma, (const float *)gammaold,
        (const float *)delta);
  else
    scalars_kernel<double><<<1, 1, 0, (cudaStream_t)stream>>>(
        (double *)alpha, (double *)beta, (const double *)gamma, (const double *)gammaold,
        (const double *)delta);
  return launch_status("ppcg_update_scalars");
}

int ispm_sblas_ppcg_update_vectors(int dtype, void *resnorm, void *gamma, void *delta,
                                   const void *alpha, const void *beta, const void *n,
                                   const void *m, void *p, void *s, void *q, void *z, void *x,
                                   void *r, void *u, void *w, int n_elts, void *stream)
{
  clear_error();
  if (int st = check_dtype(dtype))
    return st;
  if (n_elts < 0 || !resnorm || !gamma || !delta || !alpha || !beta)
    return fail(ISPM_ERR_INVALID, "bad arguments");
  if (n_elts && (!n || !m || !p || !s || !q || !z || !x || !r || !u || !w))
    return fail(ISPM_ERR_INVALID, "NULL vector");
  double *part;
  unsigned *ticket;
  if (int st = sblas_scratch(&part, &ticket))
    return st;
  if (dtype == ISPM_F32) {
    PpcgVecArgs<float> g{(float *)resnorm, (float *)gamma, (float *)delta, (const float *)alpha,
                         (const float *)beta, (const float *)n, (const float *)m, (float *)p,
                         (float *)s, (float *)q, (float *)z, (float *)x, (float *)r, (float *)u,
                         (float *)w, n_elts, 0, part, ticket};
    return ppcg_vectors_launch<float>(g, (cudaStream_t)stream);
  }
  PpcgVecArgs<double> g{(double *)resnorm, (double *)gamma, (double *)delta,
                        (const double *)alpha, (const double *)beta, (const double *)n,
                        (const double *)m, (double *)p, (double *)s, (double *)q, (double *)z,
                        (double *)x, (double *)r, (double *)u, (double *)w, n_elts, 0, part,
                        ticket};
  return ppcg_vectors_launch<double>(g, (cudaStream_t)stream);
}

}  // extern "C"
