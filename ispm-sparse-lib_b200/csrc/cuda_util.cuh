// CUDA helpers shared by the library's .cu files (sm_100a only).
#ifndef ISPM_CUDA_UTIL_CUH
#define ISPM_CUDA_UTIL_CUH

#include <cuda_runtime.h>

#include <cstdint>

#include "ispm_internal.h"

#define ISPM_CUDA_TRY(call)                                                                 \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      return ::ispm::fail(ISPM_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_),   \
                          __FILE__, __LINE__);                                              \
  } while (0)

namespace ispm {

inline bool aligned(const void *p, size_t a) { return ((uintptr_t)p & (a - 1)) == 0; }
inline bool is_pow2(unsigned v) { return v && !(v & (v - 1)); }
inline int ilog2(unsigned v) { return 31 - __builtin_clz(v); }

int device_sm_count();

// ---- device-side load helpers --------------------------------------------

// Streaming (evict-first) loads for matrix data read exactly once per SpMV.
template <int N, class V> struct Vec {
  V v[N];
};

template <int N, class V> __device__ __forceinline__ Vec<N, V> ld_stream(const V *p)
{
  Vec<N, V> r;
  constexpr int bytes = N * (int)sizeof(V);
  if constexpr (bytes == 2) {
    *reinterpret_cast<unsigned short *>(r.v) = __ldcs(reinterpret_cast<const unsigned short *>(p));
  } else if constexpr (bytes == 4) {
    *reinterpret_cast<unsigned *>(r.v) = __ldcs(reinterpret_cast<const unsigned *>(p));
  } else if constexpr (bytes == 8) {
    uint2 t = __ldcs(reinterpret_cast<const uint2 *>(p));
    *reinterpret_cast<uint2 *>(r.v) = t;
  } else if constexpr (bytes == 16) {
    uint4 t = __ldcs(reinterpret_cast<const uint4 *>(p));
    *reinterpret_cast<uint4 *>(r.v) = t;
  } else {
    static_assert(bytes == 32, "vector width");
    const uint4 *q = reinterpret_cast<const uint4 *>(p);
    uint4 a = __ldcs(q), b = __ldcs(q + 1);
    reinterpret_cast<uint4 *>(r.v)[0] = a;
    reinterpret_cast<uint4 *>(r.v)[1] = b;
  }
  return r;
}

// Programmatic dependent launch.  A kernel launched with the programmatic
// serialization attribute may start while its predecessor on the stream is
// still running: pdl_wait() blocks until the predecessor has completed and
// its writes are visible (a no-op for a kernel launched without the
// attribute), and pdl_trigger() lets the successor be scheduled once every
// block of this kernel has reached it (or exited).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;"); }

// Launch `kernel` on `s`, with the programmatic serialization attribute when
// pdl is set.
template <class... KArgs, class... Args>
cudaError_t launch_kernel(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                          cudaStream_t s, bool pdl, Args &&...args)
{
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = pdl ? attr : nullptr;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<Args &&>(args)...);
}

// Same widths through the read-only path with the default cache policy, for
// matrix data that is read again soon (several lanes sharing one matrix).
template <int N, class V> __device__ __forceinline__ Vec<N, V> ld_keep(const V *p)
{
  Vec<N, V> r;
  constexpr int bytes = N * (int)sizeof(V);
  if constexpr (bytes == 4) {
    *reinterpret_cast<unsigned *>(r.v) = __ldg(reinterpret_cast<const unsigned *>(p));
  } else if constexpr (bytes == 8) {
    *reinterpret_cast<uint2 *>(r.v) = __ldg(reinterpret_cast<const uint2 *>(p));
  } else if constexpr (bytes == 16) {
    *reinterpret_cast<uint4 *>(r.v) = __ldg(reinterpret_cast<const uint4 *>(p));
  } else {
    static_assert(bytes == 32, "vector width");
    const uint4 *q = reinterpret_cast<const uint4 *>(p);
    reinterpret_cast<uint4 *>(r.v)[0] = __ldg(q);
    reinterpret_cast<uint4 *>(r.v)[1] = __ldg(q + 1);
  }
  return r;
}

// Read-only-path load for the gathered vector x (kept in L1/L2).
template <class T> __device__ __forceinline__ T ld_x(const T *x, unsigned i) { return __ldg(x + i); }

template <class T> __device__ __forceinline__ T ld_x_guard(const T *x, unsigned i, unsigned n)
{
  return i < n ? __ldg(x + i) : T(0);
}

template <int N, class T> __device__ __forceinline__ void st_vec(T *p, const T (&v)[N])
{
  constexpr int bytes = N * (int)sizeof(T);
  if constexpr (bytes == 4 || bytes == 8 || bytes == 16) {
    if constexpr (bytes == 4)
      *reinterpret_cast<unsigned *>(p) = *reinterpret_cast<const unsigned *>(v);
    else if constexpr (bytes == 8)
      *reinterpret_cast<uint2 *>(p) = *reinterpret_cast<const uint2 *>(v);
    else
      *reinterpret_cast<uint4 *>(p) = *reinterpret_cast<const uint4 *>(v);
  } else {
    reinterpret_cast<uint4 *>(p)[0] = reinterpret_cast<const uint4 *>(v)[0];
    reinterpret_cast<uint4 *>(p)[1] = reinterpret_cast<const uint4 *>(v)[1];
  }
}

// Block-wide FP64 sum; valid in thread 0.  blockDim.x <= 1024.
__device__ __forceinline__ double block_sum_f64(double v)
{
  __shared__ double sh[32];
  for (int off = 16; off > 0; off >>= 1)
    v += __shfl_down_sync(0xffffffffu, v, off);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0)
    sh[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
    for (int off = 16; off > 0; off >>= 1)
      v += __shfl_down_sync(0xffffffffu, v, off);
  }
  return v;
}

}  // namespace ispm

#endif
