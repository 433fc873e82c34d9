/* Drop-in for util/cuda/cudamemcpy.h (reference util/cuda/cudamemcpy.h:1-48):
 * copy / copy_async of n elements, the direction taken from the pointer
 * types (devmem<T> * is device memory, T * host memory). */
#ifndef ISPM_CUDA_MEMCPY_H
#define ISPM_CUDA_MEMCPY_H

#include <cuda_runtime.h>

#include "check.h"
#include "devmem.h"

namespace ispm_compat {
template <class T> inline cudaMemcpyKind direction(devmem<T> *, const devmem<T> *)
{
  return cudaMemcpyDeviceToDevice;
}
template <class T> inline cudaMemcpyKind direction(devmem<T> *, const T *)
{
  return cudaMemcpyHostToDevice;
}
template <class T> inline cudaMemcpyKind direction(T *, const devmem<T> *)
{
  return cudaMemcpyDeviceToHost;
}
}  // namespace ispm_compat

template <typename T, typename S> static inline void copy(T *dst, const S *src, size_t n_elts)
{
  if (n_elts)
    CUDA_CHECK(cudaMemcpy(dst, src, n_elts * sizeof(T), ispm_compat::direction(dst, src)));
}

template <typename T, typename S>
static inline void copy_async(T *dst, const S *src, size_t n_elts)
{
  if (n_elts)
    CUDA_CHECK(
        cudaMemcpyAsync(dst, src, n_elts * sizeof(T), ispm_compat::direction(dst, src)));
}

#endif
