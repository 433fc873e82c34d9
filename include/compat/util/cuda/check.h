/* Drop-in for util/cuda/check.h (reference util/cuda/check.h:1-17):
 * CUDA_CHECK(call) prints the CUDA error and aborts. */
#ifndef CUDA_CHECK_H
#define CUDA_CHECK_H

#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>

static inline void report_cuda_error(cudaError_t err)
{
  fprintf(stderr, "CUDA error %x: %s\n", (unsigned)err, cudaGetErrorString(err));
  abort();
}

#define CUDA_CHECK(x)                                                                       \
  do {                                                                                      \
    cudaError_t e_ = (x);                                                                   \
    if (e_ != cudaSuccess)                                                                  \
      report_cuda_error(e_);                                                                \
  } while (0)

#endif
