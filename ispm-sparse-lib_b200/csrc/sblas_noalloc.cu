// ispm_sblas_dot_noalloc: the dot product without any device allocation.
//
// ispm_sblas_dot keeps its per-CTA partial sums in a per-device scratch area
// it cudaMalloc's on first use.  Some callers cannot have the library allocate:
// an application that reserves (nearly) all device memory up front for its own
// pool, a solver loop that must not hit the implicit device synchronisation
// cudaMalloc / cudaFree can cause, or code that has to keep a fixed, known
// device footprint.  This variant takes its scratch from a file-scope
// __device__ array that is part of the loaded library instead: 1024 partial
// sums plus an arrival counter, 8 KB + 8 bytes, held by every GPU that loads
// the library until the process exits.
//
// Limits and sharing:
//  * a launch uses at most 4 CTAs per SM and never more than 1024 CTAs (the
//    grid cap every sblas reduction shares), one partial slot each, so the
//    1024 slots always suffice: a device with more than 256 SMs runs the dot
//    with 1024 CTAs (the B200 uses 592);
//  * every call shares the one array: calls whose work overlaps on the GPU
//    (different streams or host threads) race on it and give wrong results;
//  * the arrival counter is cleared (cudaMemsetAsync on the caller's stream)
//    before every launch, so a call never depends on what an earlier call
//    left behind;
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (once per device, under a lock); make that first call
//    before capturing any stream.
#include <cuda_runtime.h>

#include <mutex>

#include "cuda_util.cuh"
#include "sblas_impl.h"

namespace {

constexpr int kNoAllocSlots = 1024;
static_assert(kNoAllocSlots >= ispm::kSblasMaxBlocks,
              "the static scratch must hold a partial for every CTA sblas_grid allows");

// Slots 0 .. kNoAllocSlots-1: per-CTA partial sums (doubles); the last word
// holds the arrival counter.
static __device__ __align__(256) unsigned long long g_dot_scratch[kNoAllocSlots + 1];

std::mutex g_mu;
unsigned long long *g_addr[64] = {};

// Device address of g_dot_scratch on the current device (set-up on first use).
int scratch_address(unsigned long long **out)
{
  int dev = 0;
  ISPM_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64)
    return ispm::fail(ISPM_ERR_INVALID, "device ordinal %d", dev);
  std::lock_guard<std::mutex> g(g_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_dot_scratch);
    if (e != cudaSuccess)
      return ispm::fail(ISPM_ERR_CUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    g_addr[dev] = static_cast<unsigned long long *>(p);
  }
  *out = g_addr[dev];
  return ISPM_OK;
}

}  // namespace

extern "C" {

int ispm_sblas_dot_noalloc(int dtype, const void *x, const void *y, void *s, int n,
                           void *stream)
{
  using namespace ispm;
  clear_error();
  if (dtype != ISPM_F32 && dtype != ISPM_F64)
    return fail(ISPM_ERR_INVALID, "dtype %d", dtype);
  if (n < 0 || !s || (n && (!x || !y)))
    return fail(ISPM_ERR_INVALID, "bad arguments");
  // dot_launch sizes its grid with sblas_grid, which never exceeds
  // kSblasMaxBlocks <= kNoAllocSlots (static_assert above)
  unsigned long long *base = nullptr;
  if (int st = scratch_address(&base))
    return st;
  double *part = reinterpret_cast<double *>(base);
  unsigned *ticket = reinterpret_cast<unsigned *>(base + kNoAllocSlots);
  cudaStream_t st = (cudaStream_t)stream;
  ISPM_CUDA_TRY(cudaMemsetAsync(ticket, 0, sizeof(unsigned), st));
  if (dtype == ISPM_F32)
    return dot_launch<float>((const float *)x, (const float *)y, (float *)s, n, part, ticket,
                             st);
  return dot_launch<double>((const double *)x, (const double *)y, (double *)s, n, part, ticket,
                            st);
}

}  // extern "C"
