// Internal SpMV launch interface (used by the C ABI, the plan and the solver).
#ifndef ISPM_SPMV_LAUNCH_H
#define ISPM_SPMV_LAUNCH_H

#include <cuda_runtime.h>

#include "ispm_internal.h"

namespace ispm {

// Validate launch parameters against a matrix (no CUDA calls).
int check_launch(int x_dtype, const ispm_launch_params &p, const ispm_slell_view &m);
// Optional fused epilogue of an SpMV: *out = sum_i y_i v_i in FP64 over the
// rows the launch writes (v has the vector type T).  part holds one partial
// per CTA (part_capacity slots), ticket is a zero-initialised arrival counter
// the launch leaves at zero.
struct SpmvDot {
  const void *v = nullptr;
  double *out = nullptr;
  double *part = nullptr;
  unsigned *ticket = nullptr;
  unsigned part_capacity = 0;
};

// Validate and launch y = A x on `s`.  `skip` (device int, may be NULL): the
// kernel returns at once when it holds a nonzero value.
int launch_spmv(int x_dtype, const ispm_launch_params &p, const ispm_slell_view &m,
                const void *x, void *y, cudaStream_t s, const int *skip = nullptr,
                const SpmvDot *ep = nullptr);
// CTAs a launch of matrix m with params p uses (partials a fused dot needs).
unsigned spmv_grid(const ispm_launch_params &p, const ispm_slell_view &m);

// Device-resident sliced-ELL matrix.
struct DeviceSlell {
  ispm_slell_view meta{};  // host copy of the metadata; pointers are device pointers
  unsigned *slice_ptr = nullptr;
  unsigned *cols = nullptr;
  void *elms = nullptr;
  ispm_slell_view view() const
  {
    ispm_slell_view v = meta;
    v.slice_ptr = slice_ptr;
    v.cols = cols;
    v.elms = elms;
    return v;
  }
  int upload(const HostSlell &h);
  int update_elms(const HostSlell &h);
  void release();
  ~DeviceSlell() { release(); }
};

// B200 launch heuristic for a matrix: threads per slice and rows per thread.
ispm_launch_params default_launch(int x_dtype, const ispm_slell_view &m);

// d.elms[map[k]] = vals[k] for k < n (device arrays; vals FP32 or FP64).
int refresh_values(DeviceSlell &d, const unsigned *map, const void *vals, int val_dtype,
                   long long n, cudaStream_t s);

}  // namespace ispm

struct ispm_dslell {
  ispm::DeviceSlell d;
};

#endif
