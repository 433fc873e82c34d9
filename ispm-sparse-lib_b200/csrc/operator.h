// Solver operators: a CSR matrix held on the device as sliced-ELL in the
// shape that needs the fewest bytes among a few candidates.
#ifndef ISPM_OPERATOR_H
#define ISPM_OPERATOR_H

#include <cuda_runtime.h>

#include <memory>
#include <vector>

#include "spmv_launch.h"

namespace ispm {

// Sliced-ELL shape with the fewest stored bytes (slice_ptr + cols + elms)
// for this CSR among the reference's guess and S in {32, 64, 128} with and
// without diagonal blocks, plus S = 64 with hblock 2.  (The guess samples
// only the first 1% of rows, which misjudges matrices whose first rows are
// atypical, e.g. the FSAI factors, whose first rows are the shortest.)
// fixed_height: variable-height shapes are not candidates.  The matrix may
// be rectangular (a band of rows of a larger matrix).
int choose_format(int elm_dtype, int n_rows, int n_cols, const int *rp, const int *ci,
                  const double *v, bool fixed_height, ispm_slell_params &out,
                  size_t *out_bytes = nullptr);
// The shape Operator::upload picks for an n x n operator without a forced
// shape (fewest stored bytes, short slices weighted up).
int choose_operator_shape(int elm_dtype, int n, const int *rp, const int *ci, const double *v,
                          ispm_slell_params &out);

// IEEE binary16 of v, rounded to nearest even (subnormals kept); |v| must be
// below 65520 (the binary16 overflow threshold).
uint16_t f16_bits(double v);
// The value of a binary16 bit pattern (finite patterns only).
double f16_value(uint16_t h);
// The FP16 split of a square CSR (ispm_csr_split_f16).
int split_f16(int n, const int *rp, const int *ci, const double *v, uint16_t *off, float *diag,
              float &scale);

struct Operator {
  DeviceSlell dev;
  ispm_launch_params lp{};
  ispm_slell_params fmt{};
  // FP16 elements hold the values times 1 / inv_scale.  Split operators
  // (upload_split_f16) add this FP32 diagonal (device, dev.meta.n_rows
  // entries, owned by diag_mem); FP16-stored factors have none.
  std::shared_ptr<float> diag_mem;
  float *diag = nullptr;
  float inv_scale = 1.f;

  // Convert (n x n CSR, FP64 values stored as elm_dtype) and upload in the
  // min-bytes shape, or in `force`.  value_pos: CSR entry -> element slot,
  // for values computed later on the device.
  // bf16_values: keep the FP32 elements as BF16 on the device.
  // f16_values: FP16 element storage for values written later on the device
  // (set_f16_values); the uploaded values must be exact binary16 values
  // (the solver passes zeros).
  int upload(int vec_dtype, int elm_dtype, int n, const int *rp, const int *ci,
             const double *v, const ispm_slell_params *force = nullptr,
             std::vector<unsigned> *value_pos = nullptr, bool fixed_height = false,
             bool bf16_values = false, bool f16_values = false);
  // Upload the FP16 split of an n x n FP64 CSR (split_f16): the off-diagonal
  // entries in the min-bytes sliced-ELL shape with FP16 elements, the
  // corrected diagonal as an FP32 vector.  FP32 vectors only.
  int upload_split_f16(int n, const int *rp, const int *ci, const double *v);
  int apply(int vdt, const void *x, void *y, cudaStream_t s, const int *skip,
            const SpmvDot *ep = nullptr, bool pdl = false) const
  {
    if (dev.meta.elm_dtype == ISPM_F16) {
      SpmvSplit sp{diag, inv_scale};
      return launch_spmv(vdt, lp, dev.view(), x, y, s, skip, ep, pdl, &sp);
    }
    return launch_spmv(vdt, lp, dev.view(), x, y, s, skip, ep, pdl);
  }
  int apply_lanes(int vdt, const void *x, void *y, cudaStream_t s, const SpmvLanes &ln) const
  {
    return launch_spmv_lanes(vdt, lp, dev.view(), x, y, s, ln);
  }
  unsigned grid() const { return spmv_grid(lp, dev.view()); }
  unsigned cta_rows() const { return spmv_cta_rows(lp, dev.view()); }
  // Bytes of the stored matrix (slice_ptr + cols + elms).
  size_t bytes() const;
};

}  // namespace ispm

#endif
