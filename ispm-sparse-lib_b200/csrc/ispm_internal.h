// Internal declarations shared by the library's translation units.
#ifndef ISPM_INTERNAL_H
#define ISPM_INTERNAL_H

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "ispm_b200.h"

namespace ispm {

// Record a failure message for ispm_last_error() and return `status`.
int fail(int status, const char *fmt, ...);
void clear_error();

// Host worker pool size: ISPM_NUM_THREADS, else hardware concurrency.
int host_threads();
// Run fn(lo, hi) over [0, n) split into contiguous chunks on host threads.
template <class F> void parallel_for(long long n, F fn);

// Host sliced-ELL matrix: the reference's slell_matrix<E, host>.
struct HostSlell {
  int n_rows = 0, n_cols = 0, n_nz = 0;
  unsigned slice_height = 0, n_slices = 0, hblock = 1;
  bool var_height = false, diags = false;
  int elm_dtype = ISPM_F64;
  unsigned min_slice_height = 0, max_slice_height = 0;
  int min_height_used = 4;  // min_height the conversion ran with
  std::vector<unsigned> slice_ptr;
  std::vector<unsigned> cols;
  std::vector<float> elms_f;   // used when elm_dtype == ISPM_F32
  std::vector<double> elms_d;  // used when elm_dtype == ISPM_F64
  size_t n_elms() const { return elm_dtype == ISPM_F32 ? elms_f.size() : elms_d.size(); }
  const void *elms_ptr() const
  {
    return elm_dtype == ISPM_F32 ? (const void *)elms_f.data() : (const void *)elms_d.data();
  }
  void *elms_ptr() { return elm_dtype == ISPM_F32 ? (void *)elms_f.data() : (void *)elms_d.data(); }
  ispm_slell_view view() const;
};

// ISPM_ERR_INVALID unless row_ptr[0] == 0, row_ptr never decreases and every
// column index lies in [0, n_cols).
int validate_csr(int n_rows, int n_cols, const int *row_ptr, const int *cols);

// Conversion entry used by the C ABI and the plan.
int convert_csr(int elm_dtype, int n_rows, int n_cols, const int *row_ptr, const int *cols,
                const void *elms, int S, int hblock, bool var_height, bool use_diags,
                int min_height, HostSlell &out);
int guess_format(int elm_dtype, int n_rows, int n_cols, const int *row_ptr, const int *cols,
                 const void *elms, int examine_ratio, int min_height, ispm_slell_params &out);
// pos[k] = element-array position of CSR entry k in m (m converted from a CSR
// with this pattern).
int value_map(const HostSlell &m, int n_rows, const int *row_ptr, const int *cols,
              std::vector<unsigned> &pos);

// Reverse Cuthill-McKee order of a symmetric pattern: perm[new] = old.
void rcm_order(int n, const int *rp, const int *ci, std::vector<int> &perm);
// max |j - i| over the entries (of P A P^T when inv, inv[old] = new, is given).
long long bandwidth(int n, const int *rp, const int *ci, const int *inv);
// P A P^T as a CSR with sorted columns (perm[new] = old, inv[old] = new).
void permute_csr(int n, const int *rp, const int *ci, const double *v,
                 const std::vector<int> &perm, const std::vector<int> &inv,
                 std::vector<int> &orp, std::vector<int> &oci, std::vector<double> &ov);

// Host CSR result (fastainv output).
struct HostCsr {
  int n_rows = 0, n_cols = 0, n_nz = 0;
  int dtype = ISPM_F64;
  std::vector<int> row_ptr, cols;
  std::vector<float> elms_f;
  std::vector<double> elms_d;
  const void *elms_ptr() const
  {
    return dtype == ISPM_F32 ? (const void *)elms_f.data() : (const void *)elms_d.data();
  }
};

}  // namespace ispm

struct ispm_slell {
  ispm::HostSlell m;
};

struct ispm_csr {
  ispm::HostCsr m;
};

#endif
