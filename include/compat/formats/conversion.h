/* Drop-in for formats/conversion.h (reference formats/conversion.h:338-492):
 * csr_to_slell and csr_to_slell_guess_format for T = float or double, over
 * ispm_csr_to_slell / ispm_csr_to_slell_guess_format.  The sliced-ELL arrays
 * are bit-identical to the reference's, and like the reference both pad the
 * caller's CSR to a multiple of 512 rows in place (conversion.h:343). */
#ifndef FORMATS_CONVERSION_H
#define FORMATS_CONVERSION_H

#include <string.h>

#include "formats/formats.h"
#include "ispm_compat_detail.h"

namespace ispm_compat {

enum { kMaxSliceHeight = 512 };

template <class T>
slell_matrix<T, host_memory_space_tag> take_host_slell(ispm_c::ispm_slell *h)
{
  ispm_c::ispm_slell_view v;
  check(ispm_c::ispm_slell_get_view(h, &v), "ispm_slell_get_view");
  slell_matrix<T, host_memory_space_tag> B;
  B.n_rows = v.n_rows;
  B.n_cols = v.n_cols;
  B.n_nz = v.n_nz;
  B.slice_height = v.slice_height;
  B.n_slices = v.n_slices;
  B.hblock = v.hblock;
  B.var_height = v.var_height != 0;
  B.diags = v.diags != 0;
  B.min_slice_height = v.min_slice_height;
  B.max_slice_height = v.max_slice_height;
  B.slice_ptr.resize((size_t)v.n_slice_ptr);
  B.cols.resize((size_t)v.n_cols_arr);
  B.elms.resize((size_t)v.n_elms);
  if (v.n_slice_ptr)
    memcpy(B.slice_ptr.data(), v.slice_ptr, sizeof(unsigned) * (size_t)v.n_slice_ptr);
  if (v.n_cols_arr)
    memcpy(B.cols.data(), v.cols, sizeof(unsigned) * (size_t)v.n_cols_arr);
  if (v.n_elms)
    memcpy(B.elms.data(), v.elms, sizeof(T) * (size_t)v.n_elms);
  ispm_c::ispm_slell_free(h);
  return B;
}

}  // namespace ispm_compat

template <class T>
slell_matrix<T, host_memory_space_tag> csr_to_slell(const csr_matrix<T> &A, int req_slice_height,
                                                    int hblock, bool var_height,
                                                    bool use_diags, int min_height = 4)
{
  csr_matrix<T> &M = const_cast<csr_matrix<T> &>(A);
  M.pad(ispm_compat::kMaxSliceHeight);
  ispm_c::ispm_slell *h = nullptr;
  ispm_compat::check(ispm_c::ispm_csr_to_slell(ispm_compat::dtype_of<T>::value, M.n_rows,
                                               M.n_cols, M.row_ptr.data(), M.cols.data(),
                                               M.elms.data(), req_slice_height, hblock,
                                               var_height ? 1 : 0, use_diags ? 1 : 0,
                                               min_height, &h),
                     "csr_to_slell");
  return ispm_compat::take_host_slell<T>(h);
}

template <class T>
slell_matrix<T, host_memory_space_tag> csr_to_slell_guess_format(const csr_matrix<T> &A,
                                                                 int examine_ratio = 1,
                                                                 int min_height = 4)
{
  // the guess looks at the caller's rows as given; the conversion pads them
  ispm_c::ispm_slell *h = nullptr;
  ispm_compat::check(ispm_c::ispm_csr_to_slell_guess_format(
                         ispm_compat::dtype_of<T>::value, A.n_rows, A.n_cols, A.row_ptr.data(),
                         A.cols.data(), A.elms.data(), examine_ratio, min_height, &h),
                     "csr_to_slell_guess_format");
  const_cast<csr_matrix<T> &>(A).pad(ispm_compat::kMaxSliceHeight);
  return ispm_compat::take_host_slell<T>(h);
}

#endif
