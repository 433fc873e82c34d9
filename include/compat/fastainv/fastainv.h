/* Drop-in for fastainv/fastainv.h (reference fastainv/fastainv.h:1-30):
 * fastainv_sym<double, out_real> for out_real = float or double, over
 * ispm_fastainv_sym.  The factors are bit-identical to the reference's;
 * returns false for an empty matrix like the reference, aborts on any other
 * failure. */
#ifndef FASTAINV_H
#define FASTAINV_H

#include <string.h>

#include "formats/formats.h"
#include "ispm_compat_detail.h"

typedef void (*progress_f)(void *);

namespace ispm_compat {

template <class T> void take_csr(ispm_c::ispm_csr *h, csr_matrix<T> &out)
{
  int n_rows = 0, n_cols = 0, n_nz = 0, dt = 0;
  check(ispm_c::ispm_csr_get_info(h, &n_rows, &n_cols, &n_nz, &dt), "ispm_csr_get_info");
  const int *rp = NULL, *ci = NULL;
  const void *v = NULL;
  check(ispm_c::ispm_csr_get_arrays(h, &rp, &ci, &v), "ispm_csr_get_arrays");
  out.n_rows = n_rows;
  out.n_cols = n_cols;
  out.n_nz = n_nz;
  out.row_ptr.resize((size_t)n_rows + 1);
  out.cols.resize((size_t)n_nz);
  out.elms.resize((size_t)n_nz);
  memcpy(out.row_ptr.data(), rp, sizeof(int) * ((size_t)n_rows + 1));
  if (n_nz) {
    memcpy(out.cols.data(), ci, sizeof(int) * (size_t)n_nz);
    memcpy(out.elms.data(), v, sizeof(T) * (size_t)n_nz);
  }
  ispm_c::ispm_csr_free(h);
}

}  // namespace ispm_compat

template <class in_real, class out_real>
bool fastainv_sym(csr_matrix<out_real> &Ainv1, csr_matrix<out_real> &Ainv2,
                  const csr_matrix<in_real> &A, progress_f progress, void *v,
                  long long max_elts = 8192000, double droptol = 0.125)
{
  static_assert(sizeof(in_real) == 8, "fastainv_sym takes a double matrix");
  ispm_c::ispm_csr *g1 = NULL, *g2 = NULL;
  const int st = ispm_c::ispm_fastainv_sym(
      ispm_compat::dtype_of<out_real>::value, A.n_rows, A.row_ptr.data(), A.cols.data(),
      A.elms.data(), progress, v, max_elts, droptol, &g1, &g2, NULL);
  if (st == ISPM_ERR_INVALID && A.n_rows <= 0)
    return false;
  ispm_compat::check(st, "fastainv_sym");
  ispm_compat::take_csr(g1, Ainv1);
  ispm_compat::take_csr(g2, Ainv2);
  return true;
}

#endif
