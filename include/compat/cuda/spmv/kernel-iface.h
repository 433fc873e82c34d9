/* Drop-in for cuda/spmv/kernel-iface.h (reference cuda/spmv/kernel-iface.h:1-74):
 * spmv_launch_params and both launch_spmv_kernel<T, E> overloads for the
 * reference's instantiations (float, float), (double, float) and
 * (double, double), over ispm_launch_spmv on the legacy default stream.
 *
 * As in the reference, a launch whose parameters the kernels do not support
 * launches nothing (cuda/spmv/dispatch.h:131-203); any other failure aborts.
 * use_tex_sliceptr / use_tex_x are accepted and ignored (sm_100 has no
 * texture references). */
#ifndef SPMV_GPU_H
#define SPMV_GPU_H

#include <cuda_runtime.h>

#include "formats/formats.h"
#include "ispm_compat_detail.h"

#define SPMV_PARAMS_VALID_P(N, S, H) ((N) >= (S) / (H) && (S) >= (H))

struct spmv_launch_params {
  unsigned N;
  unsigned S;
  unsigned H;
  bool use_tex_sliceptr;
  bool use_tex_x;

  bool valid() const { return SPMV_PARAMS_VALID_P(N, S, H); }
};

namespace ispm_compat {

template <class E> ispm_c::ispm_slell_view view_of(slell_matrix<E, device_memory_space_tag> &m)
{
  ispm_c::ispm_slell_view v;
  v.n_rows = m.n_rows;
  v.n_cols = m.n_cols;
  v.n_nz = m.n_nz;
  v.slice_height = m.slice_height;
  v.n_slices = m.n_slices;
  v.hblock = m.hblock;
  v.var_height = m.var_height ? 1 : 0;
  v.diags = m.diags ? 1 : 0;
  v.elm_dtype = dtype_of<E>::value;
  v.min_slice_height = m.min_slice_height;
  v.max_slice_height = m.max_slice_height;
  v.n_slice_ptr = (long long)m.slice_ptr.size();
  v.n_cols_arr = (long long)m.cols.size();
  v.n_elms = (long long)m.elms.size();
  v.slice_ptr = m.slice_ptr.udata();
  v.cols = m.cols.udata();
  v.elms = m.elms.udata();
  return v;
}

template <class T, class E>
void launch(const spmv_launch_params &params, slell_matrix<E, device_memory_space_tag> &m,
            T *x, T *y, cudaStream_t stream = NULL)
{
  static_assert(sizeof(T) >= sizeof(E) && (sizeof(E) == 4 || sizeof(E) == 8),
                "launch_spmv_kernel<T, E>: (float, float), (double, float) or (double, double)");
  ispm_c::ispm_launch_params p;
  p.N = params.N;
  p.S = params.S;
  p.H = params.H;
  p.use_tex_sliceptr = params.use_tex_sliceptr;
  p.use_tex_x = params.use_tex_x;
  const ispm_c::ispm_slell_view v = view_of(m);
  const int st = ispm_c::ispm_launch_spmv(dtype_of<T>::value, &p, &v, x, y, stream);
  if (st != ISPM_ERR_INVALID)  // unsupported parameters: nothing launched
    check(st, "launch_spmv_kernel");
}

}  // namespace ispm_compat

template <class T, class E>
void launch_spmv_kernel(spmv_launch_params &params, slell_matrix<E, device_memory_space_tag> &m,
                        vector<T, device_memory_space_tag> &x,
                        vector<T, device_memory_space_tag> &y)
{
  ispm_compat::launch<T, E>(params, m, x.udata(), y.udata());
}

template <class T, class E>
void launch_spmv_kernel(spmv_launch_params &params, slell_matrix<E, device_memory_space_tag> &m,
                        T *xptr, T *yptr)
{
  ispm_compat::launch<T, E>(params, m, xptr, yptr);
}

/* Additions to the reference's interface: the same launches ordered on a
 * caller's stream (asynchronous with the host). */
template <class T, class E>
void launch_spmv_kernel(spmv_launch_params &params, slell_matrix<E, device_memory_space_tag> &m,
                        vector<T, device_memory_space_tag> &x,
                        vector<T, device_memory_space_tag> &y, cudaStream_t stream)
{
  ispm_compat::launch<T, E>(params, m, x.udata(), y.udata(), stream);
}

template <class T, class E>
void launch_spmv_kernel(spmv_launch_params &params, slell_matrix<E, device_memory_space_tag> &m,
                        T *xptr, T *yptr, cudaStream_t stream)
{
  ispm_compat::launch<T, E>(params, m, xptr, yptr, stream);
}

#endif
