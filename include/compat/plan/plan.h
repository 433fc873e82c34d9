/* Drop-in for plan/plan.h (reference plan/plan.h:1-161): spmv_plan<T, E>
 * with its public members (host_matrix, device_matrix, mparams, params) and
 * methods, for (T, E) = (float, float), (double, float), (double, double).
 *
 * PLAN_DEFAULT / PLAN_ESTIMATE convert with the reference's format guess and
 * take the launch shape of the B200 heuristic (ispm_default_launch) where
 * the reference fixes N = 512, H = 1.  PLAN_EXHAUSTIVE runs the library's
 * autotuner (ispm_plan_create: the reference's format grid plus hblock 4,
 * every launch shape median-timed) and then converts the caller's CSR in
 * the winning format.  Both pad the caller's CSR to a multiple of 512 rows,
 * as the reference's conversions do.  update_device_matrix_coefs copies the
 * host element array to the device.  A plan owns both matrices and cannot be
 * copied (the reference's implicit copy would free them twice). */
#ifndef PLAN_PLAN_H
#define PLAN_PLAN_H

#include "cuda/spmv/kernel-iface.h"
#include "formats/conversion.h"
#include "formats/formats.h"
#include "ispm_compat_detail.h"
#include "util/cuda/timer.h"

enum spmv_plan_kind {
  PLAN_DEFAULT,
  PLAN_ESTIMATE,
  PLAN_EXHAUSTIVE,
};

enum spmv_plan_flags { SPMV_NO_TEXTURE_MEMORY = 001, SPMV_PLAN_NO_DEVICE = 002 };

template <class T, class E = T> struct spmv_plan {
  slell_matrix<E, host_memory_space_tag> *host_matrix;
  slell_matrix<E, device_memory_space_tag> *device_matrix;
  slell_params mparams;
  spmv_launch_params params;

  spmv_plan() : host_matrix(NULL), device_matrix(NULL) {}
  spmv_plan(const csr_matrix<E> &m, spmv_plan_kind kind = PLAN_DEFAULT, unsigned flags = 0);
  spmv_plan(const spmv_plan &) = delete;
  spmv_plan &operator=(const spmv_plan &) = delete;
  ~spmv_plan()
  {
    delete host_matrix;
    delete device_matrix;
  }

  void update_device_matrix_coefs() { device_matrix->elms = host_matrix->elms; }

  void upload()
  {
    if (device_matrix)
      delete device_matrix;
    device_matrix = new slell_matrix<E, device_memory_space_tag>(*host_matrix);
  }

  void change_host_matrix(const csr_matrix<E> &m)
  {
    delete host_matrix;
    host_matrix = new slell_matrix<E, host_memory_space_tag>(
        csr_to_slell(m, mparams.S, mparams.H, mparams.V, mparams.D));
  }

  void execute_spmv(vector<T, device_memory_space_tag> &x, vector<T, device_memory_space_tag> &y)
  {
    launch_spmv_kernel<T, E>(params, *device_matrix, x, y);
  }

  void execute_spmv(T *xptr, T *yptr) { launch_spmv_kernel<T, E>(params, *device_matrix, xptr, yptr); }
};

template <class T, class E>
spmv_plan<T, E>::spmv_plan(const csr_matrix<E> &m, spmv_plan_kind kind, unsigned flags)
    : host_matrix(NULL), device_matrix(NULL)
{
  const bool usetex = !(flags & SPMV_NO_TEXTURE_MEMORY);
  if (kind == PLAN_EXHAUSTIVE) {
    ispm_c::ispm_plan *p = NULL;
    ispm_compat::check(
        ispm_c::ispm_plan_create(ispm_compat::dtype_of<T>::value,
                                 ispm_compat::dtype_of<E>::value, m.n_rows, m.n_cols,
                                 m.row_ptr.data(), m.cols.data(), m.elms.data(),
                                 ISPM_PLAN_EXHAUSTIVE, 0u, &p),
        "spmv_plan (exhaustive)");
    ispm_c::ispm_slell_params mp;
    ispm_c::ispm_launch_params lp;
    ispm_compat::check(ispm_c::ispm_plan_get_params(p, &mp, &lp), "ispm_plan_get_params");
    ispm_c::ispm_plan_free(p);
    mparams.S = mp.S;
    mparams.H = mp.H;
    mparams.V = mp.V;
    mparams.D = mp.D;
    params.N = lp.N;
    params.S = lp.S;
    params.H = lp.H;
    params.use_tex_sliceptr = params.use_tex_x = usetex;
    host_matrix = new slell_matrix<E, host_memory_space_tag>(
        csr_to_slell(m, mparams.S, mparams.H, mparams.V, mparams.D));
    upload();
    return;
  }
  host_matrix = new slell_matrix<E, host_memory_space_tag>(csr_to_slell_guess_format(m));
  if (!(flags & SPMV_PLAN_NO_DEVICE))
    upload();
  mparams.S = host_matrix->slice_height;
  mparams.H = host_matrix->hblock;
  mparams.V = host_matrix->var_height;
  mparams.D = host_matrix->diags;
  // the launch heuristic reads only the matrix's shape
  ispm_c::ispm_slell_view v;
  v.n_rows = host_matrix->n_rows;
  v.n_cols = host_matrix->n_cols;
  v.n_nz = host_matrix->n_nz;
  v.slice_height = host_matrix->slice_height;
  v.n_slices = host_matrix->n_slices;
  v.hblock = host_matrix->hblock;
  v.var_height = host_matrix->var_height;
  v.diags = host_matrix->diags;
  v.elm_dtype = ispm_compat::dtype_of<E>::value;
  v.min_slice_height = host_matrix->min_slice_height;
  v.max_slice_height = host_matrix->max_slice_height;
  v.n_slice_ptr = (long long)host_matrix->slice_ptr.size();
  v.n_cols_arr = (long long)host_matrix->cols.size();
  v.n_elms = (long long)host_matrix->elms.size();
  v.slice_ptr = host_matrix->slice_ptr.data();
  v.cols = host_matrix->cols.data();
  v.elms = host_matrix->elms.data();
  ispm_c::ispm_launch_params lp;
  ispm_compat::check(ispm_c::ispm_default_launch(ispm_compat::dtype_of<T>::value, &v, &lp),
                     "ispm_default_launch");
  params.N = lp.N;
  params.S = lp.S;
  params.H = lp.H;
  params.use_tex_sliceptr = params.use_tex_x = usetex;
}

#endif
