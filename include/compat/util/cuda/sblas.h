/* Drop-in for util/cuda/sblas.h (reference util/cuda/sblas.h:1-56):
 * sblas::copy_indexed, add_indexed, dot, ppcg_update_scalars and
 * ppcg_update_vectors on devmem<T> pointers, T = float or double, over the
 * ispm_sblas_* entry points on the legacy default stream.  Reductions
 * accumulate in FP64 (the reference accumulates in T); add_indexed adds
 * atomically, so repeated indices all count (the reference races on them). */
#ifndef SBLAS_H
#define SBLAS_H

#include <cuda_runtime.h>

#include "ispm_compat_detail.h"
#include "util/cuda/devmem.h"

namespace sblas {

template <typename T>
void copy_indexed(devmem<T> *dst, const devmem<T> *src, const devmem<int> *i, int n_elts)
{
  ispm_compat::check(ispm_c::ispm_sblas_copy_indexed(ispm_compat::dtype_of<T>::value, dst, src,
                                                     uncast_devmem(i), n_elts, NULL),
                     "sblas::copy_indexed");
}

template <typename T>
void add_indexed(devmem<T> *dst, const devmem<T> *src, const devmem<int> *i, int n_elts)
{
  ispm_compat::check(ispm_c::ispm_sblas_add_indexed(ispm_compat::dtype_of<T>::value, dst, src,
                                                    uncast_devmem(i), n_elts, NULL),
                     "sblas::add_indexed");
}

template <typename T>
void dot(const devmem<T> *x, const devmem<T> *y, devmem<T> *s, int n_elts)
{
  ispm_compat::check(
      ispm_c::ispm_sblas_dot(ispm_compat::dtype_of<T>::value, x, y, s, n_elts, NULL),
      "sblas::dot");
}

template <typename T>
void ppcg_update_scalars(devmem<T> *alpha, devmem<T> *beta, const devmem<T> *gamma,
                         const devmem<T> *gammaold, const devmem<T> *delta)
{
  ispm_compat::check(ispm_c::ispm_sblas_ppcg_update_scalars(ispm_compat::dtype_of<T>::value,
                                                            alpha, beta, gamma, gammaold,
                                                            delta, NULL),
                     "sblas::ppcg_update_scalars");
}

template <typename T>
void ppcg_update_vectors(devmem<T> *resnorm, devmem<T> *gamma, devmem<T> *delta,
                         const devmem<T> *alpha, const devmem<T> *beta, const devmem<T> *n,
                         const devmem<T> *m, devmem<T> *p, devmem<T> *s, devmem<T> *q,
                         devmem<T> *z, devmem<T> *x, devmem<T> *r, devmem<T> *u, devmem<T> *w,
                         int n_elts)
{
  ispm_compat::check(ispm_c::ispm_sblas_ppcg_update_vectors(
                         ispm_compat::dtype_of<T>::value, resnorm, gamma, delta, alpha, beta, n,
                         m, p, s, q, z, x, r, u, w, n_elts, NULL),
                     "sblas::ppcg_update_vectors");
}

/* Additions to the reference's interface: the same operations ordered on a
 * caller's stream. */
template <typename T>
void dot(const devmem<T> *x, const devmem<T> *y, devmem<T> *s, int n_elts, cudaStream_t stream)
{
  ispm_compat::check(
      ispm_c::ispm_sblas_dot(ispm_compat::dtype_of<T>::value, x, y, s, n_elts, stream),
      "sblas::dot");
}

template <typename T>
void ppcg_update_scalars(devmem<T> *alpha, devmem<T> *beta, const devmem<T> *gamma,
                         const devmem<T> *gammaold, const devmem<T> *delta, cudaStream_t stream)
{
  ispm_compat::check(ispm_c::ispm_sblas_ppcg_update_scalars(ispm_compat::dtype_of<T>::value,
                                                            alpha, beta, gamma, gammaold,
                                                            delta, stream),
                     "sblas::ppcg_update_scalars");
}

template <typename T>
void ppcg_update_vectors(devmem<T> *resnorm, devmem<T> *gamma, devmem<T> *delta,
                         const devmem<T> *alpha, const devmem<T> *beta, const devmem<T> *n,
                         const devmem<T> *m, devmem<T> *p, devmem<T> *s, devmem<T> *q,
                         devmem<T> *z, devmem<T> *x, devmem<T> *r, devmem<T> *u, devmem<T> *w,
                         int n_elts, cudaStream_t stream)
{
  ispm_compat::check(ispm_c::ispm_sblas_ppcg_update_vectors(
                         ispm_compat::dtype_of<T>::value, resnorm, gamma, delta, alpha, beta, n,
                         m, p, s, q, z, x, r, u, w, n_elts, stream),
                     "sblas::ppcg_update_vectors");
}

}  // namespace sblas

#endif
