// Internal launch interface of the sblas kernels (shared with the solver).
#ifndef ISPM_SBLAS_IMPL_H
#define ISPM_SBLAS_IMPL_H

#include <cuda_runtime.h>

#include "ispm_internal.h"

namespace ispm {

// Partial-sum slots per reduction in a scratch area; grids never exceed it.
constexpr int kSblasMaxBlocks = 1024;

// Per-device scratch of the C-ABI reductions: 3 * kSblasMaxBlocks doubles
// followed by a zero-initialised arrival ticket.
int sblas_scratch(double **part, unsigned **ticket);
int sblas_grid(long long n, int vec);

template <class T> struct PpcgVecArgs {
  T *resnorm, *gamma, *delta;
  const T *alpha, *beta;
  const T *n, *m;
  T *p, *s, *q, *z, *x, *r, *u, *w;
  long long n_elts;
  int vec;
  double *part;
  unsigned *ticket;
};

template <class T>
int dot_launch(const T *x, const T *y, T *s, long long n, double *part, unsigned *ticket,
               cudaStream_t st);
template <class T> int ppcg_vectors_launch(PpcgVecArgs<T> g, cudaStream_t st);

}  // namespace ispm

#endif
