// Device-resident scalars of the PCG solver and the classic-CG stop test.
#ifndef ISPM_PCG_STATE_H
#define ISPM_PCG_STATE_H

#include <cuda_runtime.h>

namespace ispm {

enum Done { kRunning = 0, kConverged = 1, kBreakdown = 2, kCap = 3, kReplace = 4 };

struct PcgState {
  double gamma, gammaold, delta, alpha, beta;
  double rr;       // ||r||^2 of the recursive residual
  double rr_ref;   // ||r||^2 at the last reliable update
  double thresh2;  // recursive residual target (absolute, squared)
  double ru2;      // replacement trigger: rr < ru2 * rr_ref
  double res2;     // ||b - A x||^2 of the last true residual
  double pq;       // classic CG: p.Ap
  double rz;       // classic CG: r.z of the current direction
  double rz_new;   // classic CG: r.z of the updated residual
  int it;          // iterations since the last full restart
  int max_it;      // iteration cap for this restart
  int done;        // Done
  int fresh;       // classic CG: next direction update starts a new sequence
};

// Set the stop / replacement flags after the residual update.
__device__ __forceinline__ void cg_flags(PcgState *st, double rr)
{
  if (!isfinite(rr))
    st->done = kBreakdown;
  else if (rr <= st->thresh2)
    st->done = kConverged;
  else if (rr < st->ru2 * st->rr_ref)
    st->done = kReplace;
  else if (st->it >= st->max_it)
    st->done = kCap;
}

// Stop test at the head of a direction step (classic CG with a
// preconditioner): true when the iteration must hand over to the host.
__device__ __forceinline__ bool cg_stop(const PcgState *st, double rr)
{
  return !isfinite(rr) || rr <= st->thresh2 || rr < st->ru2 * st->rr_ref ||
         st->it >= st->max_it;
}

}  // namespace ispm

#endif
