// GPU FSAI build (fsai.cu).
#ifndef ISPM_FSAI_H
#define ISPM_FSAI_H

#include <cuda_runtime.h>

#include <vector>

#include "ispm_internal.h"

namespace ispm {

// Lower pattern of A (columns <= row, diagonal required): G's CSR pattern.
int fsai_lower_pattern(int n, const int *rp, const int *ci, std::vector<int> &g_rp,
                       std::vector<int> &g_ci);
// G^T's CSR pattern and, for each entry k of G, its position t_of[k] in G^T.
void fsai_transpose_pattern(int n, const std::vector<int> &g_rp, const std::vector<int> &g_ci,
                            std::vector<int> &t_rp, std::vector<int> &t_ci,
                            std::vector<unsigned> &t_of);
// FSAI values of G (device, in G's CSR order) from A (device CSR, FP64,
// symmetric, sorted columns); *fallbacks_d counts rows whose local matrix was
// not positive definite (Jacobi row used).
int fsai_build_values(int n, const int *a_rp_d, const int *a_ci_d, const double *a_v_d,
                      const int *g_rp_d, double *g_v_d, unsigned *fallbacks_d, cudaStream_t s);

}  // namespace ispm

#endif
