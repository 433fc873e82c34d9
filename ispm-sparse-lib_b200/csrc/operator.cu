// Solver operators (operator.h).
#include "operator.h"

#include <utility>

#include "cuda_util.cuh"

namespace ispm {

namespace {

void candidate_shapes(int elm_dtype, int n_rows, int n_cols, const int *rp, const int *ci,
                      const void *vals, bool fixed_height, std::vector<ispm_slell_params> &c)
{
  ispm_slell_params g;
  if (guess_format(elm_dtype, n_rows, n_cols, rp, ci, vals, 1, 4, g) == ISPM_OK) {
    if (fixed_height)
      g.V = 0;
    c.push_back(g);
  }
  for (unsigned S : {32u, 64u, 128u})
    for (unsigned D : {1u, 0u})
      c.push_back(ispm_slell_params{S, 1, 0, D});
  c.push_back(ispm_slell_params{64, 2, 0, 0});
}

size_t stored_bytes(const HostSlell &h)
{
  const size_t esz = h.elm_dtype == ISPM_F32 ? 4 : 8;
  return 4 * h.slice_ptr.size() + 4 * h.cols.size() + esz * h.n_elms();
}

const void *typed_values(int elm_dtype, const double *v, size_t nnz, std::vector<float> &vf)
{
  if (elm_dtype != ISPM_F32)
    return v;
  vf.resize(nnz);
  for (size_t k = 0; k < nnz; k++)
    vf[k] = (float)v[k];
  return vf.data();
}

}  // namespace

int choose_format(int elm_dtype, int n_rows, int n_cols, const int *rp, const int *ci,
                  const double *v, bool fixed_height, ispm_slell_params &out, size_t *out_bytes)
{
  std::vector<float> vf;
  const void *vals = typed_values(elm_dtype, v, (size_t)rp[n_rows], vf);
  std::vector<ispm_slell_params> cands;
  candidate_shapes(elm_dtype, n_rows, n_cols, rp, ci, vals, fixed_height, cands);
  size_t best = ~(size_t)0;
  for (const ispm_slell_params &c : cands) {
    HostSlell h;
    if (convert_csr(elm_dtype, n_rows, n_cols, rp, ci, vals, (int)c.S, (int)c.H, c.V != 0,
                    c.D != 0, 4, h))
      continue;
    const size_t bytes = stored_bytes(h);
    if (bytes < best) {
      best = bytes;
      out = c;
    }
  }
  clear_error();
  if (best == ~(size_t)0)
    return fail(ISPM_ERR_INVALID, "no sliced-ELL shape accepted the matrix");
  if (out_bytes)
    *out_bytes = best;
  return ISPM_OK;
}

int Operator::upload(int vec_dtype, int elm_dtype, int n, const int *rp, const int *ci,
                     const double *v, const ispm_slell_params *force,
                     std::vector<unsigned> *value_pos, bool fixed_height, bool bf16_values)
{
  std::vector<float> vf;
  const void *vals = typed_values(elm_dtype, v, (size_t)rp[n], vf);
  std::vector<ispm_slell_params> cands;
  if (force)
    cands.push_back(*force);
  else
    candidate_shapes(elm_dtype, n, n, rp, ci, vals, fixed_height, cands);
  // convert every candidate and keep the smallest (no second conversion)
  HostSlell best;
  size_t best_bytes = ~(size_t)0;
  for (const ispm_slell_params &c : cands) {
    HostSlell h;
    if (convert_csr(elm_dtype, n, n, rp, ci, vals, (int)c.S, (int)c.H, c.V != 0, c.D != 0, 4,
                    h))
      continue;
    const size_t bytes = stored_bytes(h);
    if (bytes < best_bytes) {
      best_bytes = bytes;
      best = std::move(h);
      fmt = c;
    }
  }
  if (best_bytes == ~(size_t)0)
    return force ? ISPM_ERR_INVALID  // the conversion's own message stands
                 : fail(ISPM_ERR_INVALID, "no sliced-ELL shape accepted the operator");
  clear_error();
  if (value_pos)
    if (int st = value_map(best, n, rp, ci, *value_pos))
      return st;
  if (int st = dev.upload(best, bf16_values && elm_dtype == ISPM_F32))
    return st;
  lp = default_launch(vec_dtype, dev.view());
  return ISPM_OK;
}

size_t Operator::bytes() const
{
  const ispm_slell_view m = dev.view();
  const size_t esz = m.elm_dtype == ISPM_F64 ? 8 : m.elm_dtype == ISPM_F32 ? 4 : 2;
  return 4 * (size_t)m.n_slice_ptr + 4 * (size_t)m.n_cols_arr + esz * (size_t)m.n_elms;
}

}  // namespace ispm
