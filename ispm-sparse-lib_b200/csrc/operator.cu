// Solver operators (operator.h).
#include "operator.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <new>
#include <thread>
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

// Convert the CSR into every candidate shape and keep the one with the
// fewest stored bytes, each candidate's bytes times weight[k] when weights
// are given (the earliest candidate on a tie).  The conversions are
// independent host passes over the matrix, so they run on up to one thread
// per core; each thread keeps only its own best, so at most that many
// converted copies exist at once.  Returns the index of the chosen
// candidate, or -1 when no shape accepted the matrix (with one candidate,
// the conversion's own error message stands).
int convert_smallest(int elm_dtype, int n_rows, int n_cols, const int *rp, const int *ci,
                     const void *vals, const std::vector<ispm_slell_params> &cands,
                     HostSlell &best, size_t &best_bytes,
                     const std::vector<double> *weight = nullptr)
{
  struct Best {
    int idx = -1;
    double cost = 0.0;
    size_t bytes = ~(size_t)0;
    HostSlell h;
  };
  auto consider = [](const Best &b, int idx, double cost) {
    return b.idx < 0 || cost < b.cost || (cost == b.cost && idx < b.idx);
  };
  const int nc = (int)cands.size();
  unsigned hw = std::thread::hardware_concurrency();
  const int nt = std::max(1, std::min(nc, (int)(hw ? hw : 1)));
  std::vector<Best> local(nt);
  std::atomic<int> next{0};
  auto work = [&](int t) {
    for (int k = next.fetch_add(1); k < nc; k = next.fetch_add(1)) {
      const ispm_slell_params &c = cands[k];
      HostSlell h;
      try {
        if (convert_csr(elm_dtype, n_rows, n_cols, rp, ci, vals, (int)c.S, (int)c.H, c.V != 0,
                        c.D != 0, 4, h))
          continue;
      } catch (const std::bad_alloc &) {
        continue;
      }
      const size_t bytes = stored_bytes(h);
      const double cost = (double)bytes * (weight ? (*weight)[k] : 1.0);
      if (consider(local[t], k, cost)) {
        local[t].idx = k;
        local[t].cost = cost;
        local[t].bytes = bytes;
        local[t].h = std::move(h);
      }
    }
  };
  if (nt == 1) {
    work(0);
  } else {
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; t++)
      pool.emplace_back(work, t);
    work(0);
    for (std::thread &th : pool)
      th.join();
  }
  int bi = -1;
  for (int t = 0; t < nt; t++)
    if (local[t].idx >= 0 && (bi < 0 || consider(local[bi], local[t].idx, local[t].cost)))
      bi = t;
  if (bi < 0)
    return -1;
  best = std::move(local[bi].h);
  best_bytes = local[bi].bytes;
  return local[bi].idx;
}

// The solver operators' cost weights per candidate shape (Operator::upload).
std::vector<double> shape_weights(const std::vector<ispm_slell_params> &cands)
{
  std::vector<double> w(cands.size(), 1.0);
  for (size_t c = 0; c < cands.size(); c++)
    w[c] = cands[c].S <= 32 ? 1.10 : cands[c].S == 64 ? 1.02 : 1.0;
  return w;
}

}  // namespace

int choose_operator_shape(int elm_dtype, int n, const int *rp, const int *ci, const double *v,
                          ispm_slell_params &out)
{
  std::vector<float> vf;
  const void *vals = typed_values(elm_dtype, v, (size_t)rp[n], vf);
  std::vector<ispm_slell_params> cands;
  candidate_shapes(elm_dtype, n, n, rp, ci, vals, false, cands);
  const std::vector<double> weight = shape_weights(cands);
  HostSlell h;
  size_t bytes = 0;
  const int k = convert_smallest(elm_dtype, n, n, rp, ci, vals, cands, h, bytes, &weight);
  clear_error();
  if (k < 0)
    return fail(ISPM_ERR_INVALID, "no sliced-ELL shape accepted the matrix");
  out = cands[k];
  return ISPM_OK;
}

int choose_format(int elm_dtype, int n_rows, int n_cols, const int *rp, const int *ci,
                  const double *v, bool fixed_height, ispm_slell_params &out, size_t *out_bytes)
{
  std::vector<float> vf;
  const void *vals = typed_values(elm_dtype, v, (size_t)rp[n_rows], vf);
  std::vector<ispm_slell_params> cands;
  candidate_shapes(elm_dtype, n_rows, n_cols, rp, ci, vals, fixed_height, cands);
  HostSlell h;
  size_t best = 0;
  const int k = convert_smallest(elm_dtype, n_rows, n_cols, rp, ci, vals, cands, h, best);
  clear_error();
  if (k < 0)
    return fail(ISPM_ERR_INVALID, "no sliced-ELL shape accepted the matrix");
  out = cands[k];
  if (out_bytes)
    *out_bytes = best;
  return ISPM_OK;
}

int Operator::upload(int vec_dtype, int elm_dtype, int n, const int *rp, const int *ci,
                     const double *v, const ispm_slell_params *force,
                     std::vector<unsigned> *value_pos, bool fixed_height, bool bf16_values,
                     bool f16_values)
{
  std::vector<float> vf;
  const void *vals = typed_values(elm_dtype, v, (size_t)rp[n], vf);
  std::vector<ispm_slell_params> cands;
  if (force)
    cands.push_back(*force);
  else
    candidate_shapes(elm_dtype, n, n, rp, ci, vals, fixed_height, cands);
  // convert every candidate and keep the smallest (no second conversion).
  // Short slices cost time that their stored bytes do not show: at the
  // default 4 rows a thread a 32-row slice is 8 threads, so a warp walks
  // four slices' diagonal lists and x windows, where a 128-row slice is one
  // warp.  Measured on a B200 (FP32, diagonal blocks): the renumbered 192^3
  // 7-point graph's A takes 82.5 us at S = 32 (its fewest bytes) and 74.8 us
  // at S = 128 (4% more bytes), its FSAI factor 49.3 / 45.8 us (3% more);
  // the 128^3 27-point A 45.5 us at S = 64 and 43.6 us at S = 128.  So
  // 32-row shapes count 10% and 64-row shapes 2% above their bytes.
  const std::vector<double> weight = shape_weights(cands);
  HostSlell best;
  size_t best_bytes = 0;
  const int k =
      convert_smallest(elm_dtype, n, n, rp, ci, vals, cands, best, best_bytes, &weight);
  if (k < 0)
    return force ? ISPM_ERR_INVALID  // the conversion's own message stands
                 : fail(ISPM_ERR_INVALID, "no sliced-ELL shape accepted the operator");
  fmt = cands[k];
  clear_error();
  if (value_pos)
    if (int st = value_map(best, n, rp, ci, *value_pos))
      return st;
  if (f16_values && elm_dtype == ISPM_F32) {
    if (int st = dev.upload_f16(best))
      return st;
    diag = nullptr;
    inv_scale = 1.f;
  } else if (int st = dev.upload(best, bf16_values && elm_dtype == ISPM_F32)) {
    return st;
  }
  lp = default_launch(vec_dtype, dev.view());
  return ISPM_OK;
}

uint16_t f16_bits(double v)
{
  const uint16_t sign = std::signbit(v) ? 0x8000u : 0u;
  const double a = std::fabs(v);
  if (a == 0.0)
    return sign;
  // quantum of the binade of a (2^-24 below the normal range), then round to
  // a multiple of it, ties to even (nearbyint under the default rounding mode)
  int e;
  std::frexp(a, &e);  // a = f * 2^e, f in [0.5, 1)
  const int qe = std::max(e - 11, -24);
  const double r = std::ldexp(std::nearbyint(std::ldexp(a, -qe)), qe);
  if (r < 0x1p-14)  // subnormal
    return (uint16_t)(sign | (uint16_t)std::ldexp(r, 24));
  int er;
  const double fr = std::frexp(r, &er);  // r = fr * 2^er, fr in [0.5, 1)
  const unsigned exp_field = (unsigned)(er - 1 + 15);
  const unsigned mant = (unsigned)std::ldexp(fr * 2.0 - 1.0, 10);
  return (uint16_t)(sign | (exp_field << 10) | mant);
}

double f16_value(uint16_t h)
{
  const double s = (h & 0x8000u) ? -1.0 : 1.0;
  const unsigned ef = (h >> 10) & 0x1fu, m = h & 0x3ffu;
  if (ef == 0)
    return s * std::ldexp((double)m, -24);
  return s * std::ldexp(1.0 + (double)m / 1024.0, (int)ef - 15);
}

int split_f16(int n, const int *rp, const int *ci, const double *v, uint16_t *off, float *diag,
              float &scale)
{
  double amax = 0.0;
  const long long nnz = rp[n];
  for (long long k = 0; k < nnz; k++)
    if (!std::isfinite(v[k]))
      return fail(ISPM_ERR_INVALID, "FP16 split: non-finite value at entry %lld", k);
  for (int i = 0; i < n; i++)
    for (int k = rp[i]; k < rp[i + 1]; k++)
      if (ci[k] != i)
        amax = std::max(amax, std::fabs(v[k]));
  // the largest magnitude lands in [2^13, 2^14): room below the binary16
  // maximum (65504), 27 binades above its normal range
  int e = 0;
  if (amax > 0.0)
    std::frexp(amax, &e);  // amax in [2^(e-1), 2^e)
  const int se = amax > 0.0 ? 14 - e : 0;
  if (se > 127 || se < -126)
    return fail(ISPM_ERR_INVALID, "FP16 split: off-diagonal magnitudes out of FP32 scale range");
  const double sc = std::ldexp(1.0, se);
  for (int i = 0; i < n; i++) {
    double d = 0.0, corr = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; k++) {
      if (ci[k] == i) {
        d += v[k];
        off[k] = 0;
        continue;
      }
      const uint16_t h = f16_bits(v[k] * sc);
      off[k] = h;
      corr += std::fabs(f16_value(h)) / sc - std::fabs(v[k]);
    }
    diag[i] = (float)(d + corr);
  }
  scale = (float)sc;
  return ISPM_OK;
}

int Operator::upload_split_f16(int n, const int *rp, const int *ci, const double *v)
{
  const long long nnz = rp[n];
  std::vector<uint16_t> h16((size_t)nnz);
  std::vector<float> dg((size_t)n);
  float sc = 1.f;
  if (int st = split_f16(n, rp, ci, v, h16.data(), dg.data(), sc))
    return st;
  // off-diagonal CSR with the scaled binary16 values (exact in FP32)
  std::vector<int> orp((size_t)n + 1), oci;
  std::vector<double> ov;
  oci.reserve((size_t)nnz);
  ov.reserve((size_t)nnz);
  orp[0] = 0;
  for (int i = 0; i < n; i++) {
    for (int k = rp[i]; k < rp[i + 1]; k++)
      if (ci[k] != i) {
        oci.push_back(ci[k]);
        ov.push_back(f16_value(h16[(size_t)k]));
      }
    orp[(size_t)i + 1] = (int)oci.size();
  }
  std::vector<float> vf;
  const void *vals = typed_values(ISPM_F32, ov.data(), ov.size(), vf);
  std::vector<ispm_slell_params> cands;
  candidate_shapes(ISPM_F32, n, n, orp.data(), oci.data(), vals, false, cands);
  HostSlell best;
  size_t best_bytes = ~(size_t)0;
  for (const ispm_slell_params &c : cands) {
    HostSlell h;
    if (convert_csr(ISPM_F32, n, n, orp.data(), oci.data(), vals, (int)c.S, (int)c.H, c.V != 0,
                    c.D != 0, 4, h))
      continue;
    const size_t bytes = stored_bytes(h);
    if (bytes < best_bytes) {
      best_bytes = bytes;
      best = std::move(h);
      fmt = c;
    }
  }
  if (best_bytes == ~(size_t)0)
    return fail(ISPM_ERR_INVALID, "no sliced-ELL shape accepted the off-diagonal part");
  clear_error();
  if (int st = dev.upload_f16(best))
    return st;
  // the diagonal, zero-padded to the matrix's padded row count
  const size_t rows = (size_t)dev.meta.n_rows;
  dg.resize(std::max(rows, (size_t)n), 0.f);
  float *d = nullptr;
  cudaError_t e = cudaMalloc(&d, rows * sizeof(float));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? ISPM_ERR_NOMEM : ISPM_ERR_CUDA,
                "cudaMalloc(%zu): %s", rows * sizeof(float), cudaGetErrorString(e));
  }
  diag_mem.reset(d, [](float *q) { cudaFree(q); });
  diag = d;
  ISPM_CUDA_TRY(cudaMemcpy(d, dg.data(), rows * sizeof(float), cudaMemcpyHostToDevice));
  inv_scale = 1.f / sc;
  lp = default_launch(ISPM_F32, dev.view());
  return ISPM_OK;
}

size_t Operator::bytes() const
{
  const ispm_slell_view m = dev.view();
  const size_t esz = m.elm_dtype == ISPM_F64 ? 8 : m.elm_dtype == ISPM_F32 ? 4 : 2;
  return 4 * (size_t)m.n_slice_ptr + 4 * (size_t)m.n_cols_arr + esz * (size_t)m.n_elms +
         (diag ? 4 * (size_t)m.n_rows : 0);
}

}  // namespace ispm

extern "C" int ispm_csr_split_f16(int n, const int *row_ptr, const int *cols, const double *vals,
                                  uint16_t *off_f16, float *diag, float *scale)
{
  ispm::clear_error();
  if (n < 0 || !row_ptr || !cols || (row_ptr[n] && !vals) || !off_f16 || !diag || !scale)
    return ispm::fail(ISPM_ERR_INVALID, "bad arguments");
  for (int i = 0; i < n; i++)
    for (int k = row_ptr[i]; k < row_ptr[i + 1]; k++)
      if (cols[k] < 0 || cols[k] >= n)
        return ispm::fail(ISPM_ERR_INVALID, "column %d out of range in row %d", cols[k], i);
  return ispm::split_f16(n, row_ptr, cols, vals, off_f16, diag, *scale);
}
