// SpMV plan: format choice plus launch shape (plan/plan.h:9-161).
//
// DEFAULT / ESTIMATE keep the reference's format guess (so the device matrix
// is the one the reference would build) and replace its fixed launch shape
// (N = 512, H = 1) with a B200 heuristic.  EXHAUSTIVE searches the reference's
// format grid -- slice height 32..512, variable height, diagonal blocks,
// hblock width -- widened with hblock 4, and for each format every launch
// shape (N in 4..1024, H in 1/2/4), each timed as the median of several CUDA
// event measurements rather than one launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <vector>

#include "cuda_util.cuh"
#include "nvtx_range.h"
#include "spmv_launch.h"

namespace ispm {
namespace {

struct DevBuf {
  void *p = nullptr;
  ~DevBuf()
  {
    if (p)
      cudaFree(p);
  }
  int alloc(size_t bytes)
  {
    cudaError_t e = cudaMalloc(&p, bytes ? bytes : 16);
    if (e != cudaSuccess) {
      p = nullptr;
      cudaGetLastError();
      return fail(ISPM_ERR_NOMEM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
    }
    e = cudaMemset(p, 0, bytes ? bytes : 16);
    if (e != cudaSuccess)
      return fail(ISPM_ERR_CUDA, "cudaMemset: %s", cudaGetErrorString(e));
    return ISPM_OK;
  }
};

struct Events {
  cudaEvent_t a = nullptr, b = nullptr;
  ~Events()
  {
    if (a)
      cudaEventDestroy(a);
    if (b)
      cudaEventDestroy(b);
  }
};

// Median time (seconds) of `reps` launches, after one warm-up launch.
int time_launch(int vdt, const ispm_launch_params &p, const ispm_slell_view &m, const void *x,
                void *y, int reps, double &secs)
{
  Events ev;
  ISPM_CUDA_TRY(cudaEventCreate(&ev.a));
  ISPM_CUDA_TRY(cudaEventCreate(&ev.b));
  if (int st = launch_spmv(vdt, p, m, x, y, 0))
    return st;
  std::vector<float> t;
  for (int r = 0; r < reps; r++) {
    ISPM_CUDA_TRY(cudaEventRecord(ev.a, 0));
    if (int st = launch_spmv(vdt, p, m, x, y, 0))
      return st;
    ISPM_CUDA_TRY(cudaEventRecord(ev.b, 0));
    ISPM_CUDA_TRY(cudaEventSynchronize(ev.b));
    float ms = 0;
    ISPM_CUDA_TRY(cudaEventElapsedTime(&ms, ev.a, ev.b));
    t.push_back(ms);
  }
  std::sort(t.begin(), t.end());
  secs = 1e-3 * t[t.size() / 2];
  return ISPM_OK;
}

}  // namespace
}  // namespace ispm

struct ispm_plan {
  int vec_dtype = ISPM_F64, elm_dtype = ISPM_F64;
  std::unique_ptr<ispm_slell> host;
  std::unique_ptr<ispm_dslell> dev;
  ispm_slell_params mparams{};
  ispm_launch_params params{};
  double tuned = 0;
  // element slot -> CSR entry (-1 for padding), built on the first device
  // refresh
  int *map = nullptr;
  long long map_n = -1;
  void drop_map()
  {
    if (map)
      cudaFree(map);
    map = nullptr;
    map_n = -1;
  }
  ~ispm_plan() { drop_map(); }
};

using namespace ispm;

static int check_pair(int vdt, int edt)
{
  if ((vdt == ISPM_F32 && edt == ISPM_F32) || (vdt == ISPM_F64 && edt == ISPM_F32) ||
      (vdt == ISPM_F64 && edt == ISPM_F64))
    return ISPM_OK;
  return fail(ISPM_ERR_INVALID, "spmv_plan<T, E> is instantiated for (float,float), "
                                "(double,float), (double,double)");
}

static int plan_exhaustive(ispm_plan *pl, int n_rows, int n_cols, const int *row_ptr,
                           const int *cols, const void *elms)
{
  double best = 1e300;
  ispm_slell_params best_m{};
  ispm_launch_params best_p{};
  const size_t vsz = pl->vec_dtype == ISPM_F32 ? 4 : 8;
  for (unsigned S = 32; S <= 512; S <<= 1)
    for (unsigned V = 0; V <= 1; V++)
      for (unsigned D = 0; D <= 1; D++)
        for (unsigned W = 1; W <= (D ? 1u : 4u); W <<= 1) {
          HostSlell h;
          if (convert_csr(pl->elm_dtype, n_rows, n_cols, row_ptr, cols, elms, (int)S, (int)W,
                          V != 0, D != 0, 4, h))
            continue;
          DeviceSlell d;
          if (int st = d.upload(h))
            return st;
          DevBuf x, y;
          if (int st = x.alloc(std::max(h.n_cols, 1) * vsz + 64))
            return st;
          if (int st = y.alloc(std::max(h.n_rows, 1) * vsz + 64))
            return st;
          const ispm_slell_view v = d.view();
          for (unsigned N = 4; N <= 1024; N <<= 1)
            for (unsigned H = 1; H <= 4; H <<= 1) {
              ispm_launch_params p{N, V ? N * H : S, H, 1, 1};
              if (check_launch(pl->vec_dtype, p, v) != ISPM_OK)
                continue;
              double t;
              if (int st = time_launch(pl->vec_dtype, p, v, x.p, y.p, 5, t))
                return st;
              if (t < best) {
                best = t;
                best_m = ispm_slell_params{S, W, V, D};
                best_p = p;
              }
            }
        }
  clear_error();
  if (best >= 1e300)
    return fail(ISPM_ERR_INVALID, "no format/launch combination is valid for this matrix");
  pl->mparams = best_m;
  pl->params = best_p;
  pl->tuned = best;
  pl->host.reset(new ispm_slell);
  if (int st = convert_csr(pl->elm_dtype, n_rows, n_cols, row_ptr, cols, elms, (int)best_m.S,
                           (int)best_m.H, best_m.V != 0, best_m.D != 0, 4, pl->host->m))
    return st;
  pl->dev.reset(new ispm_dslell);
  if (int st = pl->dev->d.upload(pl->host->m))
    return st;
  if (getenv("SPMV_TUNE_RESULT")) {
    // plan.h:137-142, with the stored / effective / CSR-equivalent byte counts
    const ispm_slell *h = pl->host.get();
    const unsigned long long csr_bytes =
        4ull * (n_rows + 1 + (unsigned long long)row_ptr[n_rows]) +
        (unsigned long long)vsz * ((unsigned long long)row_ptr[n_rows] + 2ull * n_rows);
    fprintf(stderr, "[spmv tuning] %g ms:  %g (%g eff, %g csr-equiv) GB/s\n", 1e3 * best,
            1e-9 * ispm_slell_spmv_bytes(h, 0, (int)vsz) / best,
            1e-9 * ispm_slell_spmv_bytes(h, 1, (int)vsz) / best, 1e-9 * csr_bytes / best);
  }
  return ISPM_OK;
}

extern "C" {

int ispm_plan_create(int vec_dtype, int elm_dtype, int n_rows, int n_cols, const int *row_ptr,
                     const int *cols, const void *elms, int kind, unsigned flags,
                     ispm_plan **out)
{
  clear_error();
  NvtxRange range("ispm plan create");
  if (!out)
    return fail(ISPM_ERR_INVALID, "out is NULL");
  *out = nullptr;
  if (int st = check_pair(vec_dtype, elm_dtype))
    return st;
  std::unique_ptr<ispm_plan> pl(new (std::nothrow) ispm_plan);
  if (!pl)
    return fail(ISPM_ERR_NOMEM, "host allocation");
  pl->vec_dtype = vec_dtype;
  pl->elm_dtype = elm_dtype;
  const bool upload = !(flags & ISPM_SPMV_PLAN_NO_DEVICE);
  try {
    if (kind == ISPM_PLAN_DEFAULT || kind == ISPM_PLAN_ESTIMATE) {
      ispm_slell *h = nullptr;
      if (int st = ispm_csr_to_slell_guess_format(elm_dtype, n_rows, n_cols, row_ptr, cols,
                                                  elms, 1, 4, &h))
        return st;
      pl->host.reset(h);
      const HostSlell &m = h->m;
      pl->mparams = ispm_slell_params{m.slice_height, m.hblock, (unsigned)m.var_height,
                                      (unsigned)m.diags};
      pl->params = default_launch(vec_dtype, m.view());
      if (upload) {
        pl->dev.reset(new ispm_dslell);
        if (int st = pl->dev->d.upload(m))
          return st;
      }
    } else if (kind == ISPM_PLAN_EXHAUSTIVE) {
      if (int st = plan_exhaustive(pl.get(), n_rows, n_cols, row_ptr, cols, elms))
        return st;
    } else {
      return fail(ISPM_ERR_INVALID, "plan kind %d", kind);
    }
  } catch (const std::bad_alloc &) {
    return fail(ISPM_ERR_NOMEM, "host allocation while planning");
  }
  *out = pl.release();
  return ISPM_OK;
}

int ispm_plan_execute(ispm_plan *p, const void *x, void *y, void *stream)
{
  clear_error();
  if (!p)
    return fail(ISPM_ERR_INVALID, "NULL plan");
  if (!p->dev)
    return fail(ISPM_ERR_INVALID, "plan has no device matrix (SPMV_PLAN_NO_DEVICE)");
  return launch_spmv(p->vec_dtype, p->params, p->dev->d.view(), x, y, (cudaStream_t)stream);
}

int ispm_plan_upload(ispm_plan *p)
{
  clear_error();
  if (!p || !p->host)
    return fail(ISPM_ERR_INVALID, "NULL plan or host matrix");
  std::unique_ptr<ispm_dslell> d(new (std::nothrow) ispm_dslell);
  if (!d)
    return fail(ISPM_ERR_NOMEM, "host allocation");
  if (int st = d->d.upload(p->host->m))
    return st;
  p->dev = std::move(d);
  return ISPM_OK;
}

int ispm_plan_update_device_matrix_coefs(ispm_plan *p)
{
  clear_error();
  if (!p || !p->host || !p->dev)
    return fail(ISPM_ERR_INVALID, "plan lacks a host or device matrix");
  return p->dev->d.update_elms(p->host->m);
}

int ispm_plan_change_host_matrix(ispm_plan *p, int n_rows, int n_cols, const int *row_ptr,
                                 const int *cols, const void *elms)
{
  clear_error();
  if (!p)
    return fail(ISPM_ERR_INVALID, "NULL plan");
  std::unique_ptr<ispm_slell> h(new (std::nothrow) ispm_slell);
  if (!h)
    return fail(ISPM_ERR_NOMEM, "host allocation");
  if (int st = convert_csr(p->elm_dtype, n_rows, n_cols, row_ptr, cols, elms, (int)p->mparams.S,
                           (int)p->mparams.H, p->mparams.V != 0, p->mparams.D != 0, 4, h->m))
    return st;
  p->host = std::move(h);
  p->drop_map();
  return ISPM_OK;
}

int ispm_plan_refresh_values(ispm_plan *p, int n_rows, const int *row_ptr, const int *cols,
                             const void *vals, int val_dtype, void *stream)
{
  clear_error();
  if (!p || !p->host || !p->dev)
    return fail(ISPM_ERR_INVALID, "plan lacks a host or device matrix");
  if (!row_ptr || n_rows < 0)
    return fail(ISPM_ERR_INVALID, "bad CSR pattern");
  const long long nnz = row_ptr[n_rows];
  if (!p->map || p->map_n != nnz) {
    p->drop_map();
    std::vector<int> inv;
    try {
      std::vector<unsigned> pos;
      if (int st = value_map(p->host->m, n_rows, row_ptr, cols, pos))
        return st;
      inv.assign((size_t)p->dev->d.meta.n_elms, -1);
      for (size_t k = 0; k < pos.size(); k++)
        inv[pos[k]] = (int)k;
    } catch (const std::bad_alloc &) {
      return fail(ISPM_ERR_NOMEM, "host allocation while mapping values");
    }
    ISPM_CUDA_TRY(cudaMalloc(&p->map, std::max<size_t>(inv.size(), 1) * sizeof(int)));
    if (!inv.empty())
      ISPM_CUDA_TRY(
          cudaMemcpy(p->map, inv.data(), inv.size() * sizeof(int), cudaMemcpyHostToDevice));
    p->map_n = nnz;
  }
  // slot order: coalesced writes, reads within each slice's CSR range
  return refresh_values_gather(p->dev->d, p->map, vals, val_dtype, (cudaStream_t)stream);
}

int ispm_plan_get_params(const ispm_plan *p, ispm_slell_params *mparams,
                         ispm_launch_params *params)
{
  if (!p)
    return fail(ISPM_ERR_INVALID, "NULL plan");
  if (mparams)
    *mparams = p->mparams;
  if (params)
    *params = p->params;
  return ISPM_OK;
}

ispm_slell *ispm_plan_host_matrix(ispm_plan *p) { return p ? p->host.get() : nullptr; }

const ispm_dslell *ispm_plan_device_matrix(const ispm_plan *p)
{
  return p ? p->dev.get() : nullptr;
}

double ispm_plan_tuned_seconds(const ispm_plan *p) { return p ? p->tuned : 0.0; }

void ispm_plan_free(ispm_plan *p) { delete p; }

}  // extern "C"
