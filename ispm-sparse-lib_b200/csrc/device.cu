// Device initialisation and device-resident sliced-ELL matrices.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "cuda_util.cuh"
#include "operator.h"
#include "spmv_launch.h"

namespace ispm {

int device_sm_count()
{
  static std::mutex mu;
  static int cached[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
    return 148;
  std::lock_guard<std::mutex> g(mu);
  if (!cached[dev]) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
      v = 148;
    cached[dev] = v;
  }
  return cached[dev];
}

static size_t elm_size(int dtype) { return dtype == ISPM_F64 ? 8 : dtype == ISPM_F32 ? 4 : 2; }

// Round to BF16, nearest even (finite values).
static uint16_t to_bf16(float f)
{
  uint32_t u;
  std::memcpy(&u, &f, 4);
  u += 0x7fffu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}

// ---- staged-walk tile records ----------------------------------------------

void stage_records(const HostSlell &h, std::vector<int> &rec)
{
  rec.clear();
  const unsigned S = h.slice_height;
  if (!h.diags || h.var_height || h.hblock != 1 || S < 16 || kStageTileRows % S || !h.n_slices)
    return;
  const unsigned spt = kStageTileRows / S;  // <= 16 slices per tile
  const unsigned n_tiles = (h.n_slices + spt - 1) / spt;
  rec.assign((size_t)n_tiles * kStageRecInts, 0);
  const unsigned *sp = h.slice_ptr.data();
  const long long rows = kStageTileRows;
  std::vector<long long> win, all;
  for (unsigned t = 0; t < n_tiles; t++) {
    int *r = rec.data() + (size_t)t * kStageRecInts;
    const unsigned b0 = t * spt, nsl = std::min(spt, h.n_slices - b0);
    r[2] = (int)nsl;
    // window starts of every slice's diagonals (slice b: [elms_end, cols_end,
    // diag_ptr] at 3b, conversion.h:393-402): the x column that tile row 0
    // would read, so x[w + t] serves tile row t (diag_pos is absolute)
    all.clear();
    bool ok = true, ell = false;
    for (unsigned s = 0; s < nsl; s++) {
      const unsigned b = b0 + s;
      const unsigned e0 = sp[3 * b], c0 = sp[3 * b + 1], e1 = sp[3 * b + 3], c1 = sp[3 * b + 4];
      ell = ell || c1 != c0;
      const unsigned nd = (e1 - e0 - (c1 - c0)) / S, dd = sp[3 * b + 2];
      for (unsigned k = 0; k < nd; k++) {
        const long long w = (long long)sp[dd + k] - S - (long long)s * S;
        if (k && w <= all.back())
          ok = false;
        all.push_back(w);
      }
    }
    win = all;
    std::sort(win.begin(), win.end());
    win.erase(std::unique(win.begin(), win.end()), win.end());
    const int nu = (int)win.size();
    const long long e_first = sp[3 * b0], e_count = (long long)sp[3 * (b0 + nsl)] - e_first;
    if (!ok || nu < 1 || nu > kStageMaxDiag || e_first > INT32_MAX || e_count > INT32_MAX)
      continue;  // r[0] = 0
    // runs of window starts less than rows + gap apart share a band; a band
    // covers its windows' columns for all tile rows, 16-byte aligned
    long long lo[kStageMaxDiag], hi[kStageMaxDiag];
    int band[kStageMaxDiag], nb = 0;
    for (int u = 0; u < nu; u++) {
      const long long w = win[u];
      if (u == 0 || w - win[u - 1] > rows + kStageGap) {
        lo[nb] = w;
        nb++;
      }
      hi[nb - 1] = w + rows;
      band[u] = nb - 1;
    }
    if (nb > kStageMaxBands || lo[0] < INT32_MIN / 2 || hi[nb - 1] > INT32_MAX / 2)
      continue;
    long long words = 0, dst[kStageMaxBands], c0[kStageMaxBands];
    for (int q = 0; q < nb; q++) {
      c0[q] = lo[q] >= 0 ? lo[q] / 4 * 4 : -((-lo[q] + 3) / 4) * 4;
      const long long c1 = (hi[q] + 3) / 4 * 4;
      dst[q] = words;
      r[156 + 2 * q] = (int)c0[q];
      r[157 + 2 * q] = (int)(c1 - c0[q]);
      words += c1 - c0[q];
    }
    if (words > kStageMaxXWords)
      continue;
    r[1] = nu;
    for (int u = 0; u < nu; u++)
      r[8 + u] = (int)(dst[band[u]] + (win[u] - c0[band[u]]));
    // slice masks over the window starts, slice element offsets; uniform
    // when every slice carries all nu windows and no explicit columns
    bool uniform = !ell;
    for (unsigned s = 0; s < nsl; s++) {
      const unsigned b = b0 + s;
      const unsigned e0 = sp[3 * b], c0s = sp[3 * b + 1], e1 = sp[3 * b + 3],
                     c1s = sp[3 * b + 4];
      const unsigned nd = (e1 - e0 - (c1s - c0s)) / S, dd = sp[3 * b + 2];
      unsigned long long mask = 0;
      for (unsigned k = 0; k < nd; k++) {
        const long long w = (long long)sp[dd + k] - S - (long long)s * S;
        const int u = (int)(std::lower_bound(win.begin(), win.end(), w) - win.begin());
        mask |= 1ull << u;
      }
      uniform = uniform && (int)nd == nu;
      r[72 + 2 * s] = (int)(unsigned)(mask & 0xffffffffull);
      r[73 + 2 * s] = (int)(unsigned)(mask >> 32);
      r[104 + s] = (int)((long long)e0 + (c1s - c0s) - e_first);
      r[120 + s] = (int)((c1s - c0s) / S);
      r[136 + s] = (int)c0s;
    }
    r[0] = uniform ? 1 : 2;
    r[152] = (int)e_first;
    r[153] = (int)e_count;
    r[154] = nb;
    r[155] = (int)words;
  }
}


namespace {
struct StageEntry {
  const int *rec;
  int max_x_words;
  int max_elms;
  unsigned n_slices;
};
std::mutex g_stage_mu;
std::vector<std::pair<const unsigned *, StageEntry>> g_stage;  // few live matrices
}  // namespace

bool find_stage_records(const unsigned *slice_ptr, unsigned n_slices, StageInfo &out)
{
  std::lock_guard<std::mutex> g(g_stage_mu);
  for (const auto &e : g_stage)
    if (e.first == slice_ptr && e.second.n_slices == n_slices) {
      out.rec = e.second.rec;
      out.max_x_words = e.second.max_x_words;
      out.max_elms = e.second.max_elms;
      return true;
    }
  return false;
}

int DeviceSlell::attach_stage_records(const HostSlell &h)
{
  std::vector<int> rec;
  stage_records(h, rec);
  if (rec.empty())
    return ISPM_OK;
  int mx = 0, me = 0;
  for (size_t t = 0; t < rec.size(); t += kStageRecInts)
    if (rec[t]) {
      mx = std::max(mx, rec[t + 155]);
      me = std::max(me, rec[t + 153]);
    }
  cudaError_t e = cudaMalloc(&stage_rec, rec.size() * sizeof(int));
  if (e != cudaSuccess) {
    stage_rec = nullptr;
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? ISPM_ERR_NOMEM : ISPM_ERR_CUDA,
                "cudaMalloc(stage records): %s", cudaGetErrorString(e));
  }
  ISPM_CUDA_TRY(cudaMemcpy(stage_rec, rec.data(), rec.size() * sizeof(int),
                           cudaMemcpyHostToDevice));
  std::lock_guard<std::mutex> g(g_stage_mu);
  g_stage.push_back({slice_ptr, StageEntry{stage_rec, mx, me, meta.n_slices}});
  return ISPM_OK;
}

void DeviceSlell::release()
{
  if (stage_rec) {
    {
      std::lock_guard<std::mutex> g(g_stage_mu);
      for (size_t k = 0; k < g_stage.size(); k++)
        if (g_stage[k].second.rec == stage_rec) {
          g_stage.erase(g_stage.begin() + (long)k);
          break;
        }
    }
    cudaFree(stage_rec);
    stage_rec = nullptr;
  }
  if (slice_ptr)
    cudaFree(slice_ptr);
  if (cols)
    cudaFree(cols);
  if (elms)
    cudaFree(elms);
  slice_ptr = nullptr;
  cols = nullptr;
  elms = nullptr;
}

int DeviceSlell::upload(const HostSlell &h, bool bf16_values)
{
  release();
  meta = h.view();
  if (bf16_values && h.elm_dtype != ISPM_F32)
    return fail(ISPM_ERR_INVALID, "BF16 storage converts an FP32 element array");
  const int store = bf16_values ? ISPM_BF16 : h.elm_dtype;
  meta.elm_dtype = store;
  const size_t nsp = h.slice_ptr.size(), nc = h.cols.size(), ne = h.n_elms();
  // The reference zero-fills every device allocation (util/cuda/allocator.h:14-20);
  // here every byte is overwritten by the copy that follows.
  auto alloc = [](void **p, size_t bytes) -> int {
    cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
    if (e != cudaSuccess) {
      *p = nullptr;
      cudaGetLastError();
      return fail(e == cudaErrorMemoryAllocation ? ISPM_ERR_NOMEM : ISPM_ERR_CUDA,
                  "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
    }
    return ISPM_OK;
  };
  int st;
  if ((st = alloc((void **)&slice_ptr, nsp * 4)) || (st = alloc((void **)&cols, nc * 4)) ||
      (st = alloc(&elms, ne * elm_size(store)))) {
    release();
    return st;
  }
  ISPM_CUDA_TRY(cudaMemcpy(slice_ptr, h.slice_ptr.data(), nsp * 4, cudaMemcpyHostToDevice));
  if (nc)
    ISPM_CUDA_TRY(cudaMemcpy(cols, h.cols.data(), nc * 4, cudaMemcpyHostToDevice));
  if (ne && bf16_values) {
    std::vector<uint16_t> b(ne);
    for (size_t k = 0; k < ne; k++)
      b[k] = to_bf16(h.elms_f[k]);
    ISPM_CUDA_TRY(cudaMemcpy(elms, b.data(), ne * 2, cudaMemcpyHostToDevice));
  } else if (ne) {
    ISPM_CUDA_TRY(
        cudaMemcpy(elms, h.elms_ptr(), ne * elm_size(h.elm_dtype), cudaMemcpyHostToDevice));
  }
  return attach_stage_records(h);
}

int DeviceSlell::upload_f16(const HostSlell &h)
{
  if (h.elm_dtype != ISPM_F32)
    return fail(ISPM_ERR_INVALID, "FP16 storage converts an FP32 element array");
  // the structure arrays travel unchanged, the elements as binary16
  std::vector<uint16_t> b(h.n_elms());
  for (size_t k = 0; k < b.size(); k++) {
    const double v = h.elms_f[k];
    b[k] = f16_bits(v);
    if (f16_value(b[k]) != v)
      return fail(ISPM_ERR_INVALID, "element %zu (%g) is not a binary16 value", k, v);
  }
  release();
  meta = h.view();
  meta.elm_dtype = ISPM_F16;
  const size_t nsp = h.slice_ptr.size(), nc = h.cols.size(), ne = b.size();
  auto alloc = [](void **p, size_t bytes) -> int {
    cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
    if (e != cudaSuccess) {
      *p = nullptr;
      cudaGetLastError();
      return fail(e == cudaErrorMemoryAllocation ? ISPM_ERR_NOMEM : ISPM_ERR_CUDA,
                  "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
    }
    return ISPM_OK;
  };
  int st;
  if ((st = alloc((void **)&slice_ptr, nsp * 4)) || (st = alloc((void **)&cols, nc * 4)) ||
      (st = alloc(&elms, ne * 2))) {
    release();
    return st;
  }
  ISPM_CUDA_TRY(cudaMemcpy(slice_ptr, h.slice_ptr.data(), nsp * 4, cudaMemcpyHostToDevice));
  if (nc)
    ISPM_CUDA_TRY(cudaMemcpy(cols, h.cols.data(), nc * 4, cudaMemcpyHostToDevice));
  if (ne)
    ISPM_CUDA_TRY(cudaMemcpy(elms, b.data(), ne * 2, cudaMemcpyHostToDevice));
  return attach_stage_records(h);
}

int DeviceSlell::update_elms(const HostSlell &h)
{
  if (!elms && meta.n_elms)
    return fail(ISPM_ERR_INVALID, "device matrix not uploaded");
  if ((long long)h.n_elms() != meta.n_elms || h.elm_dtype != meta.elm_dtype)
    return fail(ISPM_ERR_INVALID, "element array shape changed (%zu vs %lld)", h.n_elms(),
                meta.n_elms);
  if (meta.n_elms)
    ISPM_CUDA_TRY(cudaMemcpy(elms, h.elms_ptr(), meta.n_elms * elm_size(h.elm_dtype),
                             cudaMemcpyHostToDevice));
  return ISPM_OK;
}

// elms[map[k]] = vals[k]: new values for an unchanged sparsity pattern,
// written straight into the device sliced-ELL array.  Padding slots are not
// in the map and keep their zeros.
template <class E, class V>
__global__ void refresh_values_kernel(E *__restrict__ elms, const unsigned *__restrict__ map,
                                      const V *__restrict__ vals, long long n)
{
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x)
    elms[__ldcs(map + k)] = (E)__ldcs(vals + k);
}

template <class V>
__global__ void refresh_bf16_kernel(__nv_bfloat16 *__restrict__ elms,
                                    const unsigned *__restrict__ map, const V *__restrict__ vals,
                                    long long n)
{
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x)
    elms[__ldcs(map + k)] = __float2bfloat16_rn((float)__ldcs(vals + k));
}

template <class E, class V>
__global__ void refresh_gather_kernel(E *__restrict__ elms, const int *__restrict__ inv,
                                      const V *__restrict__ vals, long long n)
{
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const int src = __ldcs(inv + k);
    elms[k] = src >= 0 ? (E)__ldg(vals + src) : E(0);
  }
}

int refresh_values_gather(DeviceSlell &d, const int *inv, const void *vals, int val_dtype,
                          cudaStream_t s)
{
  const long long n = d.meta.n_elms;
  if (!n)
    return ISPM_OK;
  const int threads = 256;
  const long long blocks =
      std::min<long long>((n + threads - 1) / threads, (long long)device_sm_count() * 16);
  const bool e32 = d.meta.elm_dtype == ISPM_F32, v32 = val_dtype == ISPM_F32;
  if (d.meta.elm_dtype != ISPM_F32 && d.meta.elm_dtype != ISPM_F64)
    return fail(ISPM_ERR_INVALID, "slot-order refresh of an element type %d", d.meta.elm_dtype);
  if (e32 && v32)
    refresh_gather_kernel<float, float><<<blocks, threads, 0, s>>>((float *)d.elms, inv,
                                                                   (const float *)vals, n);
  else if (e32)
    refresh_gather_kernel<float, double><<<blocks, threads, 0, s>>>((float *)d.elms, inv,
                                                                    (const double *)vals, n);
  else if (v32)
    refresh_gather_kernel<double, float><<<blocks, threads, 0, s>>>((double *)d.elms, inv,
                                                                    (const float *)vals, n);
  else
    refresh_gather_kernel<double, double><<<blocks, threads, 0, s>>>((double *)d.elms, inv,
                                                                     (const double *)vals, n);
  cudaError_t e = cudaPeekAtLastError();
  return e == cudaSuccess ? ISPM_OK
                          : fail(ISPM_ERR_CUDA, "value refresh: %s", cudaGetErrorString(e));
}

// elms[map[k]] = FP16(vals[k] * scale), rounded to nearest.
__global__ void refresh_f16_kernel(__half *__restrict__ elms, const unsigned *__restrict__ map,
                                   const double *__restrict__ vals, long long n, double scale)
{
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x)
    elms[__ldcs(map + k)] = __double2half(__ldcs(vals + k) * scale);
}

// *out = max |v_k| as the bit pattern of a non-negative double (which orders
// like an unsigned integer); *out must start at 0.
__global__ void absmax_kernel(const double *__restrict__ v, long long n, unsigned long long *out)
{
  double m = 0.0;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x)
    m = fmax(m, fabs(v[k]));
  for (int off = 16; off > 0; off >>= 1)
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0)
    atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

int device_absmax(const double *vals, long long n, double &out)
{
  out = 0.0;
  if (!n)
    return ISPM_OK;
  unsigned long long *d = nullptr;
  ISPM_CUDA_TRY(cudaMalloc(&d, sizeof(unsigned long long)));
  unsigned long long h = 0;
  cudaError_t e = cudaMemset(d, 0, sizeof(h));
  if (e == cudaSuccess) {
    const long long blocks = std::min<long long>((n + 255) / 256, (long long)device_sm_count() * 8);
    absmax_kernel<<<blocks, 256>>>(vals, n, d);
    e = cudaPeekAtLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess)
    return fail(ISPM_ERR_CUDA, "absolute maximum: %s", cudaGetErrorString(e));
  std::memcpy(&out, &h, sizeof(out));
  return ISPM_OK;
}

int refresh_values_f16(DeviceSlell &d, const unsigned *map, const double *vals, long long n,
                       double scale, cudaStream_t s)
{
  if (d.meta.elm_dtype != ISPM_F16)
    return fail(ISPM_ERR_INVALID, "scaled FP16 refresh of an element type %d", d.meta.elm_dtype);
  if (!n)
    return ISPM_OK;
  const long long blocks = std::min<long long>((n + 255) / 256, (long long)device_sm_count() * 8);
  refresh_f16_kernel<<<blocks, 256, 0, s>>>((__half *)d.elms, map, vals, n, scale);
  cudaError_t e = cudaPeekAtLastError();
  return e == cudaSuccess ? ISPM_OK
                          : fail(ISPM_ERR_CUDA, "value refresh: %s", cudaGetErrorString(e));
}

int refresh_values(DeviceSlell &d, const unsigned *map, const void *vals, int val_dtype,
                   long long n, cudaStream_t s)
{
  if (d.meta.elm_dtype == ISPM_F16)
    return fail(ISPM_ERR_INVALID, "FP16 elements are refreshed with their scale");
  if (!n)
    return ISPM_OK;
  const int threads = 256;
  long long blocks = (n + threads - 1) / threads;
  blocks = std::min<long long>(blocks, (long long)device_sm_count() * 8);
  const bool e32 = d.meta.elm_dtype == ISPM_F32, v32 = val_dtype == ISPM_F32;
  if (d.meta.elm_dtype == ISPM_BF16 && v32)
    refresh_bf16_kernel<float><<<blocks, threads, 0, s>>>((__nv_bfloat16 *)d.elms, map,
                                                          (const float *)vals, n);
  else if (d.meta.elm_dtype == ISPM_BF16)
    refresh_bf16_kernel<double><<<blocks, threads, 0, s>>>((__nv_bfloat16 *)d.elms, map,
                                                           (const double *)vals, n);
  else if (e32 && v32)
    refresh_values_kernel<float, float><<<blocks, threads, 0, s>>>((float *)d.elms, map,
                                                                   (const float *)vals, n);
  else if (e32)
    refresh_values_kernel<float, double><<<blocks, threads, 0, s>>>((float *)d.elms, map,
                                                                    (const double *)vals, n);
  else if (v32)
    refresh_values_kernel<double, float><<<blocks, threads, 0, s>>>((double *)d.elms, map,
                                                                    (const float *)vals, n);
  else
    refresh_values_kernel<double, double><<<blocks, threads, 0, s>>>((double *)d.elms, map,
                                                                     (const double *)vals, n);
  cudaError_t e = cudaPeekAtLastError();
  return e == cudaSuccess ? ISPM_OK
                          : fail(ISPM_ERR_CUDA, "value refresh: %s", cudaGetErrorString(e));
}

static unsigned pow2_floor(unsigned v) { return v ? 1u << ilog2(v) : 0u; }
static unsigned pow2_ceil(unsigned v) { return v <= 1 ? 1u : 1u << (ilog2(v - 1) + 1); }

ispm_launch_params default_launch(int x_dtype, const ispm_slell_view &m)
{
  return register_walk_launch(x_dtype, m);
}

ispm_launch_params register_walk_launch(int x_dtype, const ispm_slell_view &m)
{
  (void)x_dtype;
  ispm_launch_params p{};
  const unsigned esz = m.elm_dtype == ISPM_F64 ? 8 : m.elm_dtype == ISPM_F32 ? 4 : 2;
  const unsigned hmax = m.var_height ? m.min_slice_height : m.slice_height;
  // one 128-bit load of elements per thread and step, at most 4 rows
  unsigned H = std::min(16u / esz, 4u);
  while (H > 1 && H > hmax)
    H >>= 1;
  const unsigned S = m.var_height ? m.max_slice_height : m.slice_height;
  unsigned R = S / H ? S / H : 1;
  // Enough threads to fill the GPU, split a row between several threads
  // only when rows alone do not.
  const double avg_width = m.n_rows ? (double)m.n_elms / (double)m.n_rows : 1.0;
  const double want_threads = 148.0 * 2048.0;
  const double row_threads = (double)m.n_rows / H;
  unsigned P = 1;
  if (row_threads < want_threads)
    P = pow2_ceil((unsigned)(want_threads / (row_threads > 1 ? row_threads : 1)));
  unsigned pmax = pow2_floor((unsigned)(avg_width / (m.hblock ? m.hblock : 1)));
  if (pmax < 1)
    pmax = 1;
  if (P > pmax)
    P = pmax;
  while (R * P > 1024 && P > 1)
    P >>= 1;
  unsigned N = R * P;
  if (N < 4)
    N = 4;
  while (N > 1024 && H < 4 && H * 2 <= hmax) {  // very tall slices: more rows per thread
    H *= 2;
    N = (S / H) * P;
  }
  p.N = N;
  p.S = m.var_height ? N * H : m.slice_height;
  if (m.var_height && p.S < H)
    p.S = H;
  p.H = H;
  p.use_tex_sliceptr = 1;
  p.use_tex_x = 1;
  return p;
}

}  // namespace ispm

using namespace ispm;

extern "C" {

int ispm_initialize(void)
{
  clear_error();
  int dev = 0;
  ISPM_CUDA_TRY(cudaGetDevice(&dev));
  int major = 0, minor = 0;
  ISPM_CUDA_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
  ISPM_CUDA_TRY(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev));
  if (major != 10 || minor != 0)
    return fail(ISPM_ERR_ARCH, "compiled for sm_100a, device %d is sm_%d%d", dev, major, minor);
  // The reference sets cudaDeviceMapHost (initialize.cu:28).  Once a context is
  // active the flag can no longer change; mapped host memory is on by default
  // with unified addressing, so that refusal is not an error.
  cudaError_t e = cudaSetDeviceFlags(cudaDeviceMapHost);
  if (e != cudaSuccess && e != cudaErrorSetOnActiveProcess)
    return fail(ISPM_ERR_CUDA, "cudaSetDeviceFlags: %s", cudaGetErrorString(e));
  cudaGetLastError();
  return ISPM_OK;
}

int ispm_get_device_string(char *buf, int len)
{
  clear_error();
  if (!buf || len <= 0)
    return fail(ISPM_ERR_INVALID, "NULL buffer");
  int dev = 0;
  ISPM_CUDA_TRY(cudaGetDevice(&dev));
  cudaDeviceProp p;
  ISPM_CUDA_TRY(cudaGetDeviceProperties(&p, dev));
  snprintf(buf, (size_t)len, "%04x:%02x:%02x (%s)", p.pciDomainID, p.pciBusID, p.pciDeviceID,
           p.name);
  return ISPM_OK;
}

int ispm_dslell_upload(const ispm_slell *h, ispm_dslell **out)
{
  clear_error();
  if (!h || !out)
    return fail(ISPM_ERR_INVALID, "NULL argument");
  *out = nullptr;
  ispm_dslell *d = new (std::nothrow) ispm_dslell;
  if (!d)
    return fail(ISPM_ERR_NOMEM, "host allocation");
  int st = d->d.upload(h->m);
  if (st) {
    delete d;
    return st;
  }
  *out = d;
  return ISPM_OK;
}

int ispm_dslell_upload_f16(const ispm_slell *h, ispm_dslell **out)
{
  clear_error();
  if (!h || !out)
    return fail(ISPM_ERR_INVALID, "NULL argument");
  *out = nullptr;
  ispm_dslell *d = new (std::nothrow) ispm_dslell;
  if (!d)
    return fail(ISPM_ERR_NOMEM, "host allocation");
  int st = d->d.upload_f16(h->m);
  if (st) {
    delete d;
    return st;
  }
  *out = d;
  return ISPM_OK;
}

int ispm_slell_stage_records(const ispm_slell *m, int *out, long long cap, long long *n_ints)
{
  clear_error();
  if (!m || !n_ints || (cap > 0 && !out))
    return fail(ISPM_ERR_INVALID, "NULL argument");
  std::vector<int> rec;
  stage_records(m->m, rec);
  *n_ints = (long long)rec.size();
  for (long long k = 0; k < cap && k < (long long)rec.size(); k++)
    out[k] = rec[(size_t)k];
  return ISPM_OK;
}

int ispm_dslell_update_elms(ispm_dslell *d, const ispm_slell *h)
{
  clear_error();
  if (!d || !h)
    return fail(ISPM_ERR_INVALID, "NULL argument");
  return d->d.update_elms(h->m);
}

int ispm_dslell_get_view(const ispm_dslell *d, ispm_slell_view *view)
{
  if (!d || !view)
    return fail(ISPM_ERR_INVALID, "NULL argument");
  *view = d->d.view();
  return ISPM_OK;
}

void ispm_dslell_free(ispm_dslell *d) { delete d; }

int ispm_dslell_refresh_values(ispm_dslell *d, const unsigned *map, const void *vals,
                               int val_dtype, int n_nz, void *stream)
{
  clear_error();
  if (!d || (n_nz && (!map || !vals)) || n_nz < 0)
    return fail(ISPM_ERR_INVALID, "bad arguments");
  if (val_dtype != ISPM_F32 && val_dtype != ISPM_F64)
    return fail(ISPM_ERR_INVALID, "val_dtype %d", val_dtype);
  if (n_nz != d->d.meta.n_nz)
    return fail(ISPM_ERR_INVALID, "%d values for a matrix of %d non-zeros", n_nz,
                d->d.meta.n_nz);
  return refresh_values(d->d, map, vals, val_dtype, n_nz, (cudaStream_t)stream);
}

int ispm_default_launch(int x_dtype, const ispm_slell_view *m, ispm_launch_params *out)
{
  clear_error();
  if (!m || !out)
    return fail(ISPM_ERR_INVALID, "NULL argument");
  *out = default_launch(x_dtype, *m);
  return check_launch(x_dtype, *out, *m);
}

}  // extern "C"
