// Staged diagonal walk of the sliced-ELL SpMV: FP32 vectors, diagonal-block
// matrices of fixed slice height, selected by the launch shape N = S, H = 1.
// Included by spmv.cu (uses its SpmvArgs and fused-dot finishers).
//
// In the reference walk (cuda/spmv/kernel.h:80-92) the thread of local row r
// reads x[diag_pos + r - S] for every diagonal of its slice, two dependent
// loads per element on the critical path.  Here asynchronous copies feed the
// FMAs: a persistent CTA per SM takes a contiguous run of 256-row tiles;
// copy warps move each tile's record, its elements (one contiguous range: a
// tile's slices are consecutive in elms) and the bands of x its windows read
// (zero outside x) into a ring of shared-memory slots with 16-byte cp.async
// copies, each copy lane's copies completing on the slot's mbarrier
// (cp.async.mbarrier.arrive.noinc); compute warps take the tiles in turn,
// each lane eight rows (t = lane + 32 j), reading every element and x value
// from shared memory with conflict-free 32-bit loads, and hand the slot back
// through a second mbarrier.  The element copies of the first slots go out
// before the programmatic-launch wait (the matrix is final before the
// previous kernel starts), the x copies after it.  The copy warps keep up to
// `slots` tiles in flight, so the bytes in flight per SM are set by shared
// memory, not by registers or warps.  (Measured on this walk: the bulk-copy
// engine, cp.async.bulk, moves about 17 bytes per cycle per SM, and one
// warp's 16-byte lane copies about 7, against the 25 an SM's share of HBM
// needs; hence several copy warps.)
//
// Every wait on an mbarrier is bounded (about 2^31 clock cycles): on a
// timeout the CTA records a fault code in g_stage_fault and stops issuing
// and waiting; the copy lanes wait for their own copies before the CTA
// exits.  The host reads and clears the code with ispm_spmv_stage_fault().

constexpr int kStageConsumers = 4;                     // compute warps
constexpr int kStageProducers = 4;                     // copy warps
constexpr int kStageThreads = 32 * (kStageConsumers + kStageProducers);
constexpr unsigned kStageCopyLanes = 32u * kStageProducers;
constexpr int kStageMaxSlots = 8;
constexpr int kStageSmemBudget = 220 * 1024;           // dynamic shared memory for the ring
constexpr int kStageRecBytes = kStageRecComputeInts * 4;

__device__ unsigned g_stage_fault;  // 0, or the first timeout's code (1 consumer, 2 producer)

__device__ __forceinline__ unsigned smem_u32(const void *p)
{
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned b, unsigned count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(b), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned b)
{
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(b) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned b, unsigned parity)
{
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n"
      " mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(b), "r"(parity)
      : "memory");
  return ok != 0;
}
// Phase `parity` of barrier b completed: true; false once about 2^31 clock
// cycles passed or (abort != NULL) the CTA gave up.
__device__ __forceinline__ bool mbar_wait(unsigned b, unsigned parity, const volatile int *abort)
{
  if (mbar_try_wait(b, parity))
    return true;
  const long long t0 = clock64();
  for (;;) {
    if (mbar_try_wait(b, parity))
      return true;
    if ((abort && *abort) || clock64() - t0 > (1ll << 31))
      return false;
  }
}
// 16-byte global -> shared copy (16-byte aligned addresses); the bytes past
// the first src_bytes (0..16) are zero and not read.
__device__ __forceinline__ void cp16(unsigned dst, const void *src, unsigned src_bytes)
{
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src),
               "r"(src_bytes)
               : "memory");
}
// One arrival on barrier b once every earlier cp.async of this thread has
// landed (the barrier's count includes it).
__device__ __forceinline__ void cp_arrive(unsigned b)
{
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(b) : "memory");
}
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ void stage_fault(unsigned code, volatile int *abort)
{
  atomicCAS(&g_stage_fault, 0u, code);
  *abort = 1;
}

template <class E>
__global__ void __launch_bounds__(kStageThreads, 1)
    slell_spmv_staged_kernel(SpmvArgs<float, E> a, const int *__restrict__ recs)
{
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) unsigned long long full_bar[kStageMaxSlots];
  __shared__ __align__(8) unsigned long long empty_bar[kStageMaxSlots];
  __shared__ int abort_flag;
  volatile int *abort = &abort_flag;

  const int warp = (int)(threadIdx.x >> 5), lane = (int)(threadIdx.x & 31);
  const unsigned S = a.slice_height, spt = kStageTileRows / S;
  const unsigned n_tiles = (a.n_slices + spt - 1) / spt;
  const unsigned t_beg = (unsigned)((unsigned long long)blockIdx.x * n_tiles / gridDim.x);
  const unsigned t_end = (unsigned)((unsigned long long)(blockIdx.x + 1) * n_tiles / gridDim.x);
  const unsigned cnt = t_end - t_beg;
  const unsigned NS = (unsigned)a.st_slots, slot_bytes = (unsigned)a.st_slot_bytes;
  const unsigned x_off = (unsigned)a.st_x_off;
  const unsigned ring = smem_u32(smem);
  if (threadIdx.x == 0) {
    for (unsigned s = 0; s < NS; s++) {
      mbar_init(smem_u32(&full_bar[s]), kStageCopyLanes);  // the copy warps' lanes
      mbar_init(smem_u32(&empty_bar[s]), 1);  // the consuming warp
    }
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  double dv = 0.0, dw = 0.0;
  const bool two = a.ep.out2 != nullptr;
  if (warp >= kStageConsumers) {
    // ---- copy warps ----------------------------------------------------------
    // copy lane c (of kStageCopyLanes) moves 16-byte chunks c, c + lanes, ...
    const unsigned cpl = 32u * (unsigned)(warp - kStageConsumers) + (unsigned)lane;
    // copy lists: lane l of every copy warp holds the one of tile (batch base
    // + l); this batch in cl, the next one in nx
    int cl[20] = {}, nx[20] = {};
    auto load_cl = [&](int(&d)[20], unsigned base) {
      const unsigned tl = t_beg + base + (unsigned)lane;
      if (tl < t_end) {
        const int4 *p = reinterpret_cast<const int4 *>(recs + (size_t)tl * kStageRecInts +
                                                       kStageRecComputeInts);
#pragma unroll
        for (int k = 0; k < 5; k++) {
          const int4 v = __ldg(p + k);
          d[4 * k] = v.x;
          d[4 * k + 1] = v.y;
          d[4 * k + 2] = v.z;
          d[4 * k + 3] = v.w;
        }
      } else {
#pragma unroll
        for (int f = 0; f < 20; f++)
          d[f] = 0;
      }
    };
    // record + elements of tile i into its slot, 16 bytes a lane and step
    auto issue_elms = [&](unsigned i) {
      const int src = (int)(i & 31u);
      const unsigned e_first = (unsigned)__shfl_sync(0xffffffffu, cl[0], src);
      const unsigned e_cnt = (unsigned)__shfl_sync(0xffffffffu, cl[1], src);
      const unsigned dst = ring + (i % NS) * slot_bytes;
      const char *rs = reinterpret_cast<const char *>(recs + (size_t)(t_beg + i) * kStageRecInts);
      for (unsigned o = 16u * cpl; o < (unsigned)kStageRecBytes; o += 16u * kStageCopyLanes)
        cp16(dst + o, rs + o, 16);
      const char *es = reinterpret_cast<const char *>(a.elms + e_first);
      const unsigned eb = e_cnt * (unsigned)sizeof(E);
      for (unsigned o = 16u * cpl; o < eb; o += 16u * kStageCopyLanes)
        cp16(dst + kStageRecBytes + o, es + o, 16);
    };
    // the tile's x bands (columns outside x read zero), then each lane's
    // arrival on the slot once its copies of the tile have landed
    auto issue_x = [&](unsigned i) {
      const int src = (int)(i & 31u);
      const int nb = __shfl_sync(0xffffffffu, cl[2], src);
      const unsigned slot = i % NS;
      const unsigned xb = ring + slot * slot_bytes + x_off;
      const int n = (int)a.n_cols;
      int d = 0;
#pragma unroll
      for (int q = 0; q < kStageMaxBands; q++) {
        const int c = __shfl_sync(0xffffffffu, cl[4 + 2 * q], src);
        const int w = __shfl_sync(0xffffffffu, cl[5 + 2 * q], src);
        if (q < nb) {
          for (int k = 4 * (int)cpl; k < w; k += 4 * (int)kStageCopyLanes) {
            const int col = c + k;  // a multiple of 4: no chunk straddles column 0
            const int valid = (col < 0 || col >= n) ? 0 : (n - col >= 4 ? 4 : n - col);
            cp16(xb + 4u * (unsigned)(d + k), a.x + (valid ? col : 0), 4u * (unsigned)valid);
          }
          d += w;
        }
      }
      cp_arrive(smem_u32(&full_bar[slot]));
    };

    load_cl(cl, 0);
    load_cl(nx, 32);
    const unsigned pre = cnt < NS ? cnt : NS;
    for (unsigned i = 0; i < pre; i++)
      issue_elms(i);
    pdl_wait();
    if (a.skip && *a.skip) {
      cp_wait_all();  // no copy into this CTA's shared memory outlives it
      return;
    }
    for (unsigned i = 0; i < cnt; i++) {
      if (i && (i & 31u) == 0) {
#pragma unroll
        for (int f = 0; f < 20; f++)
          cl[f] = nx[f];
        load_cl(nx, i + 32);
      }
      if (i >= pre) {
        if (!mbar_wait(smem_u32(&empty_bar[i % NS]), ((i / NS) - 1) & 1u, abort)) {
          if (lane == 0)
            stage_fault(2, abort);
          break;
        }
        issue_elms(i);
      }
      issue_x(i);
    }
    cp_wait_all();
    pdl_trigger();
  } else {
    // ---- consumers -----------------------------------------------------------
    pdl_wait();
    if (a.skip && *a.skip)
      return;
    for (unsigned i = (unsigned)warp; i < cnt; i += kStageConsumers) {
      const unsigned slot = i % NS;
      if (!mbar_wait(smem_u32(&full_bar[slot]), (i / NS) & 1u, abort)) {
        if (lane == 0)
          stage_fault(1, abort);
        break;
      }
      const unsigned char *sl = smem + slot * slot_bytes;
      const int *rc = reinterpret_cast<const int *>(sl);
      const E *el = reinterpret_cast<const E *>(sl + kStageRecBytes);
      const float *xs = reinterpret_cast<const float *>(sl + x_off);
      const unsigned tile = t_beg + i;
      const int kind = rc[0], nu = rc[1];
      const unsigned rows = (unsigned)rc[2] * S;
      const unsigned row0 = tile * kStageTileRows;
      // rows lane + 32 j; past the tile's last row, read a valid row's
      // operands (the result is not stored)
      unsigned tt[8];
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const unsigned t = (unsigned)lane + 32u * j;
        tt[j] = t < rows ? t : rows - 1;
      }
      // epilogue operands from global memory, in flight during the walk
      float vj[8], dj[8], xj[8];
#pragma unroll
      for (int j = 0; j < 8; j++) {
        vj[j] = dj[j] = xj[j] = 0.f;
        if (a.ep.out)
          vj[j] = static_cast<const float *>(a.ep.v)[row0 + tt[j]];
        if constexpr (std::is_same<E, __half>::value) {
          if (a.dg) {
            dj[j] = __ldcs(a.dg + row0 + tt[j]);
            xj[j] = ld_x_guard(a.x, row0 + tt[j], a.n_cols);
          }
        }
      }
      float acc[8];
#pragma unroll
      for (int j = 0; j < 8; j++)
        acc[j] = 0.f;
      if (kind == 1) {
        // every slice carries all nu windows: element of (row t, window u)
        // at (t / S) nu S + u S + t mod S
        const E *ep[8];
#pragma unroll
        for (int j = 0; j < 8; j++)
          ep[j] = el + (tt[j] / S) * (unsigned)nu * S + (tt[j] & (S - 1));
        for (int u = 0; u < nu; u++) {
          const float *xu = xs + rc[8 + u];
          const unsigned eo = (unsigned)u * S;
#pragma unroll
          for (int j = 0; j < 8; j++)
            acc[j] = fmaf(float(ep[j][eo]), xu[tt[j]], acc[j]);
        }
      } else if (kind == 2) {
        // slices differ: the k-th set bit of the slice's mask is its k-th
        // diagonal
        unsigned long long mk[8];
        const E *ep[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
          const unsigned s = tt[j] / S;
          mk[j] = ((unsigned long long)(unsigned)rc[73 + 2 * s] << 32) | (unsigned)rc[72 + 2 * s];
          ep[j] = el + rc[104 + s] + (tt[j] & (S - 1));
        }
        for (int u = 0; u < nu; u++) {
          const float *xu = xs + rc[8 + u];
#pragma unroll
          for (int j = 0; j < 8; j++)
            if ((mk[j] >> u) & 1ull) {
              acc[j] = fmaf(float(*ep[j]), xu[tt[j]], acc[j]);
              ep[j] += S;
            }
        }
        // entries with explicit columns (kernel.h:70-79): elements staged
        // before the slice's diagonals, columns and x from global memory
#pragma unroll
        for (int j = 0; j < 8; j++) {
          const unsigned s = tt[j] / S, r = tt[j] & (S - 1);
          const int ne = rc[120 + s];
          const E *ee = el + rc[104 + s] - ne * (int)S + r;
          const unsigned *cc = a.cols + (unsigned)rc[136 + s] + r;
          for (int q = 0; q < ne; q++)
            acc[j] = fmaf(float(ee[q * S]), ld_x_guard(a.x, __ldg(cc + q * S), a.n_cols), acc[j]);
        }
      }
      __syncwarp();
      if (lane == 0)
        mbar_arrive(smem_u32(&empty_bar[slot]));
      if (kind == 0) {
        // not staged: the slice walk from global memory (kernel.h:70-92)
#pragma unroll
        for (int j = 0; j < 8; j++) {
          const unsigned t = tt[j];
          const unsigned b = tile * spt + t / S, r = t & (S - 1);
          const unsigned *h = a.sp + 3 * (size_t)b;
          const unsigned e0 = __ldg(h), c0 = __ldg(h + 1), d0 = __ldg(h + 2);
          const unsigned e1 = __ldg(h + 3), c1 = __ldg(h + 4);
          float s = 0.f;
          for (unsigned q = 0; q < c1 - c0; q += S)
            s = fmaf(float(a.elms[e0 + q + r]), ld_x_guard(a.x, __ldg(a.cols + c0 + q + r), a.n_cols),
                     s);
          const unsigned nd = (e1 - e0 - (c1 - c0)) / S;
          for (unsigned k = 0; k < nd; k++)
            s = fmaf(float(a.elms[e0 + (c1 - c0) + k * S + r]),
                     ld_x_guard(a.x, __ldg(a.sp + d0 + k) + r - S, a.n_cols), s);
          acc[j] = s;
        }
      }
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const unsigned t = (unsigned)lane + 32u * j;
        if (t < rows) {
          float yv = acc[j];
          if constexpr (std::is_same<E, __half>::value)
            yv = a.dg ? fmaf(dj[j], xj[j], yv * a.inv_scale) : yv * a.inv_scale;
          a.y[row0 + t] = yv;
          if (a.ep.out) {
            dv = fma((double)yv, (double)vj[j], dv);
            if (two)
              dw = fma((double)vj[j], (double)vj[j], dw);
          }
        }
      }
    }
    pdl_trigger();
  }
  if (a.ep.out) {
    if (two)
      finish_dot2(dv, dw, a.ep);
    else
      finish_dot(dv, a.ep);
  }
}

// The staged walk serves this launch: FP32 vectors, diagonal blocks, fixed
// slice height in [16, 256], the shape N = S, H = 1, x 16-byte aligned,
// tile records registered for the matrix and at least three ring slots
// within the shared-memory budget.
bool staged_shape(int x_dtype, const ispm_launch_params &p, const ispm_slell_view &m,
                  const void *x, StageInfo &si, int &slots, int &slot_bytes, int &x_off)
{
  if (!(x_dtype == ISPM_F32 && m.diags && !m.var_height && m.hblock == 1 && p.H == 1 &&
        p.N == m.slice_height && m.slice_height >= 16 && kStageTileRows % m.slice_height == 0 &&
        aligned(x, 16) && find_stage_records(m.slice_ptr, m.n_slices, si)))
    return false;
  const long long esz = m.elm_dtype == ISPM_F32 ? 4 : 2;
  const long long eb = ((long long)si.max_elms * esz + 15) / 16 * 16;
  const long long bytes = kStageRecBytes + eb + 4ll * si.max_x_words;
  const long long ns = std::min<long long>(kStageMaxSlots, kStageSmemBudget / bytes);
  if (ns < 3)
    return false;
  slots = (int)ns;
  slot_bytes = (int)bytes;
  x_off = (int)(kStageRecBytes + eb);
  return true;
}

template <class E>
int launch_staged(SpmvArgs<float, E> args, const StageInfo &si, cudaStream_t stream)
{
  const unsigned spt = kStageTileRows / args.slice_height;
  const unsigned n_tiles = (args.n_slices + spt - 1) / spt;
  const unsigned grid = std::min<unsigned>(n_tiles, (unsigned)device_sm_count());
  const size_t smem = (size_t)args.st_slots * (size_t)args.st_slot_bytes;
  // the ring needs the opt-in shared-memory size, set once per device
  static std::atomic<unsigned long long> opted{0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess && (dev < 0 || dev >= 64 || !((opted.load() >> dev) & 1ull))) {
    e = cudaFuncSetAttribute(slell_spmv_staged_kernel<E>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, kStageSmemBudget);
    if (e == cudaSuccess && dev >= 0 && dev < 64)
      opted.fetch_or(1ull << dev);
  }
  if (e == cudaSuccess && grid)
    e = launch_kernel(slell_spmv_staged_kernel<E>, dim3(grid), dim3(kStageThreads), smem, stream,
                      args.pdl != 0, args, si.rec);
  if (e == cudaSuccess)
    e = cudaPeekAtLastError();
  if (e != cudaSuccess)
    return fail(ISPM_ERR_CUDA, "SpMV launch: %s", cudaGetErrorString(e));
  return ISPM_OK;
}
