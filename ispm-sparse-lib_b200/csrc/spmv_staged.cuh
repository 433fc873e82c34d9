// Staged diagonal walk of the sliced-ELL SpMV: FP32 vectors, diagonal-block
// matrices of fixed slice height, selected by the launch shape N = S, H = 1.
// Included by spmv.cu (uses its SpmvArgs and fused-dot finishers).
//
// In the reference walk (cuda/spmv/kernel.h:80-92) the thread of local row r
// reads x[diag_pos + r - S] for every diagonal of its slice.  Here a CTA of
// 256 threads takes a tile of kStageTileRows = 1024 rows, each thread four
// consecutive rows of one slice, so every element load is one 16-byte (FP32)
// or 8-byte (FP16 / BF16) vector of a diagonal's column-major block.  The
// tile's x windows -- the window starts w of all its slices' diagonals, x[w
// + t] serving tile row t -- are merged into bands that the CTA copies into
// shared memory once (16-byte loads, zero outside x).  A thread's four x
// values then sit in two aligned 16-byte shared-memory chunks, shifted by
// the window's start modulo 4; the host groups the windows by that shift, so
// each group's realignment is fixed at compile time.  In the common tile,
// every slice carries every window and an entry names the diagonal
// directly, so the element loads of a group are independent and the
// compiler batches them; tiles whose slices differ (grid faces) take a mask
// per slice over the tile's windows (its k-th diagonal is its k-th set
// bit).  All of this is computed on the host when the matrix is uploaded
// (stage_records), so a CTA's set-up is one coalesced load of its record
// beside its slice header.  Tiles with more than 64 windows, more than 8
// bands or bands beyond the buffer read x through the read-only path with
// bounds tests.

constexpr int kStageThreads = 256;
constexpr int kStageMaxChunks = 4;  // 16-byte band chunks a thread copies per pass

// x[w + t .. w + t + 3] from the two chunks holding it (shift M = (smem
// start of x[w + t]) mod 4)
template <int M> __device__ __forceinline__ float4 realign(const float4 a, const float4 b)
{
  if constexpr (M == 0)
    return a;
  else if constexpr (M == 1)
    return make_float4(a.y, a.z, a.w, b.x);
  else if constexpr (M == 2)
    return make_float4(a.z, a.w, b.x, b.y);
  else
    return make_float4(a.w, b.x, b.y, b.z);
}

template <int M, class E>
__device__ __forceinline__ void stage_fma(const Vec<4, E> &e, const float4 *__restrict__ xs4,
                                          int q, float (&acc)[4])
{
  const float4 a = xs4[q];
  const float4 b = M ? xs4[q + 1] : a;
  const float4 xv = realign<M>(a, b);
  acc[0] = fmaf(float(e.v[0]), xv.x, acc[0]);
  acc[1] = fmaf(float(e.v[1]), xv.y, acc[1]);
  acc[2] = fmaf(float(e.v[2]), xv.z, acc[2]);
  acc[3] = fmaf(float(e.v[3]), xv.w, acc[3]);
}

// A group of a uniform tile: entry i names diagonal k directly.
template <int M, class E>
__device__ __forceinline__ void group_uniform(const int *__restrict__ rec, int beg, int end,
                                              const E *__restrict__ ep, unsigned S,
                                              const float4 *__restrict__ xs4, int tid,
                                              float (&acc)[4])
{
  int i = beg;
  for (; i + 4 <= end; i += 4) {
    int vv[4];
#pragma unroll
    for (int j = 0; j < 4; j++)
      vv[j] = rec[32 + i + j];
    Vec<4, E> e[4];
#pragma unroll
    for (int j = 0; j < 4; j++)
      e[j] = ld_stream<4>(ep + (size_t)(unsigned)(vv[j] >> 24) * S);
#pragma unroll
    for (int j = 0; j < 4; j++)
      stage_fma<M>(e[j], xs4, ((vv[j] & 0xffffff) >> 2) + tid, acc);
  }
  for (; i < end; i++) {
    const int v = rec[32 + i];
    stage_fma<M>(ld_stream<4>(ep + (size_t)(unsigned)(v >> 24) * S), xs4,
                 ((v & 0xffffff) >> 2) + tid, acc);
  }
}

// A group of a tile whose slices differ: bit u of the slice's mask says
// whether it has window u, its diagonal index is the rank of u in the mask.
template <int M, class E>
__device__ __forceinline__ void group_masked(const int *__restrict__ rec, int beg, int end,
                                             unsigned long long mask, const E *__restrict__ ep,
                                             unsigned S, const float4 *__restrict__ xs4, int tid,
                                             float (&acc)[4])
{
  for (int i = beg; i < end; i++) {
    const int v = rec[32 + i];
    const int u = v >> 24;
    if ((mask >> u) & 1ull) {
      const int k = __popcll(mask & ((1ull << u) - 1ull));
      stage_fma<M>(ld_stream<4>(ep + (size_t)k * S), xs4, ((v & 0xffffff) >> 2) + tid, acc);
    }
  }
}

template <class E>
__global__ void __launch_bounds__(kStageThreads, 5)
    slell_spmv_staged_kernel(SpmvArgs<float, E> a, const int *__restrict__ recs)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float *xs = reinterpret_cast<float *>(smem_raw);
  const float4 *xs4 = reinterpret_cast<const float4 *>(smem_raw);
  __shared__ __align__(16) int rec[kStageRecInts];

  const unsigned S = a.slice_height;
  const int tid = (int)threadIdx.x;
  const unsigned spt = kStageTileRows / S;
  const unsigned tile = blockIdx.x;
  if (tid < kStageRecInts)
    rec[tid] = __ldg(recs + (size_t)tile * kStageRecInts + tid);
  // this thread's four rows: tile rows 4 tid .. 4 tid + 3 of slice s
  const unsigned t0 = 4u * (unsigned)tid;
  const unsigned s = t0 / S, r = t0 & (S - 1);
  const unsigned b = tile * spt + s;
  const bool act = b < a.n_slices;
  // slice header [elms_end, cols_end, diag_ptr] (conversion.h:393-402)
  const unsigned *h = a.sp + 3 * (size_t)(act ? b : tile * spt);
  const unsigned e0 = __ldg(h), c0 = __ldg(h + 1);
  const unsigned e1 = __ldg(h + 3), c1 = __ldg(h + 4);
  const E *__restrict__ ep = a.elms + e0 + (c1 - c0) + r;  // first diagonal element

  pdl_wait();
  if (a.skip && *a.skip)
    return;
  __syncthreads();  // rec
  const int kind = rec[2] <= a.stage_words ? rec[0] : 0;
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
  if (kind) {
    // copy the bands, 16-byte chunks: chunk g lies in the band whose running
    // total passes g
    const int nb = rec[1];
    const int n = (int)a.n_cols;
    const int nch_total = rec[5 + 3 * (nb - 1)];
    for (int g0 = 0; g0 < nch_total; g0 += kStageThreads * kStageMaxChunks) {
      float4 v[kStageMaxChunks];
      int dst[kStageMaxChunks];
#pragma unroll
      for (int i = 0; i < kStageMaxChunks; i++) {
        const int g = g0 + i * kStageThreads + tid;
        dst[i] = -1;
        if (g >= nch_total)
          continue;
        int q = 0;
        while (g >= rec[5 + 3 * q])
          q++;
        const int c = g - (q ? rec[5 + 3 * (q - 1)] : 0);
        const int col = rec[4 + 3 * q] + 4 * c;
        dst[i] = rec[6 + 3 * q] + 4 * c;
        if (a.x_al16 && col >= 0 && col + 4 <= n) {
          v[i] = __ldg(reinterpret_cast<const float4 *>(a.x + col));
        } else {
          v[i].x = (col >= 0 && col < n) ? __ldg(a.x + col) : 0.f;
          v[i].y = (col + 1 >= 0 && col + 1 < n) ? __ldg(a.x + col + 1) : 0.f;
          v[i].z = (col + 2 >= 0 && col + 2 < n) ? __ldg(a.x + col + 2) : 0.f;
          v[i].w = (col + 3 >= 0 && col + 3 < n) ? __ldg(a.x + col + 3) : 0.f;
        }
      }
#pragma unroll
      for (int i = 0; i < kStageMaxChunks; i++)
        if (dst[i] >= 0)
          *reinterpret_cast<float4 *>(xs + dst[i]) = v[i];
    }
    __syncthreads();
    if (kind == 1) {
      if (act) {
        group_uniform<0>(rec, 0, rec[28], ep, S, xs4, tid, acc);
        group_uniform<1>(rec, rec[28], rec[29], ep, S, xs4, tid, acc);
        group_uniform<2>(rec, rec[29], rec[30], ep, S, xs4, tid, acc);
        group_uniform<3>(rec, rec[30], rec[31], ep, S, xs4, tid, acc);
      }
    } else {
      const unsigned long long mask =
          act ? ((unsigned long long)(unsigned)rec[97 + 2 * s] << 32) | (unsigned)rec[96 + 2 * s]
              : 0ull;
      group_masked<0>(rec, 0, rec[28], mask, ep, S, xs4, tid, acc);
      group_masked<1>(rec, rec[28], rec[29], mask, ep, S, xs4, tid, acc);
      group_masked<2>(rec, rec[29], rec[30], mask, ep, S, xs4, tid, acc);
      group_masked<3>(rec, rec[30], rec[31], mask, ep, S, xs4, tid, acc);
    }
  } else if (act) {
    // read-only-path walk of the slice (kernel.h:80-92)
    const unsigned nd = (e1 - e0 - (c1 - c0)) / S;
    const unsigned d0 = __ldg(h + 2);
    const unsigned adj = r - S;
#pragma unroll 2
    for (unsigned k = 0; k < nd; k++) {
      const Vec<4, E> e = ld_stream<4>(ep + (size_t)k * S);
      const unsigned base = __ldg(a.sp + d0 + k) + adj;
#pragma unroll
      for (int j = 0; j < 4; j++)
        acc[j] = fmaf(float(e.v[j]), ld_x_guard(a.x, base + j, a.n_cols), acc[j]);
    }
  }
  // entries off the slice's diagonals, with explicit columns (kernel.h:70-79)
  const unsigned nell = act ? (c1 - c0) / S : 0u;
  for (unsigned jj = 0; jj < nell; jj++) {
    const size_t q = (size_t)jj * S + r;
    const Vec<4, E> e = ld_stream<4>(a.elms + e0 + q);
    const Vec<4, unsigned> cc = ld_stream<4>(a.cols + c0 + q);
#pragma unroll
    for (int j = 0; j < 4; j++)
      acc[j] = fmaf(float(e.v[j]), ld_x_guard(a.x, cc.v[j], a.n_cols), acc[j]);
  }

  pdl_trigger();
  const unsigned row = tile * kStageTileRows + t0;
  if constexpr (std::is_same<E, __half>::value) {
    // FP16 elements: y = inv_scale * (stored sum), plus diag * x for a split
    if (act) {
      if (a.dg) {
        const float4 dg = __ldcs(reinterpret_cast<const float4 *>(a.dg + row));
        acc[0] = fmaf(dg.x, ld_x_guard(a.x, row, a.n_cols), acc[0] * a.inv_scale);
        acc[1] = fmaf(dg.y, ld_x_guard(a.x, row + 1, a.n_cols), acc[1] * a.inv_scale);
        acc[2] = fmaf(dg.z, ld_x_guard(a.x, row + 2, a.n_cols), acc[2] * a.inv_scale);
        acc[3] = fmaf(dg.w, ld_x_guard(a.x, row + 3, a.n_cols), acc[3] * a.inv_scale);
      } else {
#pragma unroll
        for (int j = 0; j < 4; j++)
          acc[j] *= a.inv_scale;
      }
    }
  }
  if (act)
    *reinterpret_cast<float4 *>(a.y + row) = make_float4(acc[0], acc[1], acc[2], acc[3]);
  if (a.ep.out) {
    double dv = 0.0, dw = 0.0;
    const bool two = a.ep.out2 != nullptr;
    if (act) {
      const float4 vv =
          *reinterpret_cast<const float4 *>(static_cast<const float *>(a.ep.v) + row);
      const float w[4] = {vv.x, vv.y, vv.z, vv.w};
#pragma unroll
      for (int j = 0; j < 4; j++) {
        dv = fma((double)acc[j], (double)w[j], dv);
        if (two)
          dw = fma((double)w[j], (double)w[j], dw);
      }
    }
    if (two)
      finish_dot2(dv, dw, a.ep);
    else
      finish_dot(dv, a.ep);
  }
}

// The staged walk serves this launch: FP32 vectors, diagonal blocks, fixed
// slice height in [16, 1024] dividing the tile, the shape N = S, H = 1,
// 16-byte aligned matrix arrays and y, and tile records registered for the
// matrix.
bool staged_shape(int x_dtype, const ispm_launch_params &p, const ispm_slell_view &m,
                  const void *y, StageInfo &si)
{
  return x_dtype == ISPM_F32 && m.diags && !m.var_height && m.hblock == 1 && p.H == 1 &&
         p.N == m.slice_height && m.slice_height >= 16 &&
         kStageTileRows % m.slice_height == 0 && aligned(m.elms, 16) &&
         aligned(m.cols, 16) && aligned(y, 16) && find_stage_records(m.slice_ptr, m.n_slices, si);
}

template <class E>
int launch_staged(SpmvArgs<float, E> args, const StageInfo &si, cudaStream_t stream)
{
  const unsigned spt = kStageTileRows / args.slice_height;
  const unsigned grid = (args.n_slices + spt - 1) / spt;
  // the largest band footprint over the matrix's tiles, at most 40 KB (with
  // the static record the CTA stays inside the 48 KB a launch gets without
  // opting in to more); tiles over it read x directly
  const size_t smem = std::min<size_t>((size_t)si.max_words * sizeof(float), 40960);
  args.stage_words = (int)(smem / sizeof(float));
  cudaError_t e = launch_kernel(slell_spmv_staged_kernel<E>, dim3(grid), dim3(kStageThreads),
                                smem, stream, args.pdl != 0, args, si.rec);
  if (e == cudaSuccess)
    e = cudaPeekAtLastError();
  if (e != cudaSuccess)
    return fail(ISPM_ERR_CUDA, "SpMV launch: %s", cudaGetErrorString(e));
  return ISPM_OK;
}
