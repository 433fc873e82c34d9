// Staged diagonal walk of the sliced-ELL SpMV: the launch shape N = S, H = 1
// on diagonal-block matrices of fixed slice height.  Included by spmv.cu
// (uses its SpmvArgs and fused-dot finishers).
//
// In the reference walk (cuda/spmv/kernel.h:80-92) the thread of local row r
// reads x[diag_pos + r - S] for every diagonal of its slice.  Here a CTA of
// 256 threads takes a tile of kStageTileRows = 1024 rows, each thread the four
// rows tid, tid + 256, tid + 512, tid + 768 (every access of a warp stays
// coalesced).  When every slice of the tile carries the same diagonal offsets
// (diag_pos minus the slice's first row), the tile's x windows are the
// intervals [w_k, w_k + 1024) of one set of window starts w_k; runs of nearby
// windows form bands, which the CTA copies into shared memory once (16-byte
// loads, zero outside x).  The walk is then one streaming element load, one
// shared-memory load and one FMA per entry.  Which tiles stage, their bands
// and every window's shared-memory start are computed on the host when the
// matrix is uploaded (stage_records), so a CTA's set-up is one coalesced
// load of its 384-byte record next to its rows' slice headers and first
// elements (issued before the programmatic-launch wait: the matrix does not
// depend on the predecessor kernel), then the band copy.  Tiles whose slices
// differ (grid faces) or whose bands exceed the buffer read x through the
// read-only path with bounds tests, as the register walk does.

constexpr int kStageThreads = 256;
constexpr int kStageRowsPerThread = kStageTileRows / kStageThreads;  // 4
constexpr int kStageMaxChunks = 4;   // 16-byte band chunks a thread copies per pass

template <class T, class E>
__global__ void __launch_bounds__(kStageThreads, sizeof(T) == 8 ? 4 : 5)
    slell_spmv_staged_kernel(SpmvArgs<T, E> a, const int *__restrict__ recs)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *xs = reinterpret_cast<T *>(smem_raw);
  __shared__ __align__(16) int rec[kStageRecInts];
  constexpr int R = kStageRowsPerThread;
  constexpr int VW = 16 / (int)sizeof(T);

  const unsigned S = a.slice_height;
  const unsigned tid = threadIdx.x;
  const unsigned spt = kStageTileRows / S;
  const unsigned tile = blockIdx.x;
  if (tid < (unsigned)kStageRecInts)
    rec[tid] = __ldg(recs + (size_t)tile * kStageRecInts + tid);

  // this thread's rows: slice headers [elms_end, cols_end, diag_ptr]
  // (conversion.h:393-402) and the first diagonal's elements
  // (the other header fields are read again, from L1, where they are needed)
  unsigned ed[R], nd[R];
  E pre[R];
#pragma unroll
  for (int j = 0; j < R; j++) {
    const unsigned t = tid + (unsigned)j * kStageThreads;
    const unsigned b = tile * spt + t / S;
    const bool act = b < a.n_slices;
    const unsigned *h = a.sp + 3 * (size_t)(act ? b : tile * spt);
    const unsigned e0 = __ldg(h), c0 = __ldg(h + 1), e1 = __ldg(h + 3), c1 = __ldg(h + 4);
    ed[j] = e0 + (c1 - c0) + (t & (S - 1));  // this row's first diagonal element
    nd[j] = act ? (e1 - e0 - (c1 - c0)) / S : 0u;
    pre[j] = nd[j] ? ld_stream<1>(a.elms + ed[j]).v[0] : E(0.0f);
  }

  pdl_wait();
  if (a.skip && *a.skip)
    return;
  __syncthreads();  // rec
  const bool staged = rec[0] && rec[2] <= a.stage_words;
  const int n = (int)a.n_cols;
  if (staged) {
    // copy the bands: chunk g of the tile's concatenated bands, 16 bytes each
    const int nb = rec[1];
    int nch_total = 0;
    for (int q = 0; q < nb; q++) {
      const int lo = rec[4 + 3 * q], hi = rec[5 + 3 * q];
      const int c0q = lo >= 0 ? lo / VW * VW : -((-lo + VW - 1) / VW) * VW;
      nch_total += (hi - c0q + VW - 1) / VW;
    }
    for (int g0 = 0; g0 < nch_total; g0 += kStageThreads * kStageMaxChunks) {
      T v[kStageMaxChunks][VW];
      int dst[kStageMaxChunks];
#pragma unroll
      for (int i = 0; i < kStageMaxChunks; i++) {
        const int g = g0 + i * kStageThreads + (int)tid;
        dst[i] = -1;
        if (g >= nch_total)
          continue;
        int q = 0, base = 0, c0q = 0, nch = 0;
        for (;; q++) {
          const int lo = rec[4 + 3 * q], hi = rec[5 + 3 * q];
          c0q = lo >= 0 ? lo / VW * VW : -((-lo + VW - 1) / VW) * VW;
          nch = (hi - c0q + VW - 1) / VW;
          if (g < base + nch || q + 1 == nb)
            break;
          base += nch;
        }
        const int c = g - base;
        const int col = c0q + c * VW;
        dst[i] = rec[6 + 3 * q] - (rec[4 + 3 * q] - c0q) + c * VW;
        if (a.x_al16 && col >= 0 && col + VW <= n) {
          if constexpr (sizeof(T) == 4) {
            const float4 f = __ldg(reinterpret_cast<const float4 *>(a.x + col));
            v[i][0] = f.x;
            v[i][1] = f.y;
            v[i][2] = f.z;
            v[i][3] = f.w;
          } else {
            const double2 f = __ldg(reinterpret_cast<const double2 *>(a.x + col));
            v[i][0] = f.x;
            v[i][1] = f.y;
          }
        } else {
#pragma unroll
          for (int u = 0; u < VW; u++) {
            const int cc = col + u;
            v[i][u] = (cc >= 0 && cc < n) ? __ldg(a.x + cc) : T(0);
          }
        }
      }
#pragma unroll
      for (int i = 0; i < kStageMaxChunks; i++) {
        if (dst[i] < 0)
          continue;
        if constexpr (sizeof(T) == 4)
          *reinterpret_cast<float4 *>(xs + dst[i]) =
              make_float4(v[i][0], v[i][1], v[i][2], v[i][3]);
        else
          *reinterpret_cast<double2 *>(xs + dst[i]) = make_double2(v[i][0], v[i][1]);
      }
    }
    __syncthreads();
  }

  T acc[R];
#pragma unroll
  for (int j = 0; j < R; j++)
    acc[j] = T(0);
  if (staged) {
    // every active row of the tile walks the same nd0 diagonals
    const int nd0 = rec[3];
#pragma unroll
    for (int j = 0; j < R; j++)
      if (nd[j])
        acc[j] = fma(T(pre[j]), xs[rec[28] + (int)(tid + j * kStageThreads)], acc[j]);
#pragma unroll 2
    for (int k = 1; k < nd0; k++) {
      const int sx = rec[28 + k];
      const size_t step = (size_t)k * S;
#pragma unroll
      for (int j = 0; j < R; j++)
        if (nd[j])
          acc[j] = fma(T(ld_stream<1>(a.elms + ed[j] + step).v[0]),
                       xs[sx + (int)(tid + j * kStageThreads)], acc[j]);
    }
  } else {
    // read-only-path walk of each row's own slice (kernel.h:80-92)
#pragma unroll
    for (int j = 0; j < R; j++) {
      if (!nd[j])
        continue;
      const unsigned t = tid + j * kStageThreads;
      const unsigned d0 = __ldg(a.sp + 3 * (size_t)(tile * spt + t / S) + 2);
      const unsigned adj = (t & (S - 1)) - S;
      acc[j] = fma(T(pre[j]), ld_x_guard(a.x, __ldg(a.sp + d0) + adj, a.n_cols), acc[j]);
      for (unsigned k = 1; k < nd[j]; k++)
        acc[j] = fma(T(ld_stream<1>(a.elms + ed[j] + (size_t)k * S).v[0]),
                     ld_x_guard(a.x, __ldg(a.sp + d0 + k) + adj, a.n_cols), acc[j]);
    }
  }
  // entries off the slice's diagonals, with explicit columns (kernel.h:70-79)
#pragma unroll
  for (int j = 0; j < R; j++) {
    const unsigned t = tid + j * kStageThreads;
    const unsigned b = tile * spt + t / S;
    if (b >= a.n_slices)
      continue;
    const unsigned *h = a.sp + 3 * (size_t)b;
    const unsigned e0 = __ldg(h), c0 = __ldg(h + 1), c1 = __ldg(h + 4);
    const unsigned r = t & (S - 1);
    for (unsigned jj = 0; jj < (c1 - c0) / S; jj++) {
      const size_t q = (size_t)jj * S + r;
      acc[j] = fma(T(ld_stream<1>(a.elms + e0 + q).v[0]),
                   ld_x_guard(a.x, ld_stream<1>(a.cols + c0 + q).v[0], a.n_cols), acc[j]);
    }
  }

  pdl_trigger();
  double dv = 0.0, dw = 0.0;
  const bool two = a.ep.out2 != nullptr;
#pragma unroll
  for (int j = 0; j < R; j++) {
    const unsigned t = tid + j * kStageThreads;
    const bool act = tile * spt + t / S < a.n_slices;
    const unsigned row = tile * kStageTileRows + t;
    if constexpr (std::is_same<E, __half>::value) {
      // FP16 elements: y = inv_scale * (stored sum), plus diag * x for a split
      if (act)
        acc[j] = a.dg ? fma(__ldcs(a.dg + row), ld_x_guard(a.x, row, a.n_cols),
                            acc[j] * a.inv_scale)
                      : acc[j] * a.inv_scale;
    }
    if (act) {
      a.y[row] = acc[j];
      if (a.ep.out) {
        const double vv = (double)static_cast<const T *>(a.ep.v)[row];
        dv = fma((double)acc[j], vv, dv);
        if (two)
          dw = fma(vv, vv, dw);
      }
    }
  }
  if (a.ep.out) {
    if (two)
      finish_dot2(dv, dw, a.ep);
    else
      finish_dot(dv, a.ep);
  }
}

// The staged walk serves this launch: diagonal blocks, fixed slice height
// dividing the tile, one row per thread and S threads per slice, and tile
// records registered for the matrix.
bool staged_shape(const ispm_launch_params &p, const ispm_slell_view &m, StageInfo &si)
{
  return m.diags && !m.var_height && m.hblock == 1 && p.H == 1 && p.N == m.slice_height &&
         m.slice_height >= 1 && kStageTileRows % m.slice_height == 0 &&
         find_stage_records(m.slice_ptr, m.n_slices, si);
}

template <class T, class E>
int launch_staged(SpmvArgs<T, E> args, const StageInfo &si, cudaStream_t stream)
{
  const unsigned spt = kStageTileRows / args.slice_height;
  const unsigned grid = (args.n_slices + spt - 1) / spt;
  // the largest band footprint over the matrix's tiles, at most 40 KB (with
  // the static record the CTA stays inside the 48 KB a launch gets without
  // opting in to more); tiles over it read x directly
  const size_t smem = std::min<size_t>((size_t)si.max_words * sizeof(T), 40960);
  args.stage_words = (int)(smem / sizeof(T));
  cudaError_t e = launch_kernel(slell_spmv_staged_kernel<T, E>, dim3(grid), dim3(kStageThreads),
                                smem, stream, args.pdl != 0, args, si.rec);
  if (e == cudaSuccess)
    e = cudaPeekAtLastError();
  if (e != cudaSuccess)
    return fail(ISPM_ERR_CUDA, "SpMV launch: %s", cudaGetErrorString(e));
  return ISPM_OK;
}
