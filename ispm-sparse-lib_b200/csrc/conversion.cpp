// CSR -> sliced-ELLPACK conversion (host).
//
// Produces exactly the layout of the reference's csr_to_slell
// (formats/conversion.h:338-414) and the format choice of
// csr_to_slell_guess_format (conversion.h:416-492), so that matrices, plans and
// kernels agree bit for bit with the reference.  The work is organised
// differently: a sequential pass fixes slice boundaries, a parallel pass sizes
// every slice (padding width, hblock split, diagonal set), a prefix sum turns
// sizes into offsets and a second parallel pass fills the slices in place.
#include <algorithm>
#include <atomic>
#include <climits>
#include <cstring>
#include <mutex>

#include "host_pool.h"
#include "ispm_internal.h"

namespace ispm {
namespace {

constexpr int kPadRows = 512;       // conversion.h:2 MAX_SLICE_HEIGHT, the pad() granule
constexpr int kMinSliceHeight = 32;  // conversion.h:2 MIN_SLICE_HEIGHT

// CSR rows with the reference's padding applied virtually: rows at or past
// the caller's row count are empty.
struct CsrRows {
  int n_src;  // caller's rows
  int n_pad;  // rows after padding to kPadRows
  const int *rp;
  const int *ci;
  int begin(int r) const { return r < n_src ? rp[r] : rp[n_src]; }
  int end(int r) const { return r < n_src ? rp[r + 1] : rp[n_src]; }
  int len(int r) const { return end(r) - begin(r); }
};

unsigned floor_pow2(unsigned v) { return v ? 1u << (31 - __builtin_clz(v)) : 0u; }

// Variable slice height (conversion.h:6-47): grow the slice row by row while
// the padding stays under the waste budget and the slice under 4 elements per
// thread, then round down to a power of two.
int estimate_slice_height(const CsrRows &A, int cur_row, int n_rows, int n_threads,
                          int n_elms)
{
  const int kMaxWasteRatio = 100, kEltsPerThread = 4;
  // Same expression types as the reference: the budget is computed in double
  // and stored as float; the test below compares in float.
  float waste_per_row = 0.01 * n_elms * kMaxWasteRatio / n_rows;
  int height = 0, widest = 0, padding = 0, stored = 0;
  for (; height < n_threads && cur_row + height < n_rows; height++) {
    int len = A.len(cur_row + height);
    int new_stored = stored + len, new_padding;
    if (len > widest) {
      new_padding = padding + height * (len - widest);
    } else {
      new_padding = padding + widest - len;
      len = widest;
    }
    bool too_wasteful = height >= 32 && (float)new_padding > waste_per_row * (float)height;
    bool too_big = height >= 1 && new_stored + new_padding > n_threads * kEltsPerThread;
    if (too_wasteful || too_big)
      break;
    widest = len;
    padding = new_padding;
    stored = new_stored;
  }
  return (int)floor_pow2((unsigned)height);
}

// Diagonal discovery (conversion.h:234-284).  Candidate offsets come from the
// first longest row; an offset is accepted if every row that is still as long
// as the current longest remaining length holds it.  Appends the accepted
// positions (col - local_row + slice_size) and returns the ELL width left.
int find_diagonals(const CsrRows &A, int slice_size, int cur_row, std::vector<int> &diag_pos,
                   std::vector<int> &rowlen, std::vector<int> &rowpos)
{
  rowlen.resize(slice_size);
  rowpos.resize(slice_size);
  int longest = 0, longrow = cur_row;
  for (int k = 0; k < slice_size; k++) {
    int r = cur_row + k;
    rowlen[k] = A.len(r);
    rowpos[k] = A.begin(r);
    if (longest < rowlen[k]) {
      longest = rowlen[k];
      longrow = r;
    }
  }
  for (int e = A.begin(longrow); e < A.end(longrow); e++) {
    const int off = A.ci[e] - longrow;
    bool rejected = false;
    for (int k = 0; k < slice_size; k++) {
      const int r = cur_row + k, stop = A.end(r);
      int &pos = rowpos[k];
      while (pos < stop && A.ci[pos] - r < off)
        pos++;
      bool has = pos < stop && A.ci[pos] - r == off;
      if (!has && rowlen[k] == longest) {
        rejected = true;
        break;
      }
    }
    if (rejected)
      continue;
    diag_pos.push_back(A.ci[e] - (longrow - cur_row) + slice_size);
    longest--;
    for (int k = 0; k < slice_size; k++) {
      const int r = cur_row + k, pos = rowpos[k];
      if (pos < A.end(r) && A.ci[pos] - r == off)
        rowlen[k]--;
    }
  }
  return longest;
}

// hblock split cost model (conversion.h:83-108).
int hblk_maxslen(const int *slen, const int *blen, int n, int maxblen, int hblock)
{
  int widest = 0;
  for (int k = 0; k < n; k++) {
    int kept = std::min(maxblen, blen[k]);
    int singles = slen[k] - (maxblen - kept) + (blen[k] - kept) * hblock;
    widest = std::max(widest, singles);
  }
  return widest;
}

int hblk_cost(const int *slen, const int *blen, int n, int maxblen, int hblock, int smul,
              int bmul)
{
  return smul * hblk_maxslen(slen, blen, n, maxblen, hblock) + bmul * maxblen;
}

inline bool block_start(const CsrRows &A, int e, int stop, int W)
{
  return !(A.ci[e] & (W - 1)) && e + W - 1 < stop && A.ci[e + W - 1] - A.ci[e] == W - 1;
}

// Per-slice shape decided in the sizing pass.
struct SliceShape {
  int row0 = 0, height = 0;
  int ell = 0;     // ELL columns (plain / diagonal modes) or single columns (hblock)
  int blocks = 0;  // hblock columns
  int n_diag = 0;
  long long cols_off = 0, elms_off = 0, diag_off = 0;
};

// E is the matrix element type (it sizes the hblock cost model); V is what
// lands in the element array -- E itself, or the CSR entry number when a
// value-refresh map is built.
template <class E, class V = E> struct Converter {
  CsrRows A;
  const V *vals;
  int hblock;
  bool diags;
  std::vector<SliceShape> shapes;
  std::vector<std::vector<int>> slice_diags;
  unsigned *cols_out = nullptr;
  V *elms_out = nullptr;

  void size_slice(SliceShape &s, std::vector<int> &diag, std::vector<int> &t1,
                  std::vector<int> &t2) const
  {
    const int S = s.height, r0 = s.row0;
    if (diags) {
      s.ell = find_diagonals(A, S, r0, diag, t1, t2);
      s.n_diag = (int)diag.size();
      return;
    }
    if (hblock > 1) {
      // conversion.h:117-176: count single and block entries per row, then
      // pick the block width minimising the byte cost.
      const int W = hblock;
      t1.resize(S);
      t2.resize(S);
      int *slen = t1.data(), *blen = t2.data();
      int minblen = INT_MAX, maxblen = 0;
      for (int k = 0; k < S; k++) {
        const int r = r0 + k, stop = A.end(r);
        int ns = 0, nb = 0, e = A.begin(r);
        while (e + W - 1 < stop) {
          if (!(A.ci[e] & (W - 1)) && A.ci[e + W - 1] - A.ci[e] == W - 1) {
            nb++;
            e += W;
          } else {
            ns++;
            e++;
          }
        }
        ns += stop - e;
        slen[k] = ns;
        blen[k] = nb;
        maxblen = std::max(maxblen, nb);
        minblen = std::min(minblen, nb);
      }
      const int smul = (int)(sizeof(int) + sizeof(E));
      const int bmul = (int)(sizeof(int) + W * sizeof(E));
      while (maxblen - minblen >= 3) {
        int d = (maxblen - minblen) / 3;
        int b1 = minblen + d, b2 = b1 + d;
        int cost1 = hblk_cost(slen, blen, S, b1, W, smul, bmul);
        // The reference passes hblock and the single-entry multiplier in
        // swapped positions for the second probe (conversion.h:152-154);
        // kept so the chosen split matches.
        int cost2 = hblk_cost(slen, blen, S, b2, smul, W, bmul);
        if (cost1 <= cost2)
          maxblen = b2;
        else
          minblen = b1;
      }
      int best_cost = INT_MAX, best = INT_MAX;
      for (int b = minblen; b <= maxblen; b++) {
        int c = hblk_cost(slen, blen, S, b, W, smul, bmul);
        if (best_cost > c) {
          best_cost = c;
          best = b;
        }
      }
      s.blocks = best;
      s.ell = hblk_maxslen(slen, blen, S, best, W);
      return;
    }
    int widest = 0;
    for (int k = 0; k < S; k++)
      widest = std::max(widest, A.len(r0 + k));
    s.ell = widest;
  }

  long long cols_len(const SliceShape &s) const
  {
    return (long long)(s.ell + s.blocks) * s.height;
  }
  long long elms_len(const SliceShape &s) const
  {
    return (long long)(s.ell + s.blocks * hblock + s.n_diag) * s.height;
  }

  // Padding column = the same column of the row above (0 for the first row);
  // padding values stay 0 (conversion.h:73-79, 213-225, 326-333).
  void pad_col(long long base, int k, int S, int slot) const
  {
    long long at = base + k + (long long)slot * S;
    cols_out[at] = k ? cols_out[at - 1] : 0u;
  }

  void fill_slice(const SliceShape &s, const int *diag) const
  {
    const int S = s.height, r0 = s.row0;
    const long long co = s.cols_off, eo = s.elms_off;
    if (diags) {
      // conversion.h:286-336
      const long long ed = eo + (long long)s.ell * S;
      for (int k = 0; k < S; k++) {
        const int r = r0 + k;
        int di = 0, nc = 0;
        for (int e = A.begin(r); e < A.end(r); e++) {
          const int c = A.ci[e], d = c - k + S;
          while (di < s.n_diag && diag[di] < d)
            di++;
          if (di < s.n_diag && diag[di] == d) {
            elms_out[ed + k + (long long)di * S] = vals[e];
          } else {
            cols_out[co + k + (long long)nc * S] = (unsigned)c;
            elms_out[eo + k + (long long)nc * S] = vals[e];
            nc++;
          }
        }
        for (; nc < s.ell; nc++)
          pad_col(co, k, S, nc);
      }
      return;
    }
    if (hblock > 1) {
      // conversion.h:177-232
      const int W = hblock;
      const long long cb = co + (long long)s.ell * S, eb = eo + (long long)s.ell * S;
      for (int k = 0; k < S; k++) {
        const int r = r0 + k, stop = A.end(r);
        int ns = 0, nb = 0;
        for (int e = A.begin(r); e < stop;) {
          if (block_start(A, e, stop, W) && nb < s.blocks) {
            cols_out[cb + k + (long long)nb * S] = (unsigned)(A.ci[e] / W);
            for (int w = 0; w < W; w++)
              elms_out[eb + k + (long long)(nb * W + w) * S] = vals[e + w];
            nb++;
            e += W;
          } else if (ns < s.ell) {
            cols_out[co + k + (long long)ns * S] = (unsigned)A.ci[e];
            elms_out[eo + k + (long long)ns * S] = vals[e];
            ns++;
            e++;
          } else {
            // singles beyond the slice's single width go to a spare block slot
            cols_out[cb + k + (long long)nb * S] = (unsigned)(A.ci[e] / W);
            elms_out[eb + k + (long long)(nb * W + A.ci[e] % W) * S] = vals[e];
            nb++;
            e++;
          }
        }
        for (; ns < s.ell; ns++)
          pad_col(co, k, S, ns);
        for (; nb < s.blocks; nb++)
          pad_col(cb, k, S, nb);
      }
      return;
    }
    // conversion.h:49-81
    for (int k = 0; k < S; k++) {
      const int r = r0 + k;
      int slot = 0;
      for (int e = A.begin(r); e < A.end(r); e++, slot++) {
        cols_out[co + k + (long long)slot * S] = (unsigned)A.ci[e];
        elms_out[eo + k + (long long)slot * S] = vals[e];
      }
      for (; slot < s.ell; slot++)
        pad_col(co, k, S, slot);
    }
  }
};

template <class E, class V = E>
int convert_impl(int n_rows, int n_cols, const int *row_ptr, const int *cols, const V *vals,
                 int S_req, int hblock, bool var_height, bool use_diags, int min_height,
                 HostSlell &B, std::vector<V> &elms_vec)
{
  const long long n_pad64 = ((long long)n_rows + kPadRows - 1) / kPadRows * kPadRows;
  if (n_pad64 > INT_MAX)
    return fail(ISPM_ERR_TOO_LARGE, "padded row count %lld exceeds INT_MAX", n_pad64);
  const int n_pad = (int)n_pad64;
  const int nnz = row_ptr[n_rows];
  if (hblock > 1)
    use_diags = false;

  Converter<E, V> cv;
  cv.A = CsrRows{n_rows, n_pad, row_ptr, cols};
  cv.vals = vals;
  cv.hblock = hblock;
  cv.diags = use_diags;

  // Slice boundaries (conversion.h:379-388).
  if (var_height) {
    for (int r = 0; r < n_pad;) {
      int h = estimate_slice_height(cv.A, r, n_pad, S_req, nnz);
      if (h < min_height)
        h = min_height;
      SliceShape s;
      s.row0 = r;
      s.height = h;
      cv.shapes.push_back(s);
      r += h;
    }
    if (cv.shapes.size() && cv.shapes.back().row0 + cv.shapes.back().height > n_pad)
      return fail(ISPM_ERR_INVALID, "min_height %d does not tile the padded rows", min_height);
  } else {
    int h = S_req < min_height ? min_height : S_req;
    if (h != S_req)
      return fail(ISPM_ERR_INVALID, "slice height %d below min_height %d", S_req, min_height);
    if (n_pad % h)
      return fail(ISPM_ERR_INVALID, "slice height %d does not divide %d padded rows", h, n_pad);
    cv.shapes.resize(n_pad / h);
    for (size_t b = 0; b < cv.shapes.size(); b++) {
      cv.shapes[b].row0 = (int)b * h;
      cv.shapes[b].height = h;
    }
  }
  const long long n_slices = (long long)cv.shapes.size();
  if (use_diags)
    cv.slice_diags.resize(n_slices);

  // Sizing pass.
  parallel_for(n_slices, [&](long long lo, long long hi) {
    std::vector<int> t1, t2, scratch;
    for (long long b = lo; b < hi; b++) {
      std::vector<int> &dl = use_diags ? cv.slice_diags[b] : scratch;
      dl.clear();
      cv.size_slice(cv.shapes[b], dl, t1, t2);
    }
  });

  long long co = 0, eo = 0, dof = 0;
  unsigned max_h = 0, min_h = cv.shapes.empty() ? 0u : ~0u;
  for (auto &s : cv.shapes) {
    s.cols_off = co;
    s.elms_off = eo;
    s.diag_off = dof;
    co += cv.cols_len(s);
    eo += cv.elms_len(s);
    dof += s.n_diag;
    max_h = std::max(max_h, (unsigned)s.height);
    min_h = std::min(min_h, (unsigned)s.height);
  }
  const int per_slice = 1 + (hblock > 1) + (var_height ? 1 : 0) + (use_diags ? 2 : 0);
  const long long sp_len = (n_slices + 1) * per_slice + dof;
  if (co > UINT_MAX || eo > UINT_MAX || sp_len > UINT_MAX)
    return fail(ISPM_ERR_TOO_LARGE, "sliced-ELL arrays exceed 32-bit offsets");

  B.n_rows = n_pad;
  B.n_cols = n_cols;
  B.n_nz = nnz;
  B.slice_height = (unsigned)S_req;
  B.n_slices = (unsigned)n_slices;
  B.hblock = (unsigned)hblock;
  B.var_height = var_height;
  B.diags = use_diags;
  B.max_slice_height = max_h;
  B.min_slice_height = min_h;
  B.min_height_used = min_height;
  B.cols.assign(co, 0u);
  elms_vec.assign(eo, V(0));
  cv.cols_out = B.cols.data();
  cv.elms_out = elms_vec.data();

  parallel_for(n_slices, [&](long long lo, long long hi) {
    for (long long b = lo; b < hi; b++)
      cv.fill_slice(cv.shapes[b], use_diags ? cv.slice_diags[b].data() : nullptr);
  });

  // slice_ptr records (conversion.h:355-373, 393-402) and the diagonal list
  // appended behind them with record fields rebased to it (:405-412).
  B.slice_ptr.assign(sp_len, 0u);
  for (long long b = 0; b < n_slices; b++) {
    const SliceShape &s = cv.shapes[b];
    unsigned *rec = &B.slice_ptr[(b + 1) * per_slice];
    int f = 0;
    rec[f++] = (unsigned)(s.elms_off + cv.elms_len(s));
    if (var_height)
      rec[f++] = (unsigned)(s.row0 + s.height);
    if (hblock > 1)
      rec[f++] = (unsigned)(s.cols_off + cv.cols_len(s));
    if (use_diags) {
      rec[f++] = (unsigned)(s.cols_off + cv.cols_len(s));
      rec[f++] = (unsigned)(s.diag_off + s.n_diag);
    }
  }
  if (use_diags) {
    const unsigned base = (unsigned)((n_slices + 1) * per_slice);
    const int dfield = var_height ? 3 : 2;
    for (long long b = 0; b <= n_slices; b++)
      B.slice_ptr[b * per_slice + dfield] += base;
    parallel_for(n_slices, [&](long long lo, long long hi) {
      for (long long b = lo; b < hi; b++) {
        const SliceShape &s = cv.shapes[b];
        for (int d = 0; d < s.n_diag; d++)
          B.slice_ptr[base + s.diag_off + d] = (unsigned)cv.slice_diags[b][d];
      }
    });
  }
  return ISPM_OK;
}

template <class E>
int guess_impl(int n_rows, const int *row_ptr, const int *cols, int examine_ratio,
               ispm_slell_params &out)
{
  // conversion.h:416-492
  const int kMaxWasteRatio = 100, kEltsPerSlice = 8 * 256, kThreads = 256;
  const int kMinHblockRatio = 25, kMinDiagsRatio = 50, kTrial = 32;
  CsrRows A{n_rows, n_rows, row_ptr, cols};
  int rows = (int)(((long long)n_rows * examine_ratio + 99) / 100);
  rows = (rows + kTrial - 1) & ~(kTrial - 1);
  // The reference reads row_ptr[rows + 1] (one past the examined rows).
  int elts = std::max(1, A.begin(rows + 1));
  int waste = 0, n_hblocks2 = 0, n_diags = 0;
  std::vector<int> dl, t1, t2;
  for (int i = 0; i < rows; i += kTrial) {
    int widest = 0;
    for (int r = i; r < i + kTrial; r++)
      widest = std::max(widest, A.len(r));
    for (int r = i; r < i + kTrial; r++) {
      waste += widest - A.len(r);
      for (int e = A.begin(r); e + 1 < A.end(r); e++)
        if (!(A.ci[e] % 2) && A.ci[e + 1] == A.ci[e] + 1) {
          n_hblocks2++;
          e += 1;
        }
    }
    dl.clear();
    find_diagonals(A, kTrial, i, dl, t1, t2);
    n_diags += (int)dl.size();
  }
  int waste_ratio = 100 * waste / elts;
  bool want_var = waste_ratio > kMaxWasteRatio;
  float avg = 1.f * elts / rows;
  int want_h;
  if (want_var) {
    want_h = kThreads;
  } else {
    want_h = (int)(kEltsPerSlice / avg);
    want_h = want_h > 0 ? (int)floor_pow2((unsigned)want_h) : 0;
    if (want_h < kMinSliceHeight)
      want_h = kMinSliceHeight;
    else if (want_h > kPadRows)
      want_h = kPadRows;
  }
  bool want_diags = n_diags * kTrial > elts * kMinDiagsRatio / 100;
  int want_hb = (!want_diags && n_hblocks2 > elts * kMinHblockRatio / 100) ? 2 : 1;
  out.S = (unsigned)want_h;
  out.H = (unsigned)want_hb;
  out.V = want_var;
  out.D = want_diags;
  return ISPM_OK;
}

int check_csr(int n_rows, int n_cols, const int *row_ptr, const int *cols)
{
  if (n_rows < 0 || n_cols < 0 || !row_ptr)
    return fail(ISPM_ERR_INVALID, "bad CSR shape");
  if (row_ptr[0] != 0)
    return fail(ISPM_ERR_INVALID, "row_ptr[0] != 0");
  for (int r = 0; r < n_rows; r++)
    if (row_ptr[r + 1] < row_ptr[r])
      return fail(ISPM_ERR_INVALID, "row_ptr decreases at row %d", r);
  const int nnz = row_ptr[n_rows];
  if (nnz && !cols)
    return fail(ISPM_ERR_INVALID, "cols is NULL");
  for (int e = 0; e < nnz; e++)
    if (cols[e] < 0 || cols[e] >= n_cols)
      return fail(ISPM_ERR_INVALID, "column %d out of range at entry %d", cols[e], e);
  return ISPM_OK;
}

}  // namespace

int validate_csr(int n_rows, int n_cols, const int *row_ptr, const int *cols)
{
  return check_csr(n_rows, n_cols, row_ptr, cols);
}

ispm_slell_view HostSlell::view() const
{
  ispm_slell_view v;
  v.n_rows = n_rows;
  v.n_cols = n_cols;
  v.n_nz = n_nz;
  v.slice_height = slice_height;
  v.n_slices = n_slices;
  v.hblock = hblock;
  v.var_height = var_height;
  v.diags = diags;
  v.elm_dtype = elm_dtype;
  v.min_slice_height = min_slice_height;
  v.max_slice_height = max_slice_height;
  v.n_slice_ptr = (long long)slice_ptr.size();
  v.n_cols_arr = (long long)cols.size();
  v.n_elms = (long long)n_elms();
  v.slice_ptr = slice_ptr.data();
  v.cols = cols.data();
  v.elms = elms_ptr();
  return v;
}

int convert_csr(int elm_dtype, int n_rows, int n_cols, const int *row_ptr, const int *cols,
                const void *elms, int S, int hblock, bool var_height, bool use_diags,
                int min_height, HostSlell &out)
{
  int st = check_csr(n_rows, n_cols, row_ptr, cols);
  if (st)
    return st;
  if (elm_dtype != ISPM_F32 && elm_dtype != ISPM_F64)
    return fail(ISPM_ERR_INVALID, "elm_dtype %d", elm_dtype);
  if (hblock != 1 && hblock != 2 && hblock != 4)
    return fail(ISPM_ERR_INVALID, "hblock %d (supported: 1, 2, 4)", hblock);
  if (S <= 0 || (S & (S - 1)) || min_height <= 0)
    return fail(ISPM_ERR_INVALID, "slice height %d / min_height %d", S, min_height);
  if (row_ptr[n_rows] && !elms)
    return fail(ISPM_ERR_INVALID, "elms is NULL");
  out = HostSlell();
  out.elm_dtype = elm_dtype;
  if (elm_dtype == ISPM_F32)
    return convert_impl<float>(n_rows, n_cols, row_ptr, cols, (const float *)elms, S, hblock,
                               var_height, use_diags, min_height, out, out.elms_f);
  return convert_impl<double>(n_rows, n_cols, row_ptr, cols, (const double *)elms, S, hblock,
                              var_height, use_diags, min_height, out, out.elms_d);
}

int value_map(const HostSlell &m, int n_rows, const int *row_ptr, const int *cols,
              std::vector<unsigned> &pos)
{
  // Convert again with the CSR entry numbers (1-based) as values and the
  // matrix's own element type steering the hblock split: every entry lands
  // where its value lands in m, so elms[p] = k + 1 gives pos[k] = p.
  if (n_rows < 0 || !row_ptr || (row_ptr[n_rows] && !cols))
    return fail(ISPM_ERR_INVALID, "bad CSR pattern");
  const long long nnz = row_ptr[n_rows];
  if ((long long)m.n_nz != nnz)
    return fail(ISPM_ERR_INVALID, "pattern has %lld entries, the matrix %d", nnz, m.n_nz);
  std::vector<long long> ids(nnz);
  for (long long k = 0; k < nnz; k++)
    ids[k] = k + 1;
  HostSlell shape;
  std::vector<long long> slots;
  int st = m.elm_dtype == ISPM_F32
               ? convert_impl<float, long long>(n_rows, m.n_cols, row_ptr, cols, ids.data(),
                                                (int)m.slice_height, (int)m.hblock, m.var_height,
                                                m.diags, (int)m.min_height_used, shape, slots)
               : convert_impl<double, long long>(n_rows, m.n_cols, row_ptr, cols, ids.data(),
                                                 (int)m.slice_height, (int)m.hblock,
                                                 m.var_height, m.diags, (int)m.min_height_used,
                                                 shape, slots);
  if (st)
    return st;
  if (shape.slice_ptr != m.slice_ptr || shape.cols != m.cols || slots.size() != m.n_elms())
    return fail(ISPM_ERR_INVALID, "the CSR pattern does not produce this matrix's structure");
  pos.assign(nnz, 0u);
  for (size_t p = 0; p < slots.size(); p++)
    if (slots[p] > 0)
      pos[slots[p] - 1] = (unsigned)p;
  return ISPM_OK;
}

int guess_format(int elm_dtype, int n_rows, int n_cols, const int *row_ptr, const int *cols,
                 const void *elms, int examine_ratio, int min_height, ispm_slell_params &out)
{
  (void)elms;
  (void)min_height;
  int st = check_csr(n_rows, n_cols, row_ptr, cols);
  if (st)
    return st;
  if (examine_ratio <= 0)
    return fail(ISPM_ERR_INVALID, "examine_ratio %d", examine_ratio);
  return elm_dtype == ISPM_F32 ? guess_impl<float>(n_rows, row_ptr, cols, examine_ratio, out)
                               : guess_impl<double>(n_rows, row_ptr, cols, examine_ratio, out);
}

}  // namespace ispm

using namespace ispm;

extern "C" {

int ispm_csr_to_slell(int elm_dtype, int n_rows, int n_cols, const int *row_ptr,
                      const int *cols, const void *elms, int slice_height, int hblock,
                      int var_height, int use_diags, int min_height, ispm_slell **out)
{
  clear_error();
  if (!out)
    return fail(ISPM_ERR_INVALID, "out is NULL");
  *out = nullptr;
  ispm_slell *h = new (std::nothrow) ispm_slell;
  if (!h)
    return fail(ISPM_ERR_NOMEM, "host allocation");
  int st;
  try {
    st = convert_csr(elm_dtype, n_rows, n_cols, row_ptr, cols, elms, slice_height, hblock,
                     var_height != 0, use_diags != 0, min_height, h->m);
  } catch (const std::bad_alloc &) {
    st = fail(ISPM_ERR_NOMEM, "host allocation during conversion");
  }
  if (st) {
    delete h;
    return st;
  }
  *out = h;
  return ISPM_OK;
}

int ispm_csr_to_slell_guess_format(int elm_dtype, int n_rows, int n_cols, const int *row_ptr,
                                   const int *cols, const void *elms, int examine_ratio,
                                   int min_height, ispm_slell **out)
{
  clear_error();
  if (!out)
    return fail(ISPM_ERR_INVALID, "out is NULL");
  *out = nullptr;
  ispm_slell_params p;
  int st = guess_format(elm_dtype, n_rows, n_cols, row_ptr, cols, elms, examine_ratio,
                        min_height, p);
  if (st)
    return st;
  return ispm_csr_to_slell(elm_dtype, n_rows, n_cols, row_ptr, cols, elms, (int)p.S, (int)p.H,
                           (int)p.V, (int)p.D, min_height, out);
}

int ispm_slell_get_view(const ispm_slell *m, ispm_slell_view *view)
{
  if (!m || !view)
    return fail(ISPM_ERR_INVALID, "NULL argument");
  *view = m->m.view();
  return ISPM_OK;
}

void *ispm_slell_elms(ispm_slell *m) { return m ? m->m.elms_ptr() : nullptr; }

unsigned long long ispm_slell_spmv_bytes(const ispm_slell *m, int effective, int vec_elt_size)
{
  if (!m)
    return 0;
  const HostSlell &h = m->m;
  unsigned long long esz = h.elm_dtype == ISPM_F32 ? 4 : 8;
  unsigned long long nz = (unsigned long long)h.n_nz;
  return 4ull * h.slice_ptr.size() + 4ull * (effective ? nz : h.cols.size()) +
         esz * (effective ? nz : h.n_elms()) + (unsigned long long)vec_elt_size * 2ull * h.n_rows;
}

void ispm_slell_free(ispm_slell *m) { delete m; }

}  // extern "C"

extern "C" int ispm_slell_value_map(const ispm_slell *m, int n_rows, const int *row_ptr,
                                    const int *cols, unsigned *map)
{
  clear_error();
  if (!m || !map)
    return fail(ISPM_ERR_INVALID, "NULL argument");
  std::vector<unsigned> pos;
  try {
    if (int st = value_map(m->m, n_rows, row_ptr, cols, pos))
      return st;
  } catch (const std::bad_alloc &) {
    return fail(ISPM_ERR_NOMEM, "host allocation while mapping values");
  }
  if (!pos.empty())
    memcpy(map, pos.data(), pos.size() * sizeof(unsigned));
  return ISPM_OK;
}
