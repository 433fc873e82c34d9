// Right-looking AINV / FSAI-like approximate inverse (host).
//
// Computes the pair the reference's fastainv_sym returns
// (fastainv/fastainv.cpp:395-566): Ainv1 = G and Ainv2 = G^T (scaled by the
// unsigned root of the pivots), with Ainv2 * Ainv1 ~ A^-1, bit for bit.
//
// The arithmetic (operation order, operand types, drop test, pivot handling)
// follows the reference step by step because every one of those choices
// changes rounding: the column merge of A * w_j accumulates duplicate columns
// in the pop order of the reference's binary heap (fastainv.cpp:99-213), so
// that heap's sift rules are restated here exactly.  Storage differs: each
// factor row lives in one contiguous segment of an arena (the reference chains
// 8-entry chunks), which turns the hot row merges into linear scans.  The
// reference's chunk bookkeeping is still tracked as a counter, because it
// decides where rows are truncated once max_elts is exhausted
// (fastainv.cpp:74-78).
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <new>

#include "ispm_internal.h"

namespace ispm {
namespace {

constexpr int kChunk = 8;  // fastainv.cpp:15 CHUNK_SZ

long long maxneed(long long n)
{
  // fastainv.cpp:387-392
  n = (n + kChunk - 1) / kChunk;
  return n * (n + 1) / 2 * kChunk * kChunk;
}

// Factor rows W_j: sorted (row, value) lists, one contiguous segment each.
template <class real> struct RowStore {
  std::vector<long long> off;
  std::vector<int> len, cap;
  std::vector<int> rows;
  std::vector<real> vals;
  // Reference chunk accounting (fastainv.cpp:57-97).
  long long alloced = 0, used = 0;
  long long truncated = 0;

  void init(int n, long long chunks)
  {
    off.assign(n, 0);
    len.assign(n, 0);
    cap.assign(n, 0);
    alloced = chunks;
    rows.reserve(1 << 20);
    vals.reserve(1 << 20);
  }
  const int *row_of(int r) const { return rows.data() + off[r]; }
  const real *val_of(int r) const { return vals.data() + off[r]; }

  // chunky_storage::replace (fastainv.cpp:74-97): keep at most what the
  // chunk budget allows, leave the row untouched when nothing is kept.
  void replace(int r, int n, const int *nrow, const real *nval)
  {
    long long avail = (alloced - used + (len[r] + kChunk - 1) / kChunk) * kChunk;
    long long keep = std::min<long long>(n, avail);
    if (keep < n)
      truncated++;
    if (keep <= 0)
      return;
    if (!len[r])
      used++;
    for (long long i = kChunk; i < keep; i += kChunk)
      if (i >= len[r])
        used++;
    if (keep > cap[r]) {
      int c = std::max<int>((int)keep, 2 * cap[r]);
      c = std::max(c, kChunk);
      off[r] = (long long)rows.size();
      rows.resize(rows.size() + c);
      vals.resize(vals.size() + c);
      cap[r] = c;
    }
    memcpy(rows.data() + off[r], nrow, sizeof(int) * keep);
    memcpy(vals.data() + off[r], nval, sizeof(real) * keep);
    len[r] = (int)keep;
  }
};

// Binary min-heap over (column, source) pairs with the reference's sift
// rules (fastainv.cpp:99-213): strict comparisons, a right-child preference
// on ties, an INT_MAX sentinel one past the end.
template <class real> struct MergeHeap {
  struct Node {
    int column, idx;
  };
  std::vector<Node> node;
  std::vector<real> factor;
  std::vector<int> pos, lim;
  int sz = 0;

  void reset(int cap)
  {
    if ((int)node.size() < cap + 1) {
      node.resize(cap + 1);
      factor.resize(cap);
      pos.resize(cap);
      lim.resize(cap);
    }
    sz = 0;
  }
  void add(int o, int l, int c, real f)
  {
    node[sz].column = c;
    node[sz].idx = sz;
    factor[sz] = f;
    pos[sz] = o;
    lim[sz] = l;
    sz++;
  }
  // Move (column, idx) down from slot i to where it belongs.
  void sink(int i, int column, int idx)
  {
    for (;;) {
      int l = 2 * i + 1, r = l + 1;
      if (l >= sz)
        break;
      int mcol = std::min(node[l].column, node[r].column);
      if (!(mcol < column))
        break;
      int mc = node[l].column < node[r].column ? l : r;
      node[i].column = mcol;
      node[i].idx = node[mc].idx;
      i = mc;
    }
    node[i].column = column;
    node[i].idx = idx;
  }
  void sift(int i)
  {
    int l = 2 * i + 1;
    if (l >= sz)
      return;
    sink(i, node[i].column, node[i].idx);
  }
  void build()
  {
    node[sz].column = INT_MAX;
    for (int i = sz / 2 - 1; i >= 0; i--)
      sift(i);
  }
  void pop()
  {
    sz--;
    node[0] = node[sz];
    node[sz].column = INT_MAX;
    sift(0);
  }
  void replace_top(int c)
  {
    node[0].column = c;
    sift(0);
  }
};

template <class in_real, class real> struct Ainv {
  int n;
  const int *rp, *ci;
  const in_real *av;
  double droptol;
  // Extended build (ispm_fastainv_sym_ex): per-row drop tolerance and a
  // positive per-row factor on the pivot scale.  NULL in the reference build.
  const double *row_tol = nullptr;
  const double *row_scale = nullptr;
  RowStore<real> W;
  MergeHeap<real> heap;
  std::vector<int> u_idx, m_row;
  std::vector<in_real> u_val;
  std::vector<real> m_val;
  std::vector<real> D;
  long long breakdowns = 0;

  // u = A w_j with w_j's implicit unit entry at j (fastainv.cpp:215-264).
  int a_times_w(int j)
  {
    const int wl = W.len[j];
    const int *wr = W.row_of(j);
    const real *wv = W.val_of(j);
    heap.reset(wl + 1);
    for (int k = 0; k < wl; k++) {
      int r = wr[k];
      if (rp[r] < rp[r + 1])
        heap.add(rp[r], rp[r + 1], ci[rp[r]], wv[k]);
    }
    if (rp[j] < rp[j + 1])
      heap.add(rp[j], rp[j + 1], ci[rp[j]], (real)1);
    heap.build();
    int out = -1, prevcol = -1;
    in_real prev = 0;
    while (heap.sz > 0) {
      const int col = heap.node[0].column, src = heap.node[0].idx;
      in_real add = av[heap.pos[src]] * heap.factor[src];
      // Same expression as the reference, which also decides the sign of
      // zero when a run starts: prev - prev * next.
      int next = prevcol < col ? 1 : 0;
      prev = prev - prev * next;
      prevcol = col;
      out += next;
      u_idx[out] = col;
      u_val[out] = prev += add;
      if (++heap.pos[src] < heap.lim[src])
        heap.replace_top(ci[heap.pos[src]]);
      else
        heap.pop();
    }
    return out + 1;
  }

  // W_i <- W_i + f * (w_j with its unit entry), dropping |value| <= droptol
  // (fastainv.cpp:266-386).
  void update(int j, int i, real f)
  {
    const int jl = W.len[j], il = W.len[i];
    const int *jr = W.row_of(j), *ir = W.row_of(i);
    const real *jv = W.val_of(j), *iv = W.val_of(i);
    int a = 0, b = 0, m = 0;  // a walks W_i, b walks W_j (b == jl: the unit entry)
    int *mr = m_row.data();
    real *mv = m_val.data();
    // per-row tolerance of the row being rebuilt (the extended build only)
    const double tol = row_tol ? row_tol[i] : droptol;
    auto put = [&](int row, real v) {
      if (std::abs(v) > tol) {
        mr[m] = row;
        mv[m] = v;
        m++;
      }
    };
    while (a < il && b < jl) {
      if (jr[b] < ir[a]) {
        put(jr[b], jv[b] * f);
        b++;
      } else if (jr[b] > ir[a]) {
        put(ir[a], iv[a]);
        a++;
      } else {
        put(ir[a], iv[a] + jv[b] * f);
        a++;
        b++;
      }
    }
    while (a < il && b == jl) {
      if (j < ir[a]) {
        put(j, f);
        b++;
      } else if (j > ir[a]) {
        put(ir[a], iv[a]);
        a++;
      } else {
        put(ir[a], iv[a] + f);
        a++;
        b++;
      }
    }
    for (; a < il; a++)
      put(ir[a], iv[a]);
    for (; b < jl; b++)
      put(jr[b], jv[b] * f);
    if (b == jl)
      put(j, f);
    W.replace(i, m, mr, mv);
  }

  void run(ispm_progress_f progress, void *pv)
  {
    D.assign(n, (real)0);
    u_idx.resize(n + 1);
    u_val.resize(n + 1);
    m_row.resize(n + 1);
    m_val.resize(n + 1);
    for (int j = 0; j < n; j++) {
      if (progress)
        progress(pv);
      const int wl = W.len[j];
      const int *uidx;
      const in_real *uval;
      int un, ui = 0;
      real Djj = 0;
      if (!wl) {
        uidx = ci + rp[j];
        uval = av + rp[j];
        un = rp[j + 1] - rp[j];
      } else {
        un = a_times_w(j);
        uidx = u_idx.data();
        uval = u_val.data();
        // D_jj = u . w_j (fastainv.cpp:441-466)
        const int *wr = W.row_of(j);
        const real *wv = W.val_of(j);
        int k = 0;
        while (ui < un && k < wl) {
          if (uidx[ui] < wr[k]) {
            ui++;
          } else if (uidx[ui] > wr[k]) {
            k++;
          } else {
            Djj += uval[ui++] * wv[k];
            k++;
          }
        }
      }
      while (ui < un) {
        if (uidx[ui] < j)
          ui++;
        else if (uidx[ui] > j)
          break;
        else
          Djj += uval[ui++];
      }
      if (Djj == 0) {  // breakdown: fastainv.cpp:468-472
        D[j] = 0;
        breakdowns++;
        continue;
      }
      Djj = 1. / Djj;
      for (; ui < un; ui++) {
        real f = -uval[ui] * Djj;
        update(j, uidx[ui], f);
      }
      D[j] = Djj;
    }
  }

  // fastainv.cpp:489-558: transpose into Ainv2, copy into Ainv1.
  void emit(HostCsr &A1, HostCsr &A2, std::vector<real> &e1, std::vector<real> &e2)
  {
    A2.n_rows = A2.n_cols = n;
    A2.row_ptr.assign(n + 1, 0);
    for (int t = 0; t < n; t++) {
      const int src = n - 1 - t;
      const int *wr = W.row_of(src);
      for (int k = 0; k < W.len[src]; k++)
        A2.row_ptr[wr[k] + 1]++;
    }
    int sum = 0;
    for (int r = 1; r <= n; r++) {
      sum += A2.row_ptr[r] + 1;
      A2.row_ptr[r] = sum;
    }
    A2.n_nz = sum;
    A2.cols.assign(sum, 0);
    e2.assign(sum, (real)0);
    std::vector<int> fill(n, 0);
    for (int t = 0; t < n; t++) {
      const int src = n - 1 - t;
      real scal = std::sqrt(std::abs(D[src]));
      if (row_scale)
        scal = (real)(scal * row_scale[src]);
      D[src] = std::copysign(scal, D[src]);
      const int *wr = W.row_of(src);
      const real *wv = W.val_of(src);
      for (int k = 0; k < W.len[src]; k++) {
        int at = A2.row_ptr[wr[k]] + fill[wr[k]]++;
        A2.cols[at] = t;
        e2[at] = wv[k] * scal;
      }
      int at = A2.row_ptr[src] + fill[src]++;
      A2.cols[at] = t;
      e2[at] = scal;
    }
    A1.n_rows = A1.n_cols = n;
    A1.row_ptr.assign(1, 0);
    A1.row_ptr.reserve(n + 1);
    A1.cols.clear();
    A1.cols.reserve(sum);
    e1.clear();
    e1.reserve(sum);
    for (int t = 0; t < n; t++) {
      const int src = n - 1 - t;
      const int *wr = W.row_of(src);
      const real *wv = W.val_of(src);
      for (int k = 0; k < W.len[src]; k++) {
        A1.cols.push_back(wr[k]);
        e1.push_back(wv[k] * D[src]);
      }
      A1.cols.push_back(src);
      e1.push_back(D[src]);
      A1.row_ptr.push_back((int)A1.cols.size());
    }
    A1.n_nz = (int)A1.cols.size();
  }
};

template <class real>
int fastainv_impl(int n, const int *rp, const int *ci, const double *av, ispm_progress_f progress,
                  void *pv, long long max_elts, double droptol, HostCsr &A1, HostCsr &A2,
                  std::vector<real> &e1, std::vector<real> &e2, ispm_fastainv_stats *stats,
                  const double *row_tol = nullptr, const double *row_scale = nullptr)
{
  Ainv<double, real> f;
  f.n = n;
  f.rp = rp;
  f.ci = ci;
  f.av = av;
  f.droptol = droptol;
  f.row_tol = row_tol;
  f.row_scale = row_scale;
  max_elts = std::min(max_elts, maxneed(n));
  f.W.init(n, max_elts / kChunk);
  f.run(progress, pv);
  f.emit(A1, A2, e1, e2);
  if (stats) {
    stats->storage_chunks = f.W.alloced;
    stats->chunks_used = f.W.used;
    stats->truncated_rows = f.W.truncated;
    stats->breakdowns = f.breakdowns;
  }
  return ISPM_OK;
}

}  // namespace
}  // namespace ispm

using namespace ispm;

extern "C" {

}  // extern "C"

static int fastainv_entry(int out_dtype, int n, const int *row_ptr, const int *cols,
                          const double *elms, ispm_progress_f progress, void *v,
                          long long max_elts, double droptol, ispm_csr **ainv1,
                          ispm_csr **ainv2, ispm_fastainv_stats *stats, const double *row_tol,
                          const double *row_scale)
{
  clear_error();
  if (!ainv1 || !ainv2)
    return fail(ISPM_ERR_INVALID, "output pointers are NULL");
  *ainv1 = *ainv2 = nullptr;
  if (n <= 0)
    return fail(ISPM_ERR_INVALID, "n = %d (fastainv_sym returns false for n <= 0)", n);
  if (out_dtype != ISPM_F32 && out_dtype != ISPM_F64)
    return fail(ISPM_ERR_INVALID, "out_dtype %d", out_dtype);
  if (!row_ptr || (row_ptr[n] && (!cols || !elms)))
    return fail(ISPM_ERR_INVALID, "NULL CSR array");
  for (int r = 0; r < n; r++) {
    if (row_ptr[r + 1] < row_ptr[r])
      return fail(ISPM_ERR_INVALID, "row_ptr decreases at row %d", r);
    for (int e = row_ptr[r]; e < row_ptr[r + 1]; e++) {
      if (cols[e] < 0 || cols[e] >= n)
        return fail(ISPM_ERR_INVALID, "column %d out of range in row %d", cols[e], r);
      if (e > row_ptr[r] && cols[e] <= cols[e - 1])
        return fail(ISPM_ERR_INVALID, "row %d columns not strictly increasing", r);
    }
  }
  if (max_elts < 0)
    return fail(ISPM_ERR_INVALID, "max_elts %lld", max_elts);
  // The reference's chunk arithmetic is 32-bit (fastainv.cpp:57,108).
  if (std::min(max_elts, maxneed(n)) > (long long)INT_MAX - kChunk)
    return fail(ISPM_ERR_TOO_LARGE, "max_elts %lld above 2^31 - 8", max_elts);
  ispm_csr *g1 = new (std::nothrow) ispm_csr, *g2 = new (std::nothrow) ispm_csr;
  if (!g1 || !g2) {
    delete g1;
    delete g2;
    return fail(ISPM_ERR_NOMEM, "host allocation");
  }
  int st;
  try {
    g1->m.dtype = g2->m.dtype = out_dtype;
    if (out_dtype == ISPM_F64)
      st = fastainv_impl<double>(n, row_ptr, cols, elms, progress, v, max_elts, droptol, g1->m,
                                 g2->m, g1->m.elms_d, g2->m.elms_d, stats, row_tol, row_scale);
    else
      st = fastainv_impl<float>(n, row_ptr, cols, elms, progress, v, max_elts, droptol, g1->m,
                                g2->m, g1->m.elms_f, g2->m.elms_f, stats, row_tol, row_scale);
  } catch (const std::bad_alloc &) {
    st = fail(ISPM_ERR_NOMEM, "host allocation during fastainv");
  }
  if (st) {
    delete g1;
    delete g2;
    return st;
  }
  *ainv1 = g1;
  *ainv2 = g2;
  return ISPM_OK;
}

extern "C" {

int ispm_fastainv_sym(int out_dtype, int n, const int *row_ptr, const int *cols,
                      const double *elms, ispm_progress_f progress, void *v,
                      long long max_elts, double droptol, ispm_csr **ainv1, ispm_csr **ainv2,
                      ispm_fastainv_stats *stats)
{
  return fastainv_entry(out_dtype, n, row_ptr, cols, elms, progress, v, max_elts, droptol,
                        ainv1, ainv2, stats, nullptr, nullptr);
}

int ispm_fastainv_sym_ex(int out_dtype, int n, const int *row_ptr, const int *cols,
                         const double *elms, const double *row_droptol, const double *row_scale,
                         long long max_elts, double droptol, ispm_csr **ainv1, ispm_csr **ainv2,
                         ispm_fastainv_stats *stats)
{
  if (row_droptol)
    for (int i = 0; i < n; i++)
      if (!(row_droptol[i] >= 0))
        return fail(ISPM_ERR_INVALID, "row_droptol[%d] = %g", i, row_droptol[i]);
  if (row_scale)
    for (int i = 0; i < n; i++)
      if (!(row_scale[i] > 0) || !std::isfinite(row_scale[i]))
        return fail(ISPM_ERR_INVALID, "row_scale[%d] = %g", i, row_scale[i]);
  return fastainv_entry(out_dtype, n, row_ptr, cols, elms, nullptr, nullptr, max_elts, droptol,
                        ainv1, ainv2, stats, row_droptol, row_scale);
}

int ispm_csr_get_info(const ispm_csr *m, int *n_rows, int *n_cols, int *n_nz, int *dtype)
{
  if (!m)
    return fail(ISPM_ERR_INVALID, "NULL matrix");
  if (n_rows)
    *n_rows = m->m.n_rows;
  if (n_cols)
    *n_cols = m->m.n_cols;
  if (n_nz)
    *n_nz = m->m.n_nz;
  if (dtype)
    *dtype = m->m.dtype;
  return ISPM_OK;
}

int ispm_csr_get_arrays(const ispm_csr *m, const int **row_ptr, const int **cols,
                        const void **elms)
{
  if (!m)
    return fail(ISPM_ERR_INVALID, "NULL matrix");
  if (row_ptr)
    *row_ptr = m->m.row_ptr.data();
  if (cols)
    *cols = m->m.cols.data();
  if (elms)
    *elms = m->m.elms_ptr();
  return ISPM_OK;
}

void ispm_csr_free(ispm_csr *m) { delete m; }

}  // extern "C"
