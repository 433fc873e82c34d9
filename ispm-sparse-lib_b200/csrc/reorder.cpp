// Reverse Cuthill-McKee ordering of a symmetric sparsity pattern, used by the
// solver to restore locality in matrices whose numbering is scattered (a
// randomly permuted mesh): with the rows renumbered, the x gathers of every
// SpMV land in a narrow band again instead of anywhere in the vector.
#include <algorithm>
#include <new>
#include <vector>

#include "ispm_internal.h"

namespace ispm {

namespace {

// Breadth-first levels from `start` over unvisited nodes (mark holds the
// visit stamp); returns the nodes in visit order.
void bfs(int start, const int *rp, const int *ci, const std::vector<int> &deg,
         std::vector<int> &mark, int stamp, std::vector<int> &order, std::vector<int> &level_of,
         bool sort_by_degree)
{
  order.clear();
  order.push_back(start);
  mark[start] = stamp;
  level_of[start] = 0;
  std::vector<int> nb;
  for (size_t h = 0; h < order.size(); h++) {
    const int u = order[h];
    nb.clear();
    for (int e = rp[u]; e < rp[u + 1]; e++) {
      const int v = ci[e];
      if (mark[v] != stamp) {
        mark[v] = stamp;
        level_of[v] = level_of[u] + 1;
        nb.push_back(v);
      }
    }
    if (sort_by_degree)
      std::sort(nb.begin(), nb.end(),
                [&](int a, int b) { return deg[a] != deg[b] ? deg[a] < deg[b] : a < b; });
    order.insert(order.end(), nb.begin(), nb.end());
  }
}

}  // namespace

long long bandwidth(int n, const int *rp, const int *ci, const int *inv)
{
  long long bw = 0;
  for (int i = 0; i < n; i++)
    for (int e = rp[i]; e < rp[i + 1]; e++) {
      const long long d = inv ? (long long)inv[ci[e]] - inv[i] : (long long)ci[e] - i;
      bw = std::max(bw, d < 0 ? -d : d);
    }
  return bw;
}

void rcm_order(int n, const int *rp, const int *ci, std::vector<int> &perm)
{
  std::vector<int> deg(n), by_deg(n), mark(n, -1), level_of(n, 0), order;
  for (int i = 0; i < n; i++)
    deg[i] = rp[i + 1] - rp[i];
  for (int i = 0; i < n; i++)
    by_deg[i] = i;
  std::stable_sort(by_deg.begin(), by_deg.end(), [&](int a, int b) { return deg[a] < deg[b]; });
  std::vector<char> done(n, 0);
  perm.clear();
  perm.reserve(n);
  int stamp = 0;
  size_t next = 0;
  while (perm.size() < (size_t)n) {
    while (done[by_deg[next]])
      next++;
    // pseudo-peripheral start: from the lowest-degree unvisited node, walk to
    // a lowest-degree node of the last BFS level, twice
    int start = by_deg[next];
    for (int pass = 0; pass < 2; pass++) {
      ++stamp;  // a BFS never leaves its component, so earlier ones stay apart
      bfs(start, rp, ci, deg, mark, stamp, order, level_of, false);
      const int last = level_of[order.back()];
      int best = order.back();
      for (int v : order)
        if (level_of[v] == last && deg[v] < deg[best])
          best = v;
      if (best == start)
        break;
      start = best;
    }
    ++stamp;
    bfs(start, rp, ci, deg, mark, stamp, order, level_of, true);
    for (int v : order) {
      done[v] = 1;
      perm.push_back(v);
    }
  }
  std::reverse(perm.begin(), perm.end());
}

void permute_csr(int n, const int *rp, const int *ci, const double *v,
                 const std::vector<int> &perm, const std::vector<int> &inv, std::vector<int> &orp,
                 std::vector<int> &oci, std::vector<double> &ov)
{
  orp.assign((size_t)n + 1, 0);
  for (int i = 0; i < n; i++)
    orp[i + 1] = orp[i] + (rp[perm[i] + 1] - rp[perm[i]]);
  oci.resize((size_t)rp[n]);
  ov.resize((size_t)rp[n]);
  std::vector<std::pair<int, double>> row;
  for (int i = 0; i < n; i++) {
    const int src = perm[i];
    row.clear();
    for (int e = rp[src]; e < rp[src + 1]; e++)
      row.emplace_back(inv[ci[e]], v[e]);
    std::sort(row.begin(), row.end(),
              [](const std::pair<int, double> &a, const std::pair<int, double> &b) {
                return a.first < b.first;
              });
    for (size_t k = 0; k < row.size(); k++) {
      oci[orp[i] + k] = row[k].first;
      ov[orp[i] + k] = row[k].second;
    }
  }
}

}  // namespace ispm

extern "C" int ispm_rcm_order(int n, const int *row_ptr, const int *cols, int *perm)
{
  ispm::clear_error();
  if (n < 0 || !row_ptr || !perm)
    return ispm::fail(ISPM_ERR_INVALID, "bad arguments");
  if (int e = ispm::validate_csr(n, n, row_ptr, cols))
    return e;
  try {
    std::vector<int> p;
    ispm::rcm_order(n, row_ptr, cols, p);
    std::copy(p.begin(), p.end(), perm);
  } catch (const std::bad_alloc &) {
    return ispm::fail(ISPM_ERR_NOMEM, "host allocation");
  }
  return ISPM_OK;
}

extern "C" long long ispm_csr_bandwidth(int n, const int *row_ptr, const int *cols)
{
  ispm::clear_error();
  if (n < 0 || !row_ptr || ispm::validate_csr(n, n, row_ptr, cols))
    return -1;
  return ispm::bandwidth(n, row_ptr, cols, nullptr);
}
