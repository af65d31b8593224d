// Host construction of the combinatorial aggregation hierarchy: the
// reference's CMG hierarchy loop (vendored cmg crate hierarchy.rs:437-633)
// with its forest aggregation (forest.rs:94-607) and Galerkin contraction
// (coarsen.rs:349-460), restated.  Pure host code: the tests call it without
// a GPU, and the device engine uploads its levels.
#include "cmg_host.h"

#include <algorithm>
#include <cmath>
#include <numeric>

#include "common.h"

namespace fevcb {

namespace {

// Split the heavy-edge forest into trees of bounded diameter and conductance
// (reference `split_forest_with`, forest.rs:432-560): walks from every leaf
// cut paths longer than five edges in the middle, then a second pass cuts an
// edge whose both sides hold more than two ancestors.
std::vector<uint32_t> split_forest(const std::vector<uint32_t>& parent) {
  const size_t n = parent.size();
  std::vector<uint32_t> forest(parent);
  std::vector<int64_t> ancestors(n, 0);
  std::vector<uint32_t> indegree(n, 0);
  std::vector<uint8_t> visited(n, 0);
  for (uint32_t t : forest) indegree[t]++;
  std::vector<uint32_t> walk;
  std::vector<int64_t> fresh;
  walk.reserve(64);
  fresh.reserve(64);
  for (size_t start = 0; start < n; ++start) {
    uint32_t current = uint32_t(start);
    bool more = true;
    while (more && indegree[current] == 0 && !visited[current]) {
      more = false;
      int64_t in_path = 0;
      walk.clear();
      walk.push_back(current);
      fresh.clear();
      fresh.push_back(0);
      size_t k = 0;
      while (k <= 5 || visited[current]) {
        current = forest[current];
        if (current == walk[k] || (k > 0 && current == walk[k - 1])) break;
        ++k;
        walk.push_back(current);
        in_path += visited[current] ? 0 : 1;
        fresh.push_back(in_path);
      }
      if (k > 5) {
        size_t middle = k / 2;
        forest[walk[middle]] = walk[middle];
        uint32_t next = walk[middle + 1];
        indegree[next]--;
        int64_t removed = ancestors[walk[middle]];
        for (size_t i = middle + 1; i <= k; ++i) ancestors[walk[i]] -= removed;
        for (size_t i = 0; i <= middle; ++i) {
          visited[walk[i]] = 1;
          ancestors[walk[i]] += fresh[i];
        }
        current = next;
        more = true;
      }
      if (!more) {
        for (size_t i = 0; i <= k; ++i) {
          ancestors[walk[i]] += fresh[i];
          visited[walk[i]] = 1;
        }
      }
    }
  }
  for (size_t start = 0; start < n; ++start) {
    uint32_t current = uint32_t(start);
    for (;;) {
      if (indegree[current] != 0) break;
      uint32_t previous = current;
      bool restart = false;
      for (;;) {
        uint32_t next = forest[current];
        if (next == current || next == previous) break;
        if (ancestors[current] > 2 && ancestors[next] - ancestors[current] > 2) {
          forest[current] = current;
          indegree[next]--;
          int64_t removed = ancestors[current];
          uint32_t ap = current, ac = next;
          for (;;) {
            ancestors[ac] -= removed;
            uint32_t an = forest[ac];
            if (an == ac || an == ap) break;
            ap = ac;
            ac = an;
          }
          current = next;
          restart = true;
          break;
        }
        previous = current;
        current = next;
      }
      if (!restart) break;
    }
  }
  return forest;
}

uint32_t find_root(std::vector<uint32_t>& set, uint32_t v) {
  uint32_t r = v;
  while (set[r] != r) r = set[r];
  while (set[v] != r) {
    uint32_t next = set[v];
    set[v] = r;
    v = next;
  }
  return r;
}

// R L R' for aggregation labels (reference `contract_with`, coarsen.rs:349-400,
// and the canonical merge of graph.rs:279-360): every fine edge u < v in
// canonical order maps to its aggregates' pair, intra-aggregate edges drop,
// duplicates merge in ascending weight order with a compensated sum, and the
// diagonal accumulates the merged weights in canonical edge order.
CmgLevel contract(const CmgLevel& f, const std::vector<uint32_t>& labels, uint32_t nc) {
  struct E {
    uint64_t key;
    double w;
  };
  std::vector<E> e;
  e.reserve(f.col.size() / 2);
  for (uint32_t v = 0; v < f.n; ++v)
    for (uint32_t k = f.ptr[v]; k < f.ptr[v + 1]; ++k) {
      uint32_t u = f.col[k];
      if (u <= v) continue;
      uint32_t a = labels[v], b = labels[u];
      if (a == b) continue;
      if (a > b) std::swap(a, b);
      e.push_back(E{(uint64_t(a) << 32) | b, f.val[k]});
    }
  std::sort(e.begin(), e.end(), [](const E& x, const E& y) {
    if (x.key != y.key) return x.key < y.key;
    return total_cmp(x.w, y.w) < 0;
  });
  std::vector<uint64_t> mkey;
  std::vector<double> mval;
  std::vector<double> diag(nc, 0.0);
  for (size_t i = 0; i < e.size();) {
    uint64_t key = e[i].key;
    StableSum sum;
    while (i < e.size() && e[i].key == key) sum.add(e[i++].w);
    double w = sum.finish();
    mkey.push_back(key);
    mval.push_back(w);
    diag[key >> 32] += w;
    diag[key & 0xffffffffu] += w;
  }
  // symmetric CSR, columns ascending within each row
  CmgLevel c;
  c.n = nc;
  c.ptr.assign(nc + 1, 0);
  for (uint64_t key : mkey) {
    c.ptr[(key >> 32) + 1]++;
    c.ptr[(key & 0xffffffffu) + 1]++;
  }
  for (uint32_t v = 0; v < nc; ++v) c.ptr[v + 1] += c.ptr[v];
  c.col.assign(c.ptr[nc], 0);
  c.val.assign(c.ptr[nc], 0.0);
  std::vector<uint32_t> cur(c.ptr.begin(), c.ptr.end() - 1);
  // lower entries (u, a) with a < u come first in row u when edges are walked
  // in canonical order for the second endpoint...
  for (size_t i = 0; i < mkey.size(); ++i) {
    uint32_t b = uint32_t(mkey[i] & 0xffffffffu), a = uint32_t(mkey[i] >> 32);
    c.col[cur[b]] = a;
    c.val[cur[b]++] = mval[i];
  }
  // ...then the upper entries (a, b) with b > a
  for (size_t i = 0; i < mkey.size(); ++i) {
    uint32_t b = uint32_t(mkey[i] & 0xffffffffu), a = uint32_t(mkey[i] >> 32);
    c.col[cur[a]] = b;
    c.val[cur[a]++] = mval[i];
  }
  c.diag = std::move(diag);
  return c;
}

// Dense pseudo-inverse of a connected Laplacian: (L + a 11')^{-1} - 11'/(a n^2).
std::vector<double> dense_pseudo_inverse(const CmgLevel& l) {
  const uint32_t n = l.n;
  std::vector<double> a(size_t(n) * n, 0.0);
  double mean_degree = 0.0;
  for (uint32_t v = 0; v < n; ++v) mean_degree += l.diag[v];
  mean_degree = n ? mean_degree / n : 1.0;
  if (!(mean_degree > 0.0)) mean_degree = 1.0;
  const double shift = mean_degree / n;
  for (uint32_t v = 0; v < n; ++v) {
    a[size_t(v) * n + v] += l.diag[v];
    for (uint32_t k = l.ptr[v]; k < l.ptr[v + 1]; ++k) a[size_t(v) * n + l.col[k]] -= l.val[k];
  }
  for (auto& x : a) x += shift;
  // Cholesky (lower, in place)
  for (uint32_t j = 0; j < n; ++j) {
    double d = a[size_t(j) * n + j];
    for (uint32_t k = 0; k < j; ++k) d -= a[size_t(j) * n + k] * a[size_t(j) * n + k];
    if (!(d > 0.0) || !std::isfinite(d))
      fail(CMG_SETUP_FAILED, "cmg_direct", "coarsest Laplacian is not connected or not positive");
    d = std::sqrt(d);
    a[size_t(j) * n + j] = d;
    for (uint32_t i = j + 1; i < n; ++i) {
      double s = a[size_t(i) * n + j];
      for (uint32_t k = 0; k < j; ++k) s -= a[size_t(i) * n + k] * a[size_t(j) * n + k];
      a[size_t(i) * n + j] = s / d;
    }
  }
  // inverse column by column
  std::vector<double> inv(size_t(n) * n, 0.0), y(n);
  for (uint32_t c = 0; c < n; ++c) {
    std::fill(y.begin(), y.end(), 0.0);
    y[c] = 1.0;
    for (uint32_t i = 0; i < n; ++i) {
      double s = y[i];
      for (uint32_t k = 0; k < i; ++k) s -= a[size_t(i) * n + k] * y[k];
      y[i] = s / a[size_t(i) * n + i];
    }
    for (uint32_t i = n; i-- > 0;) {
      double s = y[i];
      for (uint32_t k = i + 1; k < n; ++k) s -= a[size_t(k) * n + i] * y[k];
      y[i] = s / a[size_t(i) * n + i];
    }
    for (uint32_t i = 0; i < n; ++i) inv[size_t(i) * n + c] = y[i];
  }
  const double corr = 1.0 / (shift * double(n) * double(n));
  for (auto& x : inv) x -= corr;
  for (uint32_t i = 0; i < n; ++i)
    for (uint32_t j = 0; j < i; ++j) {
      double s = 0.5 * (inv[size_t(i) * n + j] + inv[size_t(j) * n + i]);
      inv[size_t(i) * n + j] = inv[size_t(j) * n + i] = s;
    }
  return inv;
}

}  // namespace

uint32_t forest_aggregation(uint32_t n, const std::vector<uint32_t>& ptr, const std::vector<uint32_t>& col,
                            const std::vector<double>& val, const std::vector<double>& diag, double threshold,
                            std::vector<uint32_t>& labels) {
  // heavy forest: each vertex's maximum-weight edge, ties to the lowest
  // neighbour (reference `heavy_forest_serial` / `consider_parent`,
  // forest.rs:131-156, 320-334)
  std::vector<uint32_t> parent(n);
  std::vector<double> weight(n, 0.0);
  for (uint32_t v = 0; v < n; ++v) {
    parent[v] = v;
    for (uint32_t k = ptr[v]; k < ptr[v + 1]; ++k) {
      uint32_t u = col[k];
      double w = val[k];
      if (w > weight[v] || (w == weight[v] && u < parent[v])) {
        weight[v] = w;
        parent[v] = u;
      }
    }
  }
  std::vector<uint32_t> split = split_forest(parent);
  // low effective degree: a vertex whose tree edges carry less than
  // `threshold` of its degree becomes a singleton (forest.rs:336-378)
  bool low = false;
  for (uint32_t v = 0; v < n && !low; ++v) low = diag[v] > 0.0 && weight[v] / diag[v] < threshold;
  if (low) {
    std::vector<double> incident(n, 0.0);
    for (uint32_t v = 0; v < n; ++v)
      if (split[v] != v) {
        incident[v] += weight[v];
        incident[split[v]] += weight[v];
      }
    for (uint32_t v = 0; v < n; ++v)
      if (diag[v] > 0.0 && incident[v] / diag[v] < threshold) split[v] = v;
  }
  // union-find components, labels in first-occurrence root order
  // (forest.rs:562-607)
  std::vector<uint32_t> set(n);
  std::iota(set.begin(), set.end(), 0u);
  for (uint32_t v = 0; v < n; ++v) {
    uint32_t a = find_root(set, v), b = find_root(set, split[v]);
    if (a != b) {
      if (a < b)
        set[b] = a;
      else
        set[a] = b;
    }
  }
  labels.assign(n, 0);
  std::vector<uint32_t> root_label(n, UINT32_MAX);
  uint32_t count = 0;
  for (uint32_t v = 0; v < n; ++v) {
    uint32_t r = find_root(set, v);
    if (root_label[r] == UINT32_MAX) root_label[r] = count++;
    labels[v] = root_label[r];
  }
  return count;
}


std::vector<CmgLevel> build_cmg_hierarchy(uint32_t n, const std::vector<uint32_t>& ptr,
                                          const std::vector<uint32_t>& col, const std::vector<double>& val,
                                          const std::vector<double>& diag, const MultigridOptions& opt,
                                          MultigridReport& rep) {
  std::vector<CmgLevel> out;
  CmgLevel cur;
  cur.n = n;
  cur.ptr = ptr;
  cur.col = col;
  cur.val = val;
  cur.diag = diag;
  const uint64_t initial_nnz = cur.matrix_nnz();
  uint64_t cumulative = 0;
  rep = MultigridReport();
  for (;;) {
    rep.vertices.push_back(cur.n);
    rep.nonzeros.push_back(cur.col.size());
    if (cur.n <= 1 || cur.n < opt.direct_threshold) {
      cur.terminal = CMG_DIRECT;
      cur.pinv = dense_pseudo_inverse(cur);
      rep.terminal_reason = CMG_DIRECT;
      out.push_back(std::move(cur));
      break;
    }
    std::vector<uint32_t> labels;
    uint32_t nc = forest_aggregation(cur.n, cur.ptr, cur.col, cur.val, cur.diag, opt.low_effective_degree_threshold,
                                     labels);
    int terminal = CMG_NONE;
    if (nc == 1) {
      terminal = CMG_FULL_CONTRACTION;
    } else {
      cumulative += cur.matrix_nnz();
      if (nc >= cur.n - 1)
        terminal = CMG_STAGNATED_VERTICES;
      else if (double(cumulative) > opt.max_hierarchy_nnz_factor * double(initial_nnz))
        terminal = CMG_STAGNATED_FILL;
      else if (int(out.size()) + 1 >= opt.max_levels)
        terminal = CMG_MAX_LEVELS;
    }
    if (terminal != CMG_NONE) {
      cur.terminal = terminal;
      rep.terminal_reason = terminal;
      out.push_back(std::move(cur));
      break;
    }
    CmgLevel coarse = contract(cur, labels, nc);
    uint64_t fine_nnz = cur.matrix_nnz(), coarse_nnz = coarse.matrix_nnz();
    // repeat = max(nnz_f / nnz_c - 1, 1) (hierarchy.rs:685-690)
    cur.repeat = coarse_nnz == 0 ? 1 : int(std::max<uint64_t>(fine_nnz / coarse_nnz, 2) - 1);
    cur.nc = nc;
    cur.labels = std::move(labels);
    rep.repeat.push_back(cur.repeat);
    out.push_back(std::move(cur));
    cur = std::move(coarse);
  }
  return out;
}

}  // namespace fevcb
