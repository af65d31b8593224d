#include "hybrid.h"

#include <algorithm>
#include <cmath>
#include <numeric>

#include "common.h"
#include "radix.h"

namespace fevcb {

// Host assembly of the hybrid Laplacian (conductances) from the cells.
void build_hybrid(const Compressed& p, uint32_t max_degree, std::vector<uint32_t>& kept_worker,
                  std::vector<int32_t>& kept_index, std::vector<double>& cell_scale, std::vector<double>& worker_diag,
                  std::vector<uint32_t>& Lptr, std::vector<uint32_t>& Lcol, std::vector<double>& Lval,
                  std::vector<double>& Ldiag) {
  size_t W = p.workers, F = p.firms, C = p.cells;
  worker_diag.assign(W, 0.0);
  kept_index.assign(W, -1);
  cell_scale.assign(C, 0.0);
  const auto& wp = p.worker_index.ptr;
  for (size_t w = 0; w < W; ++w) {
    double d = 0.0;
    for (uint64_t c = wp[w]; c < wp[w + 1]; ++c) d += p.cell_weight[c];
    if (!(d > 0.0) || !std::isfinite(d))
      fail(GRAPH_UNIDENTIFIED, "operator", "worker or firm information diagonal is not positive and finite");
    worker_diag[w] = d;
    if (wp[w + 1] - wp[w] > max_degree) {
      kept_index[w] = int32_t(kept_worker.size());
      kept_worker.push_back(uint32_t(w));
    }
  }
  size_t n = F + kept_worker.size();
  // triplets (row, col, value) with row != col
  std::vector<uint64_t> key;
  std::vector<double> val;
  for (size_t w = 0; w < W; ++w) {
    uint64_t b = wp[w], e = wp[w + 1];
    if (kept_index[w] >= 0) {
      uint64_t v = F + kept_index[w];
      for (uint64_t c = b; c < e; ++c) {
        uint64_t f = p.cell_firm[c];
        key.push_back((v << 32) | f);
        val.push_back(p.cell_weight[c]);
        key.push_back((f << 32) | v);
        val.push_back(p.cell_weight[c]);
      }
    } else {
      double d = worker_diag[w];
      for (uint64_t c = b; c < e; ++c) cell_scale[c] = p.cell_weight[c] / d;
      for (uint64_t i = b; i < e; ++i)
        for (uint64_t j = b; j < e; ++j) {
          if (i == j) continue;
          key.push_back((uint64_t(p.cell_firm[i]) << 32) | p.cell_firm[j]);
          val.push_back(p.cell_weight[i] * p.cell_weight[j] / d);
        }
    }
  }
  if (key.size() > 0xffffffffull) fail(RESOURCE_LIMIT, "operator", "hybrid Laplacian has too many entries");
  std::vector<uint32_t> order(key.size());
  std::iota(order.begin(), order.end(), 0u);
  // entries ordered by (row, column); duplicate conductances of one edge keep
  // their generation (worker) order and add in it, as the reference's edge
  // map does (vckss-core/src/cmg_impl.rs.in:634-660): the radix sort is stable
  radix_sort_pairs(key, order);
  Lptr.assign(n + 1, 0);
  Lcol.clear();
  Lval.clear();
  for (size_t i = 0; i < order.size();) {
    uint64_t k = key[i];
    double s = 0.0;
    while (i < order.size() && key[i] == k) s += val[order[i++]];
    Lcol.push_back(uint32_t(k & 0xffffffffu));
    Lval.push_back(s);
    Lptr[(k >> 32) + 1]++;
  }
  for (size_t v = 0; v < n; ++v) Lptr[v + 1] += Lptr[v];
  Ldiag.assign(n, 0.0);
  for (size_t v = 0; v < n; ++v) {
    double s = 0.0;
    for (uint32_t e = Lptr[v]; e < Lptr[v + 1]; ++e) s += Lval[e];
    if (!(s > 0.0)) fail(GRAPH_UNIDENTIFIED, "operator", "hybrid Laplacian has an isolated vertex");
    Ldiag[v] = s;
  }
}


}  // namespace fevcb
