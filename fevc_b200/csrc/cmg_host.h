// Host construction of the combinatorial (CMG) aggregation hierarchy.
#pragma once

#include <cstdint>
#include <vector>

namespace fevcb {

enum CmgTerminal : int {
  CMG_NONE = 0,
  CMG_DIRECT = 1,
  CMG_FULL_CONTRACTION = 2,
  CMG_STAGNATED_VERTICES = 3,
  CMG_STAGNATED_FILL = 4,
  CMG_MAX_LEVELS = 5
};

struct MultigridReport {
  std::vector<uint32_t> vertices;  // per level
  std::vector<uint64_t> nonzeros;  // per level (off-diagonal entries, both directions)
  std::vector<int> repeat;         // per nonterminal level
  int terminal_reason = 0;         // CmgTerminal of the last level
};

struct MultigridOptions {
  uint32_t direct_threshold = 700;
  int max_levels = 32;
  double max_hierarchy_nnz_factor = 5.0;
  double low_effective_degree_threshold = 0.125;
};

// One level: the Laplacian (CSR of positive off-diagonal conductances and the
// degree diagonal), and for a nonterminal level its aggregation labels and
// the coarse repeat count; the direct terminal level holds the dense
// pseudo-inverse.
struct CmgLevel {
  uint32_t n = 0, nc = 0;
  std::vector<uint32_t> ptr, col, labels;
  std::vector<double> val, diag, pinv;
  int repeat = 0, terminal = CMG_NONE;
  uint64_t matrix_nnz() const { return uint64_t(n) + col.size(); }
};

// One forest aggregation step: labels[v] is the aggregate of vertex v,
// aggregates numbered in first-occurrence order of their union-find roots.
uint32_t forest_aggregation(uint32_t n, const std::vector<uint32_t>& ptr, const std::vector<uint32_t>& col,
                            const std::vector<double>& val, const std::vector<double>& diag, double threshold,
                            std::vector<uint32_t>& labels);

std::vector<CmgLevel> build_cmg_hierarchy(uint32_t n, const std::vector<uint32_t>& ptr,
                                          const std::vector<uint32_t>& col, const std::vector<double>& val,
                                          const std::vector<double>& diag, const MultigridOptions& opt,
                                          MultigridReport& report);

}  // namespace fevcb
