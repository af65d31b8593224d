// Hybrid Laplacian of the two-way normal equations: workers with at most
// `max_degree` cells are eliminated exactly (a clique of conductances
// w_a w_b / d_w between their firms, the firm Schur complement of the
// reference's operator.rs:205-262); workers with more cells stay as star
// vertices.  The reference eliminates degrees up to four
// (vckss-core/src/cmg_impl.rs.in:71-364); the device engine eliminates up to
// sixteen, which keeps every worker of the generated panels out of the solve.
#pragma once

#include <cstdint>
#include <vector>

#include "prep.h"

namespace fevcb {

constexpr uint32_t ELIMINATE_MAX_DEGREE = 16;
constexpr uint32_t REFERENCE_ELIMINATE_MAX_DEGREE = 4;

void build_hybrid(const Compressed& p, uint32_t max_degree, std::vector<uint32_t>& kept_worker,
                  std::vector<int32_t>& kept_index, std::vector<double>& cell_scale, std::vector<double>& worker_diag,
                  std::vector<uint32_t>& Lptr, std::vector<uint32_t>& Lcol, std::vector<double>& Lval,
                  std::vector<double>& Ldiag);

}  // namespace fevcb
