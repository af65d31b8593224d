// Aggregation multigrid preconditioner for the hybrid Laplacian.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <vector>

namespace fevcb {

class Multigrid {
 public:
  virtual ~Multigrid() = default;
  virtual int levels() const = 0;
  virtual int launches_per_apply() const = 0;
  // z = M^{-1} r for a block of K columns stored vertex-interleaved.
  virtual void apply(int K, const double* r, double* z, cudaStream_t s) = 0;
};

// Build the hierarchy from the finest-level Laplacian (CSR of positive
// off-diagonal conductances plus the diagonal).
std::unique_ptr<Multigrid> build_multigrid(uint32_t n, const std::vector<uint32_t>& ptr,
                                           const std::vector<uint32_t>& col, const std::vector<double>& val,
                                           const std::vector<double>& diag, cudaStream_t s, uint64_t& h2d_bytes);

}  // namespace fevcb
