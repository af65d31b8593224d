// Combinatorial (CMG-style) aggregation multigrid for the hybrid Laplacian:
// the device side.  The hierarchy is built on the host (cmg_host.h: the
// reference's forest aggregation and Galerkin contraction) once per prepared
// generation and uploaded; the cycle runs on the device on K vertex-
// interleaved columns.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <vector>

#include "cmg_host.h"

namespace fevcb {

class Multigrid {
 public:
  virtual ~Multigrid() = default;
  virtual int levels() const = 0;
  virtual int launches_per_apply() const = 0;
  virtual const MultigridReport& report() const = 0;
  // z = M^{-1} r for a block of K columns stored vertex-interleaved (K = 1, 8,
  // 16, 32 or 64).  Launches only kernels on `s` (capturable in a graph).
  virtual void apply(int K, const double* r, double* z, cudaStream_t s) = 0;
};

// Build the hierarchy from the finest-level Laplacian (CSR of positive
// off-diagonal conductances plus the diagonal) and upload it.
std::unique_ptr<Multigrid> build_multigrid(uint32_t n, const std::vector<uint32_t>& ptr,
                                           const std::vector<uint32_t>& col, const std::vector<double>& val,
                                           const std::vector<double>& diag, cudaStream_t s, uint64_t& h2d_bytes,
                                           const MultigridOptions& opt = MultigridOptions());

}  // namespace fevcb
