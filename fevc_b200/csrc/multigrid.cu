#include "common.h"
#include "multigrid.h"

namespace fevcb {

std::unique_ptr<Multigrid> build_multigrid(uint32_t, const std::vector<uint32_t>&, const std::vector<uint32_t>&,
                                           const std::vector<double>&, const std::vector<double>&, cudaStream_t,
                                           uint64_t&) {
  fail(UNSUPPORTED_FEATURE, "multigrid", "aggregation multigrid is not built yet");
}

}  // namespace fevcb
