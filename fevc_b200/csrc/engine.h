// Device engine: the prepared problem resident in HBM and the JLA solve.
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "prep.h"
#include "projection.h"

namespace fevcb {

struct Components {
  double worker = 0, firm = 0, covariance = 0, total = 0;
};

enum class Centering : uint32_t { None = 0, Mean = 1, Corrected = 2 };

struct SolveOptions {
  uint64_t seed = 8675309;
  uint32_t probes = 200;
  uint32_t leverage_batch_width = 8;  // reference request field; the device block width is separate
  uint32_t target_batch_width = 8;
  double pcg_tolerance = 1e-10;
  uint32_t maximum_iterations = 10000;
  uint32_t residual_replacement_interval = 100;
  double rank_tolerance = 1e-10;
  double block_tolerance = 1e-10;
  Centering centering = Centering::None;
  int block_columns = 0;      // device RHS block width (0 = automatic)
  int preconditioner = 0;     // 0 automatic, 1 Jacobi, 2 aggregation multigrid
  uint32_t deletion_mode = 1;  // 1 match, 2 observation (must equal the prepared mode)
  uint32_t solver_route = 0;   // the request's route: 2 diagonal PCG, 3 CMG PCG, 0 automatic
  int precision = 0;           // 0 double, 1 FP32 storage with FP64 replacement, 2 autotuned per generation
  int algorithm = 2;           // 1 exact leverages (match deletion, no controls), 2 JLA
  uint64_t exact_limit = 500, blocksize_limit = 5000;  // exact-estimator gates
  // Probe sharding across devices: the leverage and target probes handled
  // here are [probe_begin, probe_end) of the request's probes (end 0: all).
  // Phase 1 runs the fit and the leverage probes and returns the leverage
  // accumulators; phase 2 starts from accumulators summed over all shards
  // (shard_input), runs the adjustment and the target probes and returns
  // their draws.  Phase 0 is the whole solve.
  int shard_phase = 0;
  uint32_t probe_begin = 0, probe_end = 0;
  const double* shard_input = nullptr;
  double* shard_output = nullptr;  // phase 1: the caller's accumulator buffer (host or device)
  // Probe sets: a later set of the same request on the same generation keeps
  // the fit (plug-in components, fitted cells, residuals) of the first one,
  // which no probe seed changes.
  bool reuse_fit = false;
  // Numerical MCSE attachment (reference `run_jla_no_controls_with_numerical_mc`):
  // per-unit derivatives after the adjustment, per-unit target folds during the
  // target phase, and a replay of the leverage probes that scores each one.
  bool numerical = false;
  // Fixed-effect projection attachment of the prepared generation (generic
  // JLA only): its columns are solved on the working model after the target
  // phase and their KSS covariance streamed over the deletion units.
  const PreparedProjection* projection = nullptr;
  // Fixed-offset nuisance (generic engine with controls): the controls'
  // coefficients of the joint fit are held fixed and everything after the
  // fit runs on the worker-firm model with y - Q'beta (reference
  // NuisanceMode::FixedOffset, generic_jla.rs:2011-2046)
  bool fixed_offset = false;
};

// One receipt per solved right-hand side (reference `JlaRhsReceipt`,
// vckss-core/src/engine.rs:185-195).
struct RhsReceipt {
  uint32_t phase;  // 1 fit, 2 leverage, 3 target
  uint32_t side;   // 1 joint, 2 worker, 3 firm
  int64_t probe;   // -1 for the fit
  uint32_t iterations;
  uint32_t zero_rhs;
  double reduced_residual;
  double complete_residual;
};

struct SolveTimings {
  double total_ms = 0, fit_ms = 0, leverage_ms = 0, target_ms = 0;
  uint64_t pcg_iterations = 0;      // summed over RHS blocks (block iterations)
  uint64_t column_iterations = 0;   // summed over RHS columns
  uint64_t rhs_columns = 0;
  uint64_t kernel_launches = 0;
  uint64_t spmm_launches = 0;
  double spmm_ms = 0;               // device time of the SpMM launches (events)
  uint64_t fallbacks = 0;           // learned-preconditioner blocks finished by the Jacobi fallback
};

// Numerical MCSE attachment of a solve (reference `CompressedNumericalMcResult`,
// vckss-core/src/engine/numerical.rs:13-34, and `numerical_mc::Covariance`).
// status: 1 exact zero, 2 local, 3 local after a PSD adjustment, 4 unstable
// (not PSD), 5 nonsmooth adjustment, 6 nonfinite derivative, 7 replay failed.
struct NumericalAttachment {
  bool present = false, exact = false;
  uint32_t status = 0;
  uint32_t engine = 1;  // 1 compressed, 2 generic (leave-observation-out)
  double conditional[3][3] = {}, leverage[3][3] = {}, raw[3][3] = {}, usable[3][3] = {};
  double mcse[4] = {};
  double psd_adjustment = 0;
  uint32_t leverage_probes = 0, target_probes = 0, folds[2] = {0, 0};
  uint64_t attempted_replay_rhs = 0, generator_words = 0, allocation_bound_bytes = 0;
  uint32_t failed_replay_probe = 0xffffffffu, replay_error_code = 0;
  double score_means[2][3] = {};
  double minimum_constrained = 0, minimum_residual_margin = 0, maximum_sensitivity_ratio = 0;
  std::vector<uint32_t> replay_probe;       // certified replay directions, in order
  std::vector<double> replay_residual;      // their complete residuals
};

struct SolveResult {
  Components plugin, correction, corrected, mcse;
  double weighted_rss = 0;
  bool weighted_rss_ready = false;  // computed on request (device_weighted_rss)
  std::vector<double> fitted_cell;
  std::vector<double> unit_projection_share, unit_residual_share, unit_finite_bias, unit_finite_variance;
  std::vector<double> unit_residual_mass, unit_deleted_mass, cell_correction_weight;
  std::vector<Components> target_draws;
  std::vector<RhsReceipt> receipts;
  double max_reduced_residual = 0, max_complete_residual = 0, max_leverage = 0;
  SolveTimings timings;
  std::vector<double> shard_accumulators;  // phase 1 output
  NumericalAttachment numerical;
  ProjectionResult projection;
};

// Number of leverage accumulators a shard exchanges (match units: 5 moment
// sums each; leave-observation-out: 4 sums per row and 4 per physical copy).
uint64_t shard_accumulator_count(const Compressed& p, const JlaPlan& plan);
// Correction, corrected components and MCSE from all probes' target draws.
void finish_draws(SolveResult& res, uint32_t probes);

struct DeviceEngine;  // opaque

struct DeviceStats {
  uint64_t h2d_bytes = 0;
  uint64_t vertices = 0, edges = 0, kept_workers = 0, levels = 0, terminal_vertices = 0;
  double setup_ms = 0;
  // setup phases (wall ms): the host builders (in launch order), their
  // parallel span, device-derived units, hybrid assembly, preconditioner
  int builders = 0;
  double builder_ms[16] = {};
  double builders_span_ms = 0, device_units_ms = 0, hybrid_ms = 0, preconditioner_ms = 0;
};

// Upload the prepared problem and build the solver.  Throws Error.
std::shared_ptr<DeviceEngine> make_device_engine(const Compressed& p, const JlaPlan& plan, int preconditioner);
DeviceStats device_stats(const DeviceEngine& e);
// The autotuner's candidates (precision, preconditioner, ms) and its choice (-1: not tuned).
int device_tuning(const DeviceEngine& e, int* precision, int* preconditioner, double* ms, int* candidates);
SolveResult device_solve(DeviceEngine& e, const Compressed& p, const JlaPlan& plan, const SolveOptions& o,
                         bool want_unit_detail);

// The device-assembled hybrid Laplacian (and segments, reconstruction arrays)
// equals the host builder's bit for bit.
bool device_hybrid_matches_host(DeviceEngine& e, const Compressed& p);

// Per-unit detail of the last solve without controls, read from the device
// on request (solves keep it there).
void device_unit_detail(DeviceEngine& e, SolveResult& res);
// Weighted residual sum of squares of the last solve's full fit, computed on request.
double device_weighted_rss(DeviceEngine& e, const Compressed& p);

// Time `launches` standalone launches of one hot kernel on the prepared
// problem with CUDA events (L2 flushed before each launch).  kernel: 1 the
// persistent blocked PCG form used at this width (20 iterations), 3 leverage
// Counter-V1 atoms with the per-cell sums, 4 leverage moments, 5 / 6 the
// three- / two-barrier persistent PCG.  Returns the
// median device milliseconds per launch and the algorithmic bytes per launch.
void device_kernel_benchmark(DeviceEngine& e, int kernel, int block_columns, int launches, double* ms_per_launch,
                             double* bytes_per_launch);

// Raw Counter-V1 atoms on the device (tests): out[e * columns + j] for probe first+j.
void device_atoms(uint64_t seed, uint64_t tag, uint64_t first_probe, uint32_t columns, const uint64_t* entity,
                  const uint64_t* trials, uint64_t count, int64_t* out);

// The same atoms staged through a fixed file-scope device array (no allocation).
void device_atoms_noalloc(uint64_t seed, uint64_t tag, uint64_t first_probe, uint32_t columns, const uint64_t* entity,
                          const uint64_t* trials, uint64_t count, int64_t* out);

int device_count();
// Kernels this library has launched since it was loaded (every launch passes
// through the wrapped CUDA runtime launch calls).
uint64_t kernel_launch_count();
// Adjusts that count for kernels that run from a CUDA graph: a replay launches
// them without passing through the wrapped calls, a capture passes through
// them without launching.
void count_replayed_launches(int64_t kernels);
// Device allocations released by finished generations stay cached for the
// next one (devmem.cu); the trim returns them to the driver (bytes freed).
size_t device_cache_trim();
size_t device_cache_bytes();
// Network parameters used by preconditioner 3 (learned) for engines built afterwards.
void set_learned_params(std::vector<float> params);
void set_device_stream(void* stream);
void* device_stream();

}  // namespace fevcb
