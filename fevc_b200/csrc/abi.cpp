// C ABI of the library: the reference plugin's engine entry points over the
// host preparation and the device engine.  Semantics follow the reference
// registry (vckss-plugin/src/context.rs:100-530): one active generation,
// prepare -> solve -> result -> release, typed status codes with
// thread-local text (ffi_engine.rs:2469-2498).
#include <algorithm>
#include <cmath>
#include <chrono>
#include <cstring>
#include <thread>
#include <map>
#include <memory>
#include <mutex>
#include <string>

#include "fevc_b200.h"
#include "counter_rng.h"
#include "engine.h"
#include "numerical.h"
#include "cmg_host.h"
#include "hybrid.h"
#include "learned.h"
#include "prep.h"

using namespace fevcb;

namespace {

thread_local std::string g_last_error = "OK";

template <class F>
int32_t status(F&& f) {
  try {
    f();
    g_last_error = "OK";
    return OK;
  } catch (const Error& e) {
    g_last_error = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    g_last_error = "ALLOCATION_FAILED [host]: host allocation failed";
    return ALLOCATION_FAILED;
  } catch (const std::exception& e) {
    g_last_error = std::string("PANIC [ffi]: contained exception: ") + e.what();
    return PANIC;
  } catch (...) {
    g_last_error = "PANIC [ffi]: contained unknown exception";
    return PANIC;
  }
}

// Caller interrupt callback (reference `CallbackInterrupt::new`,
// ffi_engine.rs:1422-1461).  The callback is polled at the first checkpoint
// and again once `interval` items of work have passed; each checkpoint here
// reports the items of work (rows, right-hand sides) done since the last one.
struct Interrupt {
  VckssInterruptPollV1 poll = nullptr;
  void* ctx = nullptr;
  uint64_t interval = 0;
  mutable uint64_t remaining = 0;
  Interrupt() = default;
  Interrupt(VckssInterruptPollV1 p, void* c, uint32_t iv, uint32_t reserved, const char* label)
      : poll(p), ctx(c), interval(iv) {
    if (reserved != 0) fail(ABI_MISMATCH, "engine_ffi", std::string("reserved interrupt ") + label + " fields must be zero");
    if (!p && (c || interval != 0))
      fail(INVALID_INPUT, "engine_interrupt", "a null interrupt callback requires null context and zero interval");
    if (p && interval == 0)
      fail(INVALID_INPUT, "engine_interrupt", "a nonnull interrupt callback requires a positive checkpoint interval");
  }
  void check(const char* phase, uint64_t items = 1) const {
    if (!poll) return;
    if (remaining == 0) {
      if (poll(ctx) != VCKSS_INTERRUPT_CONTINUE) fail(USER_BREAK, phase, "interrupted by the caller");
      remaining = interval;
    }
    remaining = items >= remaining ? 0 : remaining - items;
  }
};

enum class State : uint32_t { Empty = 0, Prepared = 1, Solving = 2, Solved = 3, Failed = 4 };

struct Prepared {
  Compressed problem;
  JlaPlan plan;
  bool has_plan = false;
  GraphReceipt graph;
  std::vector<uint8_t> retained;
  uint64_t input_rows = 0;
  uint64_t memory_limit = 0, caller_copy = 0;
  uint32_t deletion_mode = VCKSS_DELETION_MATCH;
  uint32_t controls = 0;
  Centering centering = Centering::None;
  FevcbSolveOptionsV1 device_options{sizeof(FevcbSolveOptionsV1), 0, 0, 0};
  std::vector<double> control_values;  // contiguous copy for the problem view
  std::shared_ptr<DeviceEngine> device;
  int device_preconditioner = 0;  // preconditioner the device engine was built with
  Components shard_plugin;        // plug-in components of the last shard
  SolveTimings shard_timings;     // solver counts of the shards since the last finish
  uint32_t precision = 0;         // device option: 1 mixed-precision inner solves
  SolveOptions last_options;
  bool solved_once = false;
  uint64_t topology_checksum = 0;            // of the compressed problem, computed on request
  bool checksum_ready = false;
  uint32_t solve_version = 0;                // request version of the last solve: 1, 4, 5 or 8
  VckssEngineSolveRequestV4 last_request{};  // the last V4+ request (capability and batch fields)
  // ceiling on the identified dimension of an exact solve above the
  // reference's 2,000 (fevcb_engine_exact_limit_v1); 0: the request's limit
  uint64_t exact_ceiling = 0;
  // host preparation phases, wall milliseconds: ingest copy, canonical ids,
  // graph fixed point, compression, JLA plan
  double prepare_ms[5] = {0, 0, 0, 0, 0};
  // fixed-effect projection attached before the first solve
  std::shared_ptr<PreparedProjection> projection;
};

struct Registry {
  std::mutex mu;
  uint64_t next = 1, last_released = 0, generation = 0;
  State state = State::Empty;
  std::unique_ptr<Prepared> prepared;
  std::unique_ptr<SolveResult> result;
  std::string failure;

  Prepared& require(uint64_t g, const char* phase) {
    if (state == State::Empty || g != generation)
      fail(STALE_CONTEXT, phase, "generation " + std::to_string(g) + " is not the active context");
    return *prepared;
  }
};

Registry& reg() {
  static Registry r;
  return r;
}

template <class T>
void require_capacity(const void* p, uint64_t cap, const char* label) {
  if (!p) fail(INVALID_INPUT, "engine_ffi", std::string(label) + " pointer is null");
  if (cap < sizeof(T))  // a short output is an ABI mismatch (ffi_engine.rs `require_output_capacity`)
    fail(ABI_MISMATCH, "engine_ffi",
         std::string(label) + " capacity " + std::to_string(cap) + " is below " + std::to_string(sizeof(T)));
}

// Copy a caller struct after checking the size it reports (reference
// `copy_request_struct` / `copy_sized_struct`, ffi_engine.rs:10815-10830):
// requests carry struct_size at byte offset 4, descriptors at offset 0.
template <class T>
T read_struct(const T* p, const char* label, size_t size_offset = 4) {
  if (!p) fail(INVALID_INPUT, "engine_ffi", std::string(label) + " pointer is null");
  uint32_t reported = 0;
  std::memcpy(&reported, reinterpret_cast<const char*>(p) + size_offset, 4);
  if (reported < sizeof(T))
    fail(ABI_MISMATCH, "engine_ffi",
         std::string(label) + " size " + std::to_string(reported) + " is below required size " +
             std::to_string(sizeof(T)));
  T v;
  std::memcpy(&v, p, sizeof(T));
  return v;
}

void require_abi(uint32_t v) {
  if (v != VCKSS_RUST_ABI_VERSION_V1) fail(ABI_MISMATCH, "engine_ffi", "unsupported ABI version " + std::to_string(v));
}

void clear_abandoned(uint32_t flag) {
  if (flag > 1) fail(INVALID_INPUT, "engine_prepare", "cleanup_abandoned must be zero or one");
  Registry& r = reg();
  if (flag && r.state != State::Empty) {
    r.last_released = std::max(r.last_released, r.generation);
    r.state = State::Empty;
    r.prepared.reset();
    r.result.reset();
  }
}

struct PrepareArgs {
  uint64_t rows;
  uint32_t cleanup;
  bool explicit_memory = false;  // V2+ requests carry a memory budget that must be positive
  uint64_t memory_limit = 0, caller_copy = 0;
  uint32_t deletion_mode = VCKSS_DELETION_MATCH;
  uint32_t implicit_match = 0;
  const VckssEngineColumnsV1* v1 = nullptr;
  const double* const* controls = nullptr;
  uint32_t controls_count = 0;
  const double* probe_order = nullptr;
  Interrupt interrupt;
};

void prepare_common(const PrepareArgs& a, uint64_t* out, uint32_t cap) {
  require_capacity<uint64_t>(out, cap, "engine output handle");
  uint64_t zero = 0;
  std::memcpy(out, &zero, 8);
  if (a.rows == 0 || a.rows != a.v1->rows)
    fail(INVALID_INPUT, "engine_prepare", "request and column row counts must agree and be positive");
  if (a.v1->reserved != 0) fail(ABI_MISMATCH, "engine_ffi", "reserved preparation fields must be zero");
  if (a.deletion_mode != VCKSS_DELETION_MATCH && a.deletion_mode != VCKSS_DELETION_OBSERVATION)
    fail(INVALID_INPUT, "engine_prepare", "unknown deletion mode");
  if (a.implicit_match && a.deletion_mode != VCKSS_DELETION_MATCH)
    fail(INVALID_INPUT, "session_prepare", "implicit-match preparation requires match deletion");
  if (a.cleanup > 1) fail(INVALID_INPUT, "engine_prepare", "cleanup_abandoned must be zero or one");
  // the budget must be positive (reference memory.rs:33); forecasting against it is not replicated
  if (a.explicit_memory && a.memory_limit == 0)
    fail(INVALID_INPUT, "memory_budget", "an explicit memory budget must be positive");
  if (a.explicit_memory) {
    // the declared caller copy must equal the binary64 columns handed over
    // (reference vckss-plugin/src/session.rs:111-121, 218-232)
    uint64_t columns = 6 + a.controls_count + (a.probe_order ? 1 : 0);
    uint64_t expected = a.rows * columns * 8;
    if (a.caller_copy != expected)
      fail(INVALID_INPUT, "engine_memory",
           "declared caller copy is " + std::to_string(a.caller_copy) + " bytes; " +
               (columns == 6 ? std::string("six") : std::to_string(columns)) + " columns require " +
               std::to_string(expected) + " bytes");
  }
  {
    std::lock_guard<std::mutex> l(reg().mu);
    clear_abandoned(a.cleanup);
    if (reg().state != State::Empty)
      fail(CONTEXT_POISONED, "context_prepare",
           "generation " + std::to_string(reg().generation) + " is still active; release it before preparing another context");
  }
  a.interrupt.check("engine_prepare_entry");
  auto prep = std::make_unique<Prepared>();
  auto tick = std::chrono::steady_clock::now();
  auto lap = [&](int phase) {
    auto t = std::chrono::steady_clock::now();
    prep->prepare_ms[phase] = std::chrono::duration<double, std::milli>(t - tick).count();
    tick = t;
  };
  InputColumns in = copy_columns(a.rows, a.v1->worker, a.v1->firm, a.v1->deletion, a.v1->outcome, a.v1->frequency,
                                 a.v1->target_weight, a.controls, a.controls_count, a.probe_order);
  lap(0);
  a.interrupt.check("engine_ingest", a.rows);
  Canonical canon = canonicalize(std::move(in), a.implicit_match != 0);
  lap(1);
  a.interrupt.check("canonicalize_final", a.rows);
  if (a.deletion_mode == VCKSS_DELETION_OBSERVATION)
    prep->retained = select_observation_graph(canon, prep->graph);
  else if (a.implicit_match)
    prep->retained = select_implicit_match_graph(canon, prep->graph);
  else
    prep->retained = select_match_graph(canon, prep->graph);
  lap(2);
  a.interrupt.check("graph_final", a.rows);
  prep->problem = compress(canon, prep->retained, a.implicit_match != 0);
  lap(3);
  a.interrupt.check("compression_final", a.rows);
  if (a.deletion_mode == VCKSS_DELETION_MATCH)
    prep->plan = prep->problem.controls.empty() ? build_plan(prep->problem) : build_generic_plan(prep->problem);
  else
    prep->plan = build_generic_plan(prep->problem, Deletion::Observation);
  lap(4);
  prep->has_plan = true;
  prep->input_rows = a.rows;
  prep->memory_limit = a.memory_limit;
  prep->caller_copy = a.caller_copy;
  prep->deletion_mode = a.deletion_mode;
  prep->controls = a.controls_count;
  a.interrupt.check("engine_prepare_final", a.rows);
  std::lock_guard<std::mutex> l(reg().mu);
  Registry& r = reg();
  if (r.state != State::Empty) fail(CONTEXT_POISONED, "context_prepare", "another generation became active");
  r.generation = r.next++;
  r.state = State::Prepared;
  r.prepared = std::move(prep);
  r.result.reset();
  std::memcpy(out, &r.generation, 8);
}

SolveOptions options_from_v1(const VckssEngineSolveRequestV1& q, bool observation_allowed = false,
                             bool exact = false) {
  require_abi(q.abi_version);
  if (q.deletion_mode != VCKSS_DELETION_MATCH &&
      !(observation_allowed && q.deletion_mode == VCKSS_DELETION_OBSERVATION))
    fail(UNSUPPORTED_FEATURE, "jla_validate", "the compressed JLA engine supports match deletion only");
  if (!exact && q.rng_contract != VCKSS_RNG_COUNTER_V1)
    fail(UNSUPPORTED_FEATURE, "jla_validate", "the JLA engine supports VCKSS-COUNTER-V1 only");
  if (!exact && q.probes < 2) fail(INVALID_INPUT, "jla_validate", "JLA probe count must be at least two");
  if (q.leverage_batch_width == 0 || q.target_batch_width == 0)
    fail(INVALID_INPUT, "jla_validate", "leverage and target batch widths must be positive");
  if (!(q.rank_tolerance >= 1e-14 && q.rank_tolerance < 0.1))
    fail(INVALID_INPUT, "jla_validate", "rank tolerance must be finite and lie in [1e-14, 0.1)");
  if (!(q.block_tolerance >= 1e-14 && q.block_tolerance < 1.0))
    fail(INVALID_INPUT, "jla_validate", "block tolerance must be finite and lie in [1e-14, 1)");
  if (!(q.pcg_tolerance > 0.0 && q.pcg_tolerance < 1.0))
    fail(INVALID_INPUT, "pcg", "PCG tolerance must lie in (0, 1)");
  if (q.maximum_iterations == 0) fail(INVALID_INPUT, "pcg", "maximum iterations must be positive");
  if (q.residual_replacement_interval == 0) fail(INVALID_INPUT, "pcg", "residual replacement interval must be positive");
  if (q.solver_route > VCKSS_ROUTE_CMG_PCG) fail(INVALID_INPUT, "solver_router", "unknown solver route");
  SolveOptions o;
  o.seed = q.seed;
  o.probes = q.probes;
  o.leverage_batch_width = q.leverage_batch_width;
  o.target_batch_width = q.target_batch_width;
  o.pcg_tolerance = q.pcg_tolerance;
  o.maximum_iterations = q.maximum_iterations;
  o.residual_replacement_interval = q.residual_replacement_interval;
  o.rank_tolerance = q.rank_tolerance;
  o.block_tolerance = q.block_tolerance;
  o.deletion_mode = q.deletion_mode;
  o.solver_route = q.solver_route;
  return o;
}

// ---- request capability (restated from vckss-plugin/src/ffi_engine.rs:9304-9532)

VckssBackendRequestCapabilityRequestV3 capability_request_for_solve(const VckssEngineSolveRequestV4& q,
                                                                    uint32_t controls_count) {
  VckssBackendRequestCapabilityRequestV3 c{};
  c.v2.v1.abi_version = q.v3.v2.v1.abi_version;
  c.v2.v1.struct_size = sizeof(c);
  c.v2.v1.request_schema = q.v3.capability_schema;
  c.v2.v1.algorithm = q.v3.v2.algorithm;
  c.v2.v1.deletion_mode = q.v3.v2.v1.deletion_mode;
  c.v2.v1.nuisance_mode = q.v3.v2.nuisance_mode;
  c.v2.v1.solver_route = q.v3.v2.v1.solver_route;
  c.v2.v1.rng_contract = q.v3.v2.v1.rng_contract;
  c.v2.v1.controls_count = controls_count;
  c.v2.v1.frequency_use = q.v3.frequency_use;
  c.v2.engine = q.v3.engine;
  c.v2.batch_mode = q.v3.batch_mode;
  c.v2.stayers_mode = q.v3.stayers_mode;
  c.v2.target_weight_mode = q.v3.target_weight_mode;
  c.v2.deletion_unit_source = q.v3.deletion_unit_source;
  c.v2.probeorder_supplied = q.v3.probeorder_supplied;
  c.v2.wallseconds_supplied = q.v3.wallseconds_supplied;
  c.v2.physical_limit = q.v3.physical_limit;
  c.leverage_batch_mode = q.leverage_batch_mode;
  c.target_batch_mode = q.target_batch_mode;
  c.allow_automatic_cmg_setup_fallback = q.v3.v2.v1.allow_automatic_cmg_setup_fallback;
  c.wallseconds = q.wallseconds;
  return c;
}

// FNV-1a over the schema tag, the capability fields (little-endian u32),
// the physical limit and the bits of the wall-seconds value.
uint64_t capability_signature(const VckssBackendRequestCapabilityRequestV3& c) {
  uint64_t h = 0xcbf29ce484222325ull;
  auto eat = [&](const void* data, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(data);
    for (size_t i = 0; i < n; ++i) {
      h ^= b[i];
      h *= 0x100000001b3ull;
    }
  };
  static const char tag[] = "VCKSS-REQUEST-CAPABILITY-V3";
  eat(tag, sizeof(tag) - 1);
  const uint32_t fields[] = {c.v2.v1.request_schema, c.v2.v1.algorithm, c.v2.v1.deletion_mode, c.v2.v1.nuisance_mode,
                             c.v2.v1.solver_route, c.v2.v1.rng_contract, c.v2.v1.controls_count,
                             c.v2.v1.frequency_use, c.v2.engine, c.v2.batch_mode, c.v2.stayers_mode,
                             c.v2.target_weight_mode, c.v2.deletion_unit_source, c.v2.probeorder_supplied,
                             c.v2.wallseconds_supplied, c.leverage_batch_mode, c.target_batch_mode,
                             c.allow_automatic_cmg_setup_fallback};
  for (uint32_t f : fields) eat(&f, 4);  // little-endian host
  eat(&c.v2.physical_limit, 8);
  uint64_t bits;
  std::memcpy(&bits, &c.wallseconds, 8);
  eat(&bits, 8);
  return h;
}

uint32_t capability_reason(const VckssBackendRequestCapabilityRequestV3& c) {
  const auto& v = c.v2.v1;
  const auto& r = c.v2;
  auto known_batch = [](uint32_t m) { return m == VCKSS_BATCH_MODE_AUTO || m == VCKSS_BATCH_MODE_EXPLICIT; };
  uint32_t summary = (c.leverage_batch_mode == VCKSS_BATCH_MODE_AUTO && c.target_batch_mode == VCKSS_BATCH_MODE_AUTO)
                         ? VCKSS_BATCH_MODE_AUTO
                     : (c.leverage_batch_mode == VCKSS_BATCH_MODE_EXPLICIT &&
                        c.target_batch_mode == VCKSS_BATCH_MODE_EXPLICIT)
                         ? VCKSS_BATCH_MODE_EXPLICIT
                         : VCKSS_BATCH_MODE_INDEPENDENT;
  bool source_matches = (v.deletion_mode == VCKSS_DELETION_MATCH &&
                         (r.deletion_unit_source == VCKSS_DELETION_SOURCE_CELL_DEFAULT ||
                          r.deletion_unit_source == VCKSS_DELETION_SOURCE_MATCH_ID_EXPLICIT)) ||
                        (v.deletion_mode == VCKSS_DELETION_OBSERVATION &&
                         r.deletion_unit_source == VCKSS_DELETION_SOURCE_OBSERVATION_ROW);
  const bool all_stayers = r.stayers_mode == VCKSS_STAYERS_ALL;
  if (v.request_schema != VCKSS_REQUEST_CAPABILITY_SCHEMA_V3) return VCKSS_REQUEST_REASON_UNKNOWN_SCHEMA;
  if (v.algorithm > VCKSS_ALGORITHM_JLA) return VCKSS_REQUEST_REASON_UNKNOWN_ALGORITHM;
  if (v.deletion_mode != VCKSS_DELETION_MATCH && v.deletion_mode != VCKSS_DELETION_OBSERVATION)
    return VCKSS_REQUEST_REASON_UNKNOWN_DELETION;
  if (v.nuisance_mode != VCKSS_NUISANCE_JOINT && v.nuisance_mode != VCKSS_NUISANCE_FIXED_OFFSET)
    return VCKSS_REQUEST_REASON_UNKNOWN_NUISANCE;
  if (v.solver_route > VCKSS_ROUTE_CMG_PCG) return VCKSS_REQUEST_REASON_UNKNOWN_SOLVER_ROUTE;
  if (v.rng_contract != VCKSS_RNG_NONE && v.rng_contract != VCKSS_RNG_COUNTER_V1)
    return VCKSS_REQUEST_REASON_UNKNOWN_RNG_CONTRACT;
  if (v.frequency_use != VCKSS_REQUEST_FREQUENCY_UNIT && v.frequency_use != VCKSS_REQUEST_FREQUENCY_LITERAL)
    return VCKSS_REQUEST_REASON_UNKNOWN_FREQUENCY_USE;
  if (r.engine > VCKSS_ENGINE_GENERIC) return VCKSS_REQUEST_REASON_UNKNOWN_ENGINE;
  if (!known_batch(c.leverage_batch_mode) || !known_batch(c.target_batch_mode))
    return VCKSS_REQUEST_REASON_UNKNOWN_BATCH_MODE;
  if (r.batch_mode > VCKSS_BATCH_MODE_INDEPENDENT || r.batch_mode != summary)
    return VCKSS_REQUEST_REASON_BATCH_SUMMARY_MISMATCH;
  if (r.stayers_mode != VCKSS_STAYERS_MOVERS && r.stayers_mode != VCKSS_STAYERS_ALL)
    return VCKSS_REQUEST_REASON_UNKNOWN_STAYERS_MODE;
  if (r.target_weight_mode > VCKSS_TARGET_WEIGHT_STORED_ROW_EXPLICIT)
    return VCKSS_REQUEST_REASON_UNKNOWN_TARGET_WEIGHT_MODE;
  if (r.deletion_unit_source < VCKSS_DELETION_SOURCE_CELL_DEFAULT ||
      r.deletion_unit_source > VCKSS_DELETION_SOURCE_OBSERVATION_ROW)
    return VCKSS_REQUEST_REASON_UNKNOWN_DELETION_UNIT_SOURCE;
  if (!source_matches) return VCKSS_REQUEST_REASON_DELETION_UNIT_SOURCE_MISMATCH;
  if (r.probeorder_supplied > 1) return VCKSS_REQUEST_REASON_PROBEORDER_UNSUPPORTED;
  if (r.wallseconds_supplied > 1 || (r.wallseconds_supplied == 0 && c.wallseconds != 0.0) ||
      (r.wallseconds_supplied == 1 && (!std::isfinite(c.wallseconds) || c.wallseconds <= 0.0)))
    return VCKSS_REQUEST_REASON_WALLSECONDS_VALUE;
  if (c.allow_automatic_cmg_setup_fallback > 1 ||
      (c.allow_automatic_cmg_setup_fallback == 1 && v.solver_route != VCKSS_ROUTE_AUTO))
    return VCKSS_REQUEST_REASON_FALLBACK_ROUTE_MISMATCH;
  if (r.physical_limit == 0 || r.physical_limit > MAX_EXACT_BINARY64_INTEGER)
    return VCKSS_REQUEST_REASON_PHYSICAL_LIMIT;
  if (v.controls_count > 32) return VCKSS_REQUEST_REASON_CONTROLS_LIMIT;
  if (v.algorithm == VCKSS_ALGORITHM_EXACT) {
    if (r.engine == VCKSS_ENGINE_COMPRESSED) return VCKSS_REQUEST_REASON_EXACT_ENGINE;
    if (all_stayers && v.deletion_mode != VCKSS_DELETION_MATCH) return VCKSS_REQUEST_REASON_STAYERS_MODE_UNSUPPORTED;
    if (all_stayers && r.probeorder_supplied != 0) return VCKSS_REQUEST_REASON_PROBEORDER_UNSUPPORTED;
    if (all_stayers && r.wallseconds_supplied != 0) return VCKSS_REQUEST_REASON_WALLSECONDS_UNSUPPORTED;
    if (v.rng_contract != VCKSS_RNG_NONE) return VCKSS_REQUEST_REASON_EXACT_RNG;
    if (v.solver_route != VCKSS_ROUTE_AUTO && v.solver_route != VCKSS_ROUTE_EXACT)
      return VCKSS_REQUEST_REASON_EXACT_SOLVER_ROUTE;
    return VCKSS_REQUEST_REASON_SUPPORTED;
  }
  if (all_stayers && v.deletion_mode != VCKSS_DELETION_MATCH) return VCKSS_REQUEST_REASON_STAYERS_MODE_UNSUPPORTED;
  if (all_stayers && r.engine == VCKSS_ENGINE_COMPRESSED)
    return VCKSS_REQUEST_REASON_COMPRESSED_SCIENTIFIC_INELIGIBILITY;
  if (all_stayers && r.probeorder_supplied != 0) return VCKSS_REQUEST_REASON_PROBEORDER_UNSUPPORTED;
  if (all_stayers && r.wallseconds_supplied != 0) return VCKSS_REQUEST_REASON_WALLSECONDS_UNSUPPORTED;
  if (v.algorithm == VCKSS_ALGORITHM_AUTO) {
    if (v.rng_contract != VCKSS_RNG_COUNTER_V1) return VCKSS_REQUEST_REASON_AUTO_RNG;
    if (v.solver_route != VCKSS_ROUTE_AUTO) return VCKSS_REQUEST_REASON_EXACT_SOLVER_ROUTE;
    if (r.engine == VCKSS_ENGINE_COMPRESSED) return VCKSS_REQUEST_REASON_AUTO_ENGINE_COMPRESSED;
    return VCKSS_REQUEST_REASON_SUPPORTED;
  }
  if (v.rng_contract != VCKSS_RNG_COUNTER_V1) return VCKSS_REQUEST_REASON_JLA_RNG;
  if (v.solver_route == VCKSS_ROUTE_EXACT) return VCKSS_REQUEST_REASON_JLA_GENERIC_SOLVER_ROUTE;
  if (r.engine == VCKSS_ENGINE_COMPRESSED &&
      (v.deletion_mode != VCKSS_DELETION_MATCH || v.controls_count != 0))
    return VCKSS_REQUEST_REASON_COMPRESSED_SCIENTIFIC_INELIGIBILITY;
  return VCKSS_REQUEST_REASON_SUPPORTED;
}

// The V4+ solve gate (reference ffi_engine.rs:4808-4839): the request's
// probe-order declaration must match the prepared input, and its profile and
// signature must be those the capability receipt reports for it.
void reconcile_capability(const Prepared& p, const VckssEngineSolveRequestV4& q) {
  if (q.v3.probeorder_supplied != (p.problem.probe_order.empty() ? 0u : 1u))
    fail(INVALID_INPUT, "engine_solve", "solve probe-order declaration differs from prepared input");
  auto c = capability_request_for_solve(q, uint32_t(p.problem.controls.size()));
  uint32_t reason = capability_reason(c);
  uint32_t profile = reason == VCKSS_REQUEST_REASON_SUPPORTED ? VCKSS_REQUEST_PROFILE_PLANNED_V1
                                                               : VCKSS_REQUEST_PROFILE_NONE;
  if (reason != VCKSS_REQUEST_REASON_SUPPORTED || profile != q.v3.capability_profile ||
      capability_signature(c) != q.v3.request_signature)
    fail(UNSUPPORTED_FEATURE, "engine_solve", "V4 solve does not reconcile with its V3 capability receipt");
}

SolveOptions options_from_v4(const VckssEngineSolveRequestV4& q) {
  // preamble of the reference's V4 solve (ffi_engine.rs:4727-4766)
  if (q.v3.v2.v1.struct_size < sizeof(VckssEngineSolveRequestV4))
    fail(ABI_MISMATCH, "engine_ffi", "V4 solve request reports a short structure size");
  if (q.v3.reserved_3 != 0 || q.reserved_4 != 0)
    fail(ABI_MISMATCH, "engine_ffi", "reserved V4 solve request fields must be zero");
  if (q.v3.capability_schema != VCKSS_REQUEST_CAPABILITY_SCHEMA_V3 ||
      q.v3.capability_profile != VCKSS_REQUEST_PROFILE_PLANNED_V1)
    fail(UNSUPPORTED_FEATURE, "engine_solve", "V4 solve requires the planned-command V3 capability profile");
  if (q.v3.v2.algorithm != VCKSS_ALGORITHM_EXACT && q.v3.v2.v1.probes < 2)
    fail(INVALID_INPUT, "engine_solve", "JLA-capable V4 requests require at least two probes");
  VckssEngineSolveRequestV1 v1 = q.v3.v2.v1;
  if (v1.leverage_batch_width == 0) v1.leverage_batch_width = 8;
  if (v1.target_batch_width == 0) v1.target_batch_width = 8;
  if (q.v3.v2.algorithm == VCKSS_ALGORITHM_EXACT) {
    // the reference's exact-estimator option gates
    // (vckss-core/src/exact_estimator.rs:76-125)
    if (q.v3.v2.exact_estimator_limit < 2 || q.v3.v2.exact_estimator_limit > 2000)
      fail(INVALID_INPUT, "exact_estimator", "exact limit must lie in [2, 2000]");
    if (q.v3.v2.blocksize_limit == 0 || q.v3.v2.blocksize_limit > 1000000)
      fail(INVALID_INPUT, "exact_estimator", "block-size limit must lie in [1, 1000000]");
    SolveOptions o = options_from_v1(v1, false, true);
    o.algorithm = 1;
    o.exact_limit = q.v3.v2.exact_estimator_limit;
    o.blocksize_limit = q.v3.v2.blocksize_limit;
    return o;
  }
  SolveOptions o = options_from_v1(v1, true);
  o.fixed_offset = q.v3.v2.nuisance_mode == VCKSS_NUISANCE_FIXED_OFFSET;
  return o;
}

// The exact path covers match deletion without controls: every deletion
// block is one match whose rows share a design row.  The identified
// dimension W + F - 1 must fit the request's exact limit (or the ceiling a
// caller raised with fevcb_engine_exact_limit_v1), as in the reference's
// estimator (exact_estimator.rs:511-526); so must each block's rows.
void exact_gate(const Prepared& p, const SolveOptions& o) {
  if (p.controls != 0 || p.plan.generic || p.deletion_mode != VCKSS_DELETION_MATCH)
    fail(UNSUPPORTED_FEATURE, "exact_estimator",
         "the device exact estimator covers match deletion without controls");
  const uint64_t parameters = uint64_t(p.problem.workers) + p.problem.firms - 1;
  const uint64_t limit = std::max<uint64_t>(o.exact_limit, p.exact_ceiling);
  if (parameters > limit)
    fail(RESOURCE_LIMIT, "exact_estimator", "identified coefficient dimension exceeds exact_limit()");
  const auto& di = p.problem.deletion_index.ptr;
  for (size_t g = 0; g + 1 < di.size(); ++g)
    if (di[g + 1] - di[g] > o.blocksize_limit)
      fail(RESOURCE_LIMIT, "exact_estimator", "a deletion block exceeds blocksize_limit()");
}

void solve_common(uint64_t g, SolveOptions o, const Interrupt& intr, bool generic_allowed,
                  const VckssEngineSolveRequestV4* v4 = nullptr, uint32_t version = 1) {
  Registry& r = reg();
  std::unique_lock<std::mutex> l(r.mu);
  Prepared& p = r.require(g, "context_solve");
  if (p.has_plan && p.plan.generic && !generic_allowed)
    fail(UNSUPPORTED_FEATURE, "engine_solve", "the frozen V1 JLA solve requires a prepared no-control match plan");
  if (r.state != State::Prepared)
    fail(STALE_CONTEXT, "context_solve", "generation " + std::to_string(g) + " is not in the prepared state");
  if (!p.has_plan)
    fail(UNSUPPORTED_FEATURE, "engine_solve", "the compressed JLA solve requires a prepared no-control match plan");
  if (v4) reconcile_capability(p, *v4);
  if (o.deletion_mode != p.deletion_mode)
    fail(INVALID_INPUT, "engine_solve", "solve deletion mode differs from the prepared graph mode");
  if (o.algorithm == 1) exact_gate(p, o);
  if (p.projection) {  // ffi_engine.rs:4936-4944
    if (!p.plan.generic || o.algorithm == 1)
      fail(UNSUPPORTED_FEATURE, "engine_solve",
           "prepared projection or component-inference attachments require the generic JLA engine");
    o.projection = p.projection.get();
  }
  r.state = State::Solving;
  try {
    intr.check("jla_full_fit");
    o.centering = p.centering;
    o.block_columns = int(p.device_options.block_columns);
    o.precision = int(p.precision);
    // the device option wins; otherwise the request's route picks the
    // preconditioner (CMG route -> aggregation multigrid, else Jacobi)
    o.preconditioner = int(p.device_options.preconditioner);
    if (o.preconditioner == 0) o.preconditioner = o.solver_route == VCKSS_ROUTE_CMG_PCG ? 2 : 1;
    if (p.device && p.device_preconditioner != o.preconditioner) p.device.reset();
    if (!p.device) {
      p.device = make_device_engine(p.problem, p.plan, o.preconditioner);
      p.device_preconditioner = o.preconditioner;
    }
    // per-unit detail stays on the device until a caller asks for it
    auto res = std::make_unique<SolveResult>(device_solve(*p.device, p.problem, p.plan, o, false));
    intr.check("jla_finalize");
    p.last_options = o;
    p.solved_once = true;
    p.solve_version = version;
    p.last_request = v4 ? *v4 : VckssEngineSolveRequestV4{};
    r.result = std::move(res);
    r.state = State::Solved;
  } catch (...) {
    r.state = State::Failed;
    throw;
  }
}


// Detailed receipt of the last solve (reference `detailed_receipt` ..
// `detailed_receipt_v6` and the execution plan, vckss-plugin/src/
// ffi_engine.rs:7443-8100, 6297-6330).  Filled: the request and what this
// engine did with it (seed, probes, widths, tolerances, routes, counts, the
// fit, residual maxima, maximum leverage, accounting, topology checksum, the
// CMG structure, the capability fields); the reference's CPU memory, thread
// and wall forecasts have no counterpart here and stay zero.
VckssEngineDetailedReceiptV7 detailed_receipt(uint64_t g, const Prepared& p, const SolveResult& res) {
  const SolveOptions& o = p.last_options;
  const VckssEngineSolveRequestV3& q3 = p.last_request.v3;
  VckssEngineDetailedReceiptV7 d{};
  VckssEngineDetailedReceiptV2& v2 = d.v6.v5.v4.v3.v2;
  DeviceStats st = p.device ? device_stats(*p.device) : DeviceStats{};
  const uint32_t route = o.preconditioner == 2 ? VCKSS_ROUTE_CMG_PCG : VCKSS_ROUTE_DIAGONAL_PCG;
  v2.struct_size = sizeof(VckssEngineDetailedReceiptV2);
  v2.generation = g;
  v2.seed = o.seed;
  v2.probes_requested = o.probes;
  v2.leverage_probes_accepted = o.probes;
  v2.target_probes_accepted = o.probes;
  v2.solver_requested = o.solver_route;
  v2.solver_selected = route;
  v2.solver_fallback = res.timings.fallbacks ? 1 : 0;
  // the grounded firm quotient F - 1; the generic estimator's joint system
  // keeps all F firms and adds the control block
  v2.solver_dimension = p.plan.generic ? p.problem.firms + p.controls : p.problem.firms - 1;
  v2.leverage_batch_width = o.leverage_batch_width;
  v2.target_batch_width = o.target_batch_width;
  v2.rank_tolerance = o.rank_tolerance;
  v2.block_tolerance = o.block_tolerance;
  v2.full_residual_tolerance = std::max(10.0 * o.pcg_tolerance, 1e-11);
  uint64_t lev = 0, tgt = 0;
  for (const RhsReceipt& r : res.receipts) {
    if (r.phase == 1) {
      v2.full_fit_route = route;
      v2.full_fit_iterations = r.iterations;
      v2.full_fit_reduced_residual = r.reduced_residual;
      v2.full_fit_complete_residual = r.complete_residual;
      v2.full_fit_zero_rhs = r.zero_rhs;
    }
    lev += r.phase == 2;
    tgt += r.phase == 3;
  }
  v2.leverage_rhs_count = lev;
  v2.target_rhs_count = tgt;
  v2.max_reduced_residual = res.max_reduced_residual;
  v2.max_complete_residual = res.max_complete_residual;
  v2.max_leverage = res.max_leverage;
  // |M (1/M) - 1| over the units' residual shares (reference engine.rs:2347-2382)
  for (double share : res.unit_residual_share)
    if (share > 0.0) v2.max_reciprocal_residual = std::max(v2.max_reciprocal_residual, std::fabs(share * (1.0 / share) - 1.0));
  // scaled |total - worker - firm - 2 cov| over the plug-in, correction,
  // corrected components and every draw (reference engine.rs:3227-3317)
  auto identity = [](const Components& c) {
    double scale = std::max({std::fabs(c.worker), std::fabs(c.firm), std::fabs(c.covariance), std::fabs(c.total), 1.0});
    return std::fabs(c.total - c.worker - c.firm - 2.0 * c.covariance) / scale;
  };
  v2.accounting_residual = std::max({identity(res.plugin), identity(res.correction), identity(res.corrected)});
  for (const Components& dr : res.target_draws) v2.accounting_residual = std::max(v2.accounting_residual, identity(dr));
  v2.topology_checksum = p.topology_checksum;
  if (o.preconditioner == 2) {
    v2.cmg_levels = st.levels;
    v2.cmg_fine_vertices = st.vertices;
    v2.cmg_fine_edges = st.edges;
    v2.cmg_terminal_vertices = st.terminal_vertices;
  }
  v2.full_fit_weighted_rss = res.weighted_rss;
  v2.memory_limit_bytes = p.memory_limit;
  v2.caller_copy_bytes = p.caller_copy;
  v2.prepared_resident_bytes = st.h2d_bytes;
  VckssEngineDetailedReceiptV3& v3 = d.v6.v5.v4.v3;
  v3.rng_contract = VCKSS_RNG_COUNTER_V1;
  v3.rhs_receipt_rows = res.receipts.size();
  v3.caller_result_copy_bytes = p.plan.generic ? 0 : res.receipts.size() * 14 * 8;
  VckssEngineDetailedReceiptV4& v4 = d.v6.v5.v4;
  v4.algorithm_requested = p.solve_version >= 4 ? q3.v2.algorithm : VCKSS_ALGORITHM_JLA;
  v4.algorithm_selected = VCKSS_ALGORITHM_JLA;
  v4.deletion_mode = p.deletion_mode;
  v4.nuisance_mode = p.solve_version >= 4 ? q3.v2.nuisance_mode : 0;
  v4.parameters = p.problem.workers + p.problem.firms - 1 + p.controls;
  v4.full_parameters = v4.parameters;
  v4.correction_parameters = v4.parameters;
  VckssEngineDetailedReceiptV5& v5 = d.v6.v5;
  v5.working_fit_complete_residual = v2.full_fit_complete_residual;
  v5.actual_accounting_residual = v2.accounting_residual;
  VckssEngineDetailedReceiptV6& v6 = d.v6;
  v6.engine_requested = p.solve_version >= 4 ? q3.engine : VCKSS_ENGINE_AUTO_OR_UNSPECIFIED;
  v6.engine_selected = p.plan.generic ? VCKSS_ENGINE_GENERIC : VCKSS_ENGINE_COMPRESSED;
  v6.controls_count = p.controls;
  v6.rhs_receipt_schema = p.plan.generic ? 2 : 1;
  if (p.solve_version >= 4) {
    v6.capability_schema = q3.capability_schema;
    v6.capability_profile = q3.capability_profile;
    v6.batch_mode = q3.batch_mode;
    v6.stayers_mode = q3.stayers_mode;
    v6.target_weight_mode = q3.target_weight_mode;
    v6.deletion_unit_source = q3.deletion_unit_source;
    v6.probeorder_supplied = q3.probeorder_supplied;
    v6.wallseconds_supplied = q3.wallseconds_supplied;
    v6.frequency_use = q3.frequency_use;
    v6.physical_limit = q3.physical_limit;
    v6.request_signature = q3.request_signature;
  }
  // execution plan (V5 and V8 solves)
  VckssExecutionPlanReceiptV1& x = d.execution;
  x.struct_size = sizeof(VckssExecutionPlanReceiptV1);
  x.schema_version = 1;
  x.generation = g;
  x.request_signature = v6.request_signature;
  x.resolution.algorithm_schema = 1;
  x.resolution.algorithm_requested = v4.algorithm_requested;
  x.resolution.algorithm_selected = VCKSS_ALGORITHM_JLA;
  x.resolution.engine_schema = 1;
  x.resolution.engine_requested = v6.engine_requested;
  x.resolution.engine_selected = v6.engine_selected;
  x.resolution.resolved_before_rng = 1;
  x.solver.schema_version = 1;
  x.solver.requested_route = o.solver_route;
  x.solver.selected_route = route;
  x.solver.fallback_used = v2.solver_fallback;
  x.solver.full_setup_complete = 1;
  x.solver.fe_setup_complete = 1;
  x.solver.plan_frozen_before_rng = 1;
  x.solver.threads_requested = 1;
  x.solver.threads_used = 1;
  x.solver.planned_rhs = 1 + 3 * uint64_t(o.probes);
  x.solver.full_solver_dimension = v2.solver_dimension;
  x.solver.fe_solver_dimension = p.plan.generic ? p.problem.firms : p.problem.firms - 1;
  x.batch.schema_version = 1;
  x.batch.deterministic = 1;
  x.batch.leverage.requested_width = o.leverage_batch_width;
  x.batch.leverage.selected_width = o.block_columns ? uint64_t(o.block_columns) : 64;
  x.batch.target.requested_width = o.target_batch_width;
  x.batch.target.selected_width = x.batch.leverage.selected_width;
  x.wall.schema_version = 1;
  x.counter.schema_version = 1;
  x.counter.rng_contract = VCKSS_RNG_COUNTER_V1;
  x.counter.completed = 1;
  x.memory.schema_version = 1;
  x.memory.hard_limit_bytes = p.memory_limit;
  x.memory.prepared_persistent_bytes = st.h2d_bytes;
  return d;
}

template <class T>
void write_receipt_prefix(const VckssEngineDetailedReceiptV7& d, T* out) {
  static_assert(sizeof(T) <= sizeof(VckssEngineDetailedReceiptV7), "receipt prefix");
  std::memcpy(out, &d, sizeof(T));
}

// The solved result a detailed receipt describes, with the quantities the
// solve leaves on the device (weighted RSS, the units' residual shares) read.
const SolveResult& solved_result(uint64_t g, Prepared*& p, const char* phase) {
  p = &reg().require(g, phase);
  if (reg().state != State::Solved || !reg().result) fail(STALE_CONTEXT, phase, "generation has no solved result");
  SolveResult& res = *reg().result;
  if (p->device && !res.weighted_rss_ready) {
    res.weighted_rss = device_weighted_rss(*p->device, p->problem);
    res.weighted_rss_ready = true;
  }
  if (p->device && !p->plan.generic) device_unit_detail(*p->device, res);
  if (!p->checksum_ready) {
    p->topology_checksum = compressed_topology_checksum(p->problem);
    p->checksum_ready = true;
  }
  return res;
}
}  // namespace

namespace fevcb {
// Reference entry points outside the replaced solve path (abi_unsupported.cpp).
int32_t unsupported_entry(const char* name) {
  return status([&] {
    fail(UNSUPPORTED_FEATURE, "engine_ffi",
         std::string(name) + " is outside the B200 engine's solve path and is not provided");
  });
}
}  // namespace fevcb

extern "C" {

uint32_t vckss_rust_abi_version(void) { return VCKSS_RUST_ABI_VERSION_V1; }

const char* vckss_rust_backend_version(void) { return "fevc-b200 0.1.0 (sm_100a)"; }

const char* vckss_rust_capabilities_json(void) {
  return "{\"backend\":\"fevc-b200\",\"abi\":1,\"device\":\"sm_100a\",\"rng\":\"VCKSS-COUNTER-V1\","
         "\"algorithms\":[\"jla\",\"exact\"],\"engines\":[\"compressed\",\"generic\"],"
         "\"deletion\":[\"match\",\"observation\"],\"controls\":8,\"centering\":[\"none\",\"mean\"],"
         "\"solver\":\"blocked-pcg-hybrid-laplacian\","
         "\"preconditioners\":[\"jacobi\",\"cmg\",\"learned\",\"polynomial\"],\"precision\":[\"f64\",\"mixed\",\"autotuned\"]}";
}

const char* vckss_rust_last_error(void) { return g_last_error.c_str(); }
const char* vckss_rust_engine_last_error(void) { return g_last_error.c_str(); }

int32_t vckss_rust_selftest(void) {
  return status([] {
    // frozen Counter-V1 vectors (reference rust/crates/vckss-core/src/rng.rs:366-419)
    uint64_t b[4];
    philox_block(philox_key(123456789), 99, 17, 3, TAG_LEVERAGE, b);
    if (b[0] != 0x9f4b6ea90b26b57dull || b[1] != 0x529b58b961489b78ull || b[2] != 0x9d84fab11898a6a0ull ||
        b[3] != 0x469459830d836d27ull)
      fail(RNG_CONTRACT_FAILED, "selftest", "Philox block vector mismatch");
    int64_t s[4];
    rademacher_block_sums(philox_key(123), TAG_LEVERAGE, 1, 7, 65, s);
    if (s[1] != -5) fail(RNG_CONTRACT_FAILED, "selftest", "Rademacher sum vector mismatch");
  });
}

int32_t vckss_rust_backend_capabilities_v1(VckssBackendCapabilitiesV1* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssBackendCapabilitiesV1>(out, cap, "capabilities");
    VckssBackendCapabilitiesV1 c{};
    c.struct_size = sizeof(c);
    c.abi_version = 1;
    c.core_ready_flags = (1ull << 0) | (1ull << 2) | (1ull << 3) | (1ull << 5) | (1ull << 6) | (1ull << 7);
    c.support_flags = (1ull << 1) | (1ull << 2) | (1ull << 5) | (1ull << 6);
    c.deterministic_parallelism = 1;
    std::memcpy(out, &c, sizeof(c));
  });
}

int32_t vckss_rust_engine_default_solve_request_v1(VckssEngineSolveRequestV1* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssEngineSolveRequestV1>(out, cap, "engine default solve request");
    VckssEngineSolveRequestV1 q{};
    q.abi_version = 1;
    q.struct_size = sizeof(q);
    q.seed = 8675309;
    q.probes = 200;
    q.leverage_batch_width = 8;
    q.target_batch_width = 8;
    q.deletion_mode = VCKSS_DELETION_MATCH;
    q.rng_contract = VCKSS_RNG_COUNTER_V1;
    q.solver_route = VCKSS_ROUTE_AUTO;
    q.allow_automatic_cmg_setup_fallback = 1;
    q.exact_dimension_limit = 500;
    q.cmg_minimum_dimension = 2000;
    q.pcg_tolerance = 1e-10;
    q.maximum_iterations = 10000;
    q.residual_replacement_interval = 100;
    q.rank_tolerance = 1e-10;
    q.block_tolerance = 1e-10;
    // CMG fields carry the reference defaults (vckss-core/src/cmg/hierarchy.rs:38-55)
    q.cmg_terminal_vertices = 128;
    q.cmg_dense_vertex_cap = 6144;
    q.cmg_maximum_levels = 96;
    q.cmg_aggregate_cap = 8;
    q.cmg_minimum_reduction = 0.20;
    q.cmg_jacobi_weight = 2.0 / 3.0;
    q.cmg_pre_sweeps = 1;
    q.cmg_post_sweeps = 1;
    q.cmg_maximum_edge_complexity = 12.0;
    q.cmg_maximum_vertex_complexity = 5.0;
    q.cmg_memory_limit_bytes = 2ull << 30;
    std::memcpy(out, &q, sizeof(q));
  });
}

int32_t vckss_rust_engine_default_solve_request_v2(VckssEngineSolveRequestV2* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssEngineSolveRequestV2>(out, cap, "V2 engine default solve request");
    VckssEngineSolveRequestV2 q{};
    if (vckss_rust_engine_default_solve_request_v1(&q.v1, sizeof(q.v1)) != OK) fail(PANIC, "defaults", "V1 defaults");
    q.v1.struct_size = sizeof(q);
    q.algorithm = VCKSS_ALGORITHM_JLA;
    q.nuisance_mode = VCKSS_NUISANCE_JOINT;
    q.exact_estimator_limit = 500;
    q.blocksize_limit = 5000;
    std::memcpy(out, &q, sizeof(q));
  });
}

int32_t vckss_rust_engine_default_solve_request_v3(VckssEngineSolveRequestV3* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssEngineSolveRequestV3>(out, cap, "V3 engine default solve request");
    VckssEngineSolveRequestV3 q{};
    if (vckss_rust_engine_default_solve_request_v2(&q.v2, sizeof(q.v2)) != OK) fail(PANIC, "defaults", "V2 defaults");
    q.v2.v1.struct_size = sizeof(q);
    q.v2.v1.solver_route = VCKSS_ROUTE_DIAGONAL_PCG;
    q.v2.v1.allow_automatic_cmg_setup_fallback = 0;
    q.engine = 2;
    q.batch_mode = 1;
    q.stayers_mode = 1;
    q.target_weight_mode = 0;
    q.deletion_unit_source = 1;
    q.capability_schema = 2;
    q.capability_profile = 3;
    q.frequency_use = 0;
    q.physical_limit = 50000000;
    std::memcpy(out, &q, sizeof(q));
  });
}

int32_t vckss_rust_engine_default_solve_request_v4(VckssEngineSolveRequestV4* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssEngineSolveRequestV4>(out, cap, "V4 engine default solve request");
    VckssEngineSolveRequestV4 q{};
    if (vckss_rust_engine_default_solve_request_v3(&q.v3, sizeof(q.v3)) != OK) fail(PANIC, "defaults", "V3 defaults");
    q.v3.v2.v1.struct_size = sizeof(q);
    q.v3.v2.v1.solver_route = VCKSS_ROUTE_AUTO;
    q.v3.v2.v1.leverage_batch_width = 0;
    q.v3.v2.v1.target_batch_width = 0;
    q.v3.v2.algorithm = VCKSS_ALGORITHM_AUTO;
    q.v3.engine = 0;
    q.v3.batch_mode = 0;
    q.v3.capability_schema = 3;
    q.v3.capability_profile = 4;
    std::memcpy(out, &q, sizeof(q));
  });
}

int32_t vckss_rust_engine_default_solve_request_v5(VckssEngineSolveRequestV5* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssEngineSolveRequestV5>(out, cap, "V5 engine default solve request");
    VckssEngineSolveRequestV5 q{};
    if (vckss_rust_engine_default_solve_request_v4(&q.v4, sizeof(q.v4)) != OK) fail(PANIC, "defaults", "V4 defaults");
    q.v4.v3.v2.v1.struct_size = sizeof(q);
    q.threads = 1;
    std::memcpy(out, &q, sizeof(q));
  });
}

int32_t vckss_rust_engine_default_solve_request_interrupt_v1(VckssEngineSolveRequestInterruptV1* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssEngineSolveRequestInterruptV1>(out, cap, "interrupt solve request");
    VckssEngineSolveRequestInterruptV1 q{};
    if (vckss_rust_engine_default_solve_request_v1(&q.options, sizeof(q.options)) != OK) fail(PANIC, "defaults", "V1");
    q.options.struct_size = sizeof(q);
    std::memcpy(out, &q, sizeof(q));
  });
}

int32_t vckss_rust_engine_default_solve_request_interrupt_v5(VckssEngineSolveRequestInterruptV5* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssEngineSolveRequestInterruptV5>(out, cap, "interrupt V5 solve request");
    VckssEngineSolveRequestInterruptV5 q{};
    if (vckss_rust_engine_default_solve_request_v5(&q.options, sizeof(q.options)) != OK) fail(PANIC, "defaults", "V5");
    q.options.v4.v3.v2.v1.struct_size = sizeof(q);
    std::memcpy(out, &q, sizeof(q));
  });
}

int32_t vckss_rust_engine_default_prepare_request_v3(VckssEnginePrepareRequestV3* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssEnginePrepareRequestV3>(out, cap, "V3 engine default prepare request");
    VckssEnginePrepareRequestV3 q{};
    q.v2.abi_version = 1;
    q.v2.struct_size = sizeof(q);
    q.deletion_mode = VCKSS_DELETION_MATCH;
    std::memcpy(out, &q, sizeof(q));
  });
}

int32_t vckss_rust_engine_default_prepare_request_interrupt_v1(VckssEnginePrepareRequestInterruptV1* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssEnginePrepareRequestInterruptV1>(out, cap, "interrupt prepare request");
    VckssEnginePrepareRequestInterruptV1 q{};
    q.options.abi_version = 1;
    q.options.struct_size = sizeof(q);
    std::memcpy(out, &q, sizeof(q));
  });
}

int32_t vckss_rust_engine_default_prepare_request_interrupt_v2(VckssEnginePrepareRequestInterruptV2* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssEnginePrepareRequestInterruptV2>(out, cap, "V2 interrupt prepare request");
    VckssEnginePrepareRequestInterruptV2 q{};
    q.options.v2.abi_version = 1;
    q.options.v2.struct_size = sizeof(q);
    q.options.deletion_mode = VCKSS_DELETION_MATCH;
    std::memcpy(out, &q, sizeof(q));
  });
}

int32_t vckss_rust_engine_default_prepare_request_interrupt_v3(VckssEnginePrepareRequestInterruptV3* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssEnginePrepareRequestInterruptV3>(out, cap, "V3 interrupt prepare request");
    VckssEnginePrepareRequestInterruptV3 q{};
    q.options.v3.v2.abi_version = 1;
    q.options.v3.v2.struct_size = sizeof(q);
    q.options.v3.deletion_mode = VCKSS_DELETION_MATCH;
    std::memcpy(out, &q, sizeof(q));
  });
}

int32_t vckss_rust_engine_prepare_v1(const VckssEnginePrepareRequestV1* request, const VckssEngineColumnsV1* columns,
                                     uint64_t* out, uint32_t cap) {
  return status([&] {
    auto q = read_struct(request, "engine prepare request");
    auto c = read_struct(columns, "engine column descriptor", 0);
    require_abi(q.abi_version);
    if (q.reserved != 0) fail(ABI_MISMATCH, "engine_ffi", "reserved preparation fields must be zero");
    PrepareArgs a{q.rows, q.cleanup_abandoned};
    a.v1 = &c;
    prepare_common(a, out, cap);
  });
}

int32_t vckss_rust_engine_prepare_v2(const VckssEnginePrepareRequestV2* request, const VckssEngineColumnsV1* columns,
                                     uint64_t* out, uint32_t cap) {
  return status([&] {
    auto q = read_struct(request, "V2 engine prepare request");
    auto c = read_struct(columns, "engine column descriptor", 0);
    require_abi(q.abi_version);
    if (q.reserved != 0) fail(ABI_MISMATCH, "engine_ffi", "reserved preparation fields must be zero");
    PrepareArgs a{q.rows, q.cleanup_abandoned, true, q.memory_limit_bytes, q.caller_copy_bytes};
    a.v1 = &c;
    prepare_common(a, out, cap);
  });
}

static void prepare_v3_impl(const VckssEnginePrepareRequestV3& q, const VckssEngineColumnsV2& c, const double* probe,
                            uint32_t implicit, const Interrupt& intr, uint64_t* out, uint32_t cap) {
  require_abi(q.v2.abi_version);
  if (q.v2.reserved != 0 || q.reserved_2 != 0 || c.reserved_2 != 0)
    fail(ABI_MISMATCH, "engine_ffi", "reserved V2 column fields must be zero");
  if (q.controls_count != c.controls_count)
    fail(INVALID_INPUT, "engine_prepare", "request and descriptor control counts disagree");
  PrepareArgs a{q.v2.rows, q.v2.cleanup_abandoned, true, q.v2.memory_limit_bytes, q.v2.caller_copy_bytes};
  a.deletion_mode = q.deletion_mode;
  a.implicit_match = implicit;
  a.v1 = &c.v1;
  a.controls = c.controls;
  a.controls_count = c.controls_count;
  a.probe_order = probe;
  a.interrupt = intr;
  prepare_common(a, out, cap);
}

int32_t vckss_rust_engine_prepare_v3(const VckssEnginePrepareRequestV3* request, const VckssEngineColumnsV2* columns,
                                     uint64_t* out, uint32_t cap) {
  return status([&] {
    auto q = read_struct(request, "V3 engine prepare request");
    auto c = read_struct(columns, "V2 engine column descriptor", 0);
    prepare_v3_impl(q, c, nullptr, 0, Interrupt{}, out, cap);
  });
}

int32_t vckss_rust_engine_prepare_interrupt_v1(const VckssEnginePrepareRequestInterruptV1* request,
                                               const VckssEngineColumnsV1* columns, uint64_t* out, uint32_t cap) {
  return status([&] {
    auto q = read_struct(request, "interrupt engine prepare request");
    auto c = read_struct(columns, "engine column descriptor", 0);
    require_abi(q.options.abi_version);
    PrepareArgs a{q.options.rows, q.options.cleanup_abandoned, true, q.options.memory_limit_bytes,
                  q.options.caller_copy_bytes};
    a.v1 = &c;
    a.interrupt = Interrupt(q.interrupt_poll, q.interrupt_context, q.checkpoint_interval, q.reserved, "prepare");
    prepare_common(a, out, cap);
  });
}

int32_t vckss_rust_engine_prepare_interrupt_v2(const VckssEnginePrepareRequestInterruptV2* request,
                                               const VckssEngineColumnsV2* columns, uint64_t* out, uint32_t cap) {
  return status([&] {
    auto q = read_struct(request, "V2 interrupt engine prepare request");
    auto c = read_struct(columns, "V2 engine column descriptor", 0);
    prepare_v3_impl(q.options, c, nullptr, 0,
                    Interrupt(q.interrupt_poll, q.interrupt_context, q.checkpoint_interval, q.reserved, "prepare"), out, cap);
  });
}

int32_t vckss_rust_engine_prepare_interrupt_v4(const VckssEnginePrepareRequestInterruptV3* request,
                                               const VckssEngineColumnsV3* columns, uint64_t* out, uint32_t cap) {
  return status([&] {
    auto q = read_struct(request, "V3 interrupt engine prepare request");
    auto c = read_struct(columns, "V3 engine column descriptor", 0);
    if (q.options.reserved_3 != 0 || c.reserved_3 != 0) fail(ABI_MISMATCH, "engine_ffi", "reserved V3 fields must be zero");
    if (q.options.implicit_match > 1) fail(INVALID_INPUT, "engine_prepare", "implicit_match must be zero or one");
    if (c.probeorder_supplied > 1) fail(INVALID_INPUT, "engine_prepare", "probeorder_supplied must be zero or one");
    prepare_v3_impl(q.options.v3, c.v2, c.probeorder_supplied ? c.probe_order : nullptr, q.options.implicit_match,
                    Interrupt(q.interrupt_poll, q.interrupt_context, q.checkpoint_interval, q.reserved, "prepare"), out,
                    cap);
  });
}

int32_t vckss_rust_engine_centering_v1(uint64_t generation, uint32_t mode) {
  return status([&] {
    if (mode > 2) fail(INVALID_INPUT, "centering", "invalid mode");
    if (mode == 2) fail(UNSUPPORTED_FEATURE, "centering", "Corrected centering is not provided by this backend");
    std::lock_guard<std::mutex> l(reg().mu);
    Prepared& p = reg().require(generation, "centering");
    if (reg().state != State::Prepared) fail(STALE_CONTEXT, "centering", "generation is not in the prepared state");
    p.centering = Centering(mode);
  });
}

int32_t vckss_rust_engine_solve_v1(uint64_t generation, const VckssEngineSolveRequestV1* request) {
  return status([&] {
    auto q = read_struct(request, "engine solve request");
    if (q.struct_size < sizeof(q)) fail(ABI_MISMATCH, "engine_ffi", "solve request struct_size is too small");
    solve_common(generation, options_from_v1(q), Interrupt{}, false);
  });
}

int32_t vckss_rust_engine_solve_interrupt_v1(uint64_t generation, const VckssEngineSolveRequestInterruptV1* request) {
  return status([&] {
    auto q = read_struct(request, "interrupt engine solve request");
    solve_common(generation, options_from_v1(q.options),
                 Interrupt(q.interrupt_poll, q.interrupt_context, q.checkpoint_interval, q.reserved, "solve"), false);
  });
}

static SolveOptions options_from_v5(const VckssEngineSolveRequestV5& q) {
  SolveOptions o = options_from_v4(q.v4);
  // Without a supplied tolerance the reference full-CMG route solves probes
  // at 1e-6 (vckss-core/src/full_cmg.rs:29,56-69); the device engine keeps the
  // request's fit tolerance for every right-hand side, which is never looser.
  return o;
}

int32_t vckss_rust_engine_solve_v5(uint64_t generation, const VckssEngineSolveRequestV5* request) {
  return status([&] {
    auto q = read_struct(request, "V5 engine solve request");
    solve_common(generation, options_from_v5(q), Interrupt{}, true, &q.v4, 5);
  });
}

int32_t vckss_rust_engine_solve_interrupt_v5(uint64_t generation, const VckssEngineSolveRequestInterruptV5* request) {
  return status([&] {
    auto q = read_struct(request, "V5 interrupt engine solve request");
    solve_common(generation, options_from_v5(q.options),
                 Interrupt(q.interrupt_poll, q.interrupt_context, q.checkpoint_interval, q.reserved, "solve"), true,
                 &q.options.v4, 5);
  });
}

int32_t vckss_rust_engine_solve_v4(uint64_t generation, const VckssEngineSolveRequestV4* request) {
  return status([&] {
    auto q = read_struct(request, "V4 engine solve request");
    require_abi(q.v3.v2.v1.abi_version);
    solve_common(generation, options_from_v4(q), Interrupt{}, true, &q, 4);
  });
}

int32_t vckss_rust_engine_solve_interrupt_v4(uint64_t generation, const VckssEngineSolveRequestInterruptV4* request) {
  return status([&] {
    auto q = read_struct(request, "V4 interrupt engine solve request");
    require_abi(q.options.v3.v2.v1.abi_version);
    solve_common(generation, options_from_v4(q.options),
                 Interrupt(q.interrupt_poll, q.interrupt_context, q.checkpoint_interval, q.reserved, "solve"), true,
                 &q.options, 4);
  });
}

int32_t vckss_rust_engine_default_solve_request_v8(VckssEngineSolveRequestV8* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssEngineSolveRequestV8>(out, cap, "V8 engine default solve request");
    VckssEngineSolveRequestV8 q{};
    if (vckss_rust_engine_default_solve_request_v4(&q.v7.v6.v4, sizeof(q.v7.v6.v4)) != OK)
      fail(PANIC, "defaults", "V4 defaults");
    auto& v4 = q.v7.v6.v4;
    v4.v3.v2.v1.struct_size = sizeof(q);
    v4.v3.v2.v1.solver_route = VCKSS_ROUTE_DIAGONAL_PCG;
    v4.v3.v2.algorithm = VCKSS_ALGORITHM_JLA;
    v4.v3.engine = VCKSS_ENGINE_GENERIC;
    q.v7.v6.execution_mode = 3;
    q.v7.v6.threads = 1;
    q.resolved_execution_mode = 3;
    std::memcpy(out, &q, sizeof(q));
  });
}

int32_t vckss_rust_engine_default_solve_request_interrupt_v8(VckssEngineSolveRequestInterruptV8* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssEngineSolveRequestInterruptV8>(out, cap, "V8 interrupt default solve request");
    VckssEngineSolveRequestInterruptV8 q{};
    if (vckss_rust_engine_default_solve_request_v8(&q.options, sizeof(q.options)) != OK)
      fail(PANIC, "defaults", "V8 defaults");
    q.options.v7.v6.v4.v3.v2.v1.struct_size = sizeof(q);
    std::memcpy(out, &q, sizeof(q));
  });
}

int32_t vckss_rust_engine_solve_v8(uint64_t generation, const VckssEngineSolveRequestV8* request) {
  return status([&] {
    auto q = read_struct(request, "V8 engine solve request");
    require_abi(q.v7.v6.v4.v3.v2.v1.abi_version);
    solve_common(generation, options_from_v4(q.v7.v6.v4), Interrupt{}, true, &q.v7.v6.v4, 8);
  });
}

int32_t vckss_rust_engine_solve_interrupt_v8(uint64_t generation, const VckssEngineSolveRequestInterruptV8* request) {
  return status([&] {
    auto q = read_struct(request, "V8 interrupt engine solve request");
    require_abi(q.options.v7.v6.v4.v3.v2.v1.abi_version);
    solve_common(generation, options_from_v4(q.options.v7.v6.v4),
                 Interrupt(q.interrupt_poll, q.interrupt_context, q.checkpoint_interval, q.reserved, "solve"), true,
                 &q.options.v7.v6.v4, 8);
  });
}

int32_t vckss_rust_backend_request_capability_v3(const VckssBackendRequestCapabilityRequestV3* request,
                                                 VckssBackendRequestCapabilityReceiptV3* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssBackendRequestCapabilityReceiptV3>(out, cap, "V3 request capability receipt");
    if (!request) fail(INVALID_INPUT, "engine_ffi", "V3 request capability pointer is null");
    VckssBackendRequestCapabilityRequestV3 c;
    std::memcpy(&c, request, sizeof(c));
    require_abi(c.v2.v1.abi_version);
    if (c.v2.v1.struct_size < sizeof(c))
      fail(ABI_MISMATCH, "engine_ffi", "V3 request capability reports a short structure size");
    if (c.v2.v1.reserved != 0 || c.v2.reserved_2 != 0 || c.reserved_3 != 0 || c.reserved_4 != 0)
      fail(ABI_MISMATCH, "engine_ffi", "reserved V3 request capability fields must be zero");
    uint32_t reason = capability_reason(c);
    VckssBackendRequestCapabilityReceiptV3 r{};
    auto& r1 = r.v2.v1;
    r1.struct_size = sizeof(r);
    r1.abi_version = VCKSS_RUST_ABI_VERSION_V1;
    r1.request_schema = c.v2.v1.request_schema;
    r1.supported = reason == VCKSS_REQUEST_REASON_SUPPORTED;
    r1.reason_code = reason;
    r1.profile_code = reason == VCKSS_REQUEST_REASON_SUPPORTED ? VCKSS_REQUEST_PROFILE_PLANNED_V1
                                                               : VCKSS_REQUEST_PROFILE_NONE;
    r1.algorithm = c.v2.v1.algorithm;
    r1.deletion_mode = c.v2.v1.deletion_mode;
    r1.nuisance_mode = c.v2.v1.nuisance_mode;
    r1.solver_route = c.v2.v1.solver_route;
    r1.rng_contract = c.v2.v1.rng_contract;
    r1.controls_count = c.v2.v1.controls_count;
    r1.frequency_use = c.v2.v1.frequency_use;
    r1.request_signature = capability_signature(c);
    r.v2.engine = c.v2.engine;
    r.v2.batch_mode = c.v2.batch_mode;
    r.v2.stayers_mode = c.v2.stayers_mode;
    r.v2.target_weight_mode = c.v2.target_weight_mode;
    r.v2.deletion_unit_source = c.v2.deletion_unit_source;
    r.v2.probeorder_supplied = c.v2.probeorder_supplied;
    r.v2.wallseconds_supplied = c.v2.wallseconds_supplied;
    r.v2.physical_limit = c.v2.physical_limit;
    r.leverage_batch_mode = c.leverage_batch_mode;
    r.target_batch_mode = c.target_batch_mode;
    r.allow_automatic_cmg_setup_fallback = c.allow_automatic_cmg_setup_fallback;
    r.wallseconds = c.wallseconds;
    r.algorithm_resolution_deferred = c.v2.v1.algorithm == VCKSS_ALGORITHM_AUTO;
    r.engine_resolution_deferred = c.v2.v1.algorithm == VCKSS_ALGORITHM_AUTO ||
                                   (c.v2.v1.algorithm == VCKSS_ALGORITHM_JLA &&
                                    c.v2.engine == VCKSS_ENGINE_AUTO_OR_UNSPECIFIED);
    r.route_resolution_deferred = c.v2.v1.algorithm != VCKSS_ALGORITHM_EXACT &&
                                  c.v2.v1.solver_route == VCKSS_ROUTE_AUTO;
    r.leverage_batch_resolution_deferred = c.leverage_batch_mode == VCKSS_BATCH_MODE_AUTO;
    r.target_batch_resolution_deferred = c.target_batch_mode == VCKSS_BATCH_MODE_AUTO;
    r.wall_advisory_only = 1;
    std::memcpy(out, &r, sizeof(r));
  });
}

int32_t vckss_rust_engine_detailed_receipt_v1(uint64_t generation, VckssEngineDetailedReceiptV1* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssEngineDetailedReceiptV1>(out, cap, "engine detailed receipt");
    std::lock_guard<std::mutex> l(reg().mu);
    Prepared* p = nullptr;
    const SolveResult& res = solved_result(generation, p, "engine_detailed_receipt");
    if (p->plan.generic)
      fail(UNSUPPORTED_FEATURE, "engine_detailed_receipt", "the V1 receipt describes a no-control match solve");
    VckssEngineDetailedReceiptV7 d = detailed_receipt(generation, *p, res);
    d.v6.v5.v4.v3.v2.struct_size = sizeof(VckssEngineDetailedReceiptV1);
    write_receipt_prefix(d, out);
  });
}

#define FEVCB_DETAILED_RECEIPT(N, TYPE, LABEL)                                                   \
  int32_t vckss_rust_engine_detailed_receipt_v##N(uint64_t generation, TYPE* out, uint32_t cap) { \
    return status([&] {                                                                          \
      require_capacity<TYPE>(out, cap, LABEL);                                                   \
      std::lock_guard<std::mutex> l(reg().mu);                                                   \
      Prepared* p = nullptr;                                                                     \
      const SolveResult& res = solved_result(generation, p, "engine_detailed_receipt");          \
      write_receipt_prefix(detailed_receipt(generation, *p, res), out);                          \
    });                                                                                          \
  }
FEVCB_DETAILED_RECEIPT(2, VckssEngineDetailedReceiptV2, "V2 engine detailed receipt")
FEVCB_DETAILED_RECEIPT(3, VckssEngineDetailedReceiptV3, "V3 engine detailed receipt")
FEVCB_DETAILED_RECEIPT(4, VckssEngineDetailedReceiptV4, "V4 engine detailed receipt")
FEVCB_DETAILED_RECEIPT(5, VckssEngineDetailedReceiptV5, "V5 engine detailed receipt")
FEVCB_DETAILED_RECEIPT(6, VckssEngineDetailedReceiptV6, "V6 engine detailed receipt")
#undef FEVCB_DETAILED_RECEIPT

int32_t vckss_rust_engine_detailed_receipt_v7(uint64_t generation, VckssEngineDetailedReceiptV7* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssEngineDetailedReceiptV7>(out, cap, "V7 engine detailed receipt");
    std::lock_guard<std::mutex> l(reg().mu);
    Prepared* p = nullptr;
    const SolveResult& res = solved_result(generation, p, "engine_detailed_receipt");
    if (p->solve_version != 5 && p->solve_version != 8)
      fail(UNSUPPORTED_FEATURE, "engine_detailed_receipt",
           "the V7 execution-plan receipt is unavailable for a legacy solve");
    write_receipt_prefix(detailed_receipt(generation, *p, res), out);
  });
}

int32_t vckss_rust_engine_full_cmg_receipt_v1(uint64_t generation, VckssFullCmgReceiptV1* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssFullCmgReceiptV1>(out, cap, "full-CMG receipt");
    std::lock_guard<std::mutex> l(reg().mu);
    Prepared& p = reg().require(generation, "engine_full_cmg_receipt");
    if (reg().state != State::Solved || !reg().result || !p.device)
      fail(STALE_CONTEXT, "engine_full_cmg_receipt", "generation has no solved result");
    const SolveResult& s = *reg().result;
    DeviceStats st = device_stats(*p.device);
    VckssFullCmgReceiptV1 r{};
    r.struct_size = sizeof(r);
    r.schema_version = 1;
    r.generation = generation;
    static const char id[] = "fevc-b200 device engine";
    std::memcpy(r.cmg_source_commit, id, sizeof(id) - 1);
    r.threads_requested = 1;
    r.threads_used = 1;
    r.maximum_concurrency = 1;
    r.vertices = st.vertices;
    r.edges = st.edges;
    r.hierarchy_levels = st.levels;
    r.terminal_vertices = st.terminal_vertices;
    r.fit_effective_tolerance = p.last_options.pcg_tolerance;
    r.probe_effective_tolerance = p.last_options.pcg_tolerance;
    r.fit_initial_inner_tolerance = p.last_options.pcg_tolerance;
    r.probe_initial_inner_tolerance = p.last_options.pcg_tolerance;
    r.rhs_count = s.timings.rhs_columns;
    r.batch_calls = s.timings.pcg_iterations ? s.receipts.size() : 0;
    r.total_iterations = s.timings.column_iterations;
    r.total_operator_applications = s.timings.column_iterations;
    r.total_preconditioner_applications = s.timings.column_iterations + s.timings.rhs_columns;
    r.maximum_reduced_residual = s.max_reduced_residual;
    r.maximum_complete_residual = s.max_complete_residual;
    r.solve_ns = uint64_t(s.timings.total_ms * 1e6);
    r.maximum_batch_rhs = uint64_t(p.last_options.block_columns ? p.last_options.block_columns : 64);
    std::memcpy(out, &r, sizeof(r));
  });
}

int32_t vckss_rust_engine_result_v1(uint64_t generation, VckssEngineResultV1* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssEngineResultV1>(out, cap, "engine result");
    std::lock_guard<std::mutex> l(reg().mu);
    reg().require(generation, "engine_result");
    if (reg().state != State::Solved || !reg().result)
      fail(STALE_CONTEXT, "engine_result", "generation has no solved result");
    const SolveResult& s = *reg().result;
    VckssEngineResultV1 r{};
    r.struct_size = sizeof(r);
    r.generation = generation;
    r.plugin = {s.plugin.worker, s.plugin.firm, s.plugin.covariance, s.plugin.total};
    r.correction = {s.correction.worker, s.correction.firm, s.correction.covariance, s.correction.total};
    r.corrected = {s.corrected.worker, s.corrected.firm, s.corrected.covariance, s.corrected.total};
    r.numerical_mcse = {s.mcse.worker, s.mcse.firm, s.mcse.covariance, s.mcse.total};
    std::memcpy(out, &r, sizeof(r));
  });
}

static VckssEnginePreparationReceiptV4 receipt_v4(uint64_t generation) {
  Prepared& p = reg().require(generation, "engine_receipt");
  const Compressed& c = p.problem;
  VckssEnginePreparationReceiptV4 r{};
  auto& v2 = r.v3.v2;
  v2.generation = generation;
  v2.input_rows = p.input_rows;
  v2.retained_rows = c.rows();
  v2.workers = c.workers;
  v2.firms = c.firms;
  v2.cells = c.cells;
  v2.deletion_units = p.deletion_mode == VCKSS_DELETION_OBSERVATION ? c.physical_total : c.deletion_units;
  v2.target_strata = (p.has_plan && !p.plan.generic) ? p.plan.tgt_cell.size() : c.exact_target_strata;
  v2.memory_limit_bytes = p.memory_limit;
  v2.caller_copy_bytes = p.caller_copy;
  uint64_t resident = c.rows() * (4 * 6 + 8 * 3) + c.cells * (4 * 2 + 8 * 3);
  v2.preparation_peak_forecast_bytes = p.caller_copy + 2 * resident;
  v2.prepared_resident_bytes = resident;
  const GraphReceipt& g = p.graph;
  v2.graph_input_rows = g.input_rows;
  v2.graph_retained_rows = g.retained_rows;
  v2.graph_input_physical_mass = g.input_physical_mass;
  v2.graph_retained_physical_mass = g.retained_physical_mass;
  v2.graph_initial_components = g.initial_components;
  v2.graph_maximum_components = g.maximum_components;
  v2.graph_initial_component_rows = g.initial_component_rows;
  v2.graph_mover_input_rows = g.mover_input_rows;
  v2.graph_initial_deletion_edges = g.initial_deletion_edges;
  v2.graph_retained_deletion_edges = g.retained_deletion_edges;
  v2.graph_insufficient_workers_removed = g.insufficient_workers_removed;
  v2.graph_articulation_workers_removed = g.articulation_workers_removed;
  v2.graph_bridge_units_removed = g.bridge_units_removed;
  v2.graph_bridge_rows_removed = g.bridge_rows_removed;
  v2.graph_degree_iterations = g.degree_iterations;
  v2.graph_articulation_iterations = g.articulation_iterations;
  v2.graph_bridge_iterations = g.bridge_iterations;
  v2.graph_fixed_point_iterations = g.fixed_point_iterations;
  r.v3.target_weight_sum = c.target_total;
  r.controls_count = p.controls;
  r.deletion_mode = p.deletion_mode;
  return r;
}

int32_t vckss_rust_engine_preparation_receipt_v1(uint64_t generation, VckssEnginePreparationReceiptV1* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssEnginePreparationReceiptV1>(out, cap, "preparation receipt");
    std::lock_guard<std::mutex> l(reg().mu);
    auto r4 = receipt_v4(generation);
    VckssEnginePreparationReceiptV1 r{};
    r.struct_size = sizeof(r);
    const auto& v2 = r4.v3.v2;
    r.generation = v2.generation;
    r.input_rows = v2.input_rows;
    r.retained_rows = v2.retained_rows;
    r.workers = v2.workers;
    r.firms = v2.firms;
    r.cells = v2.cells;
    r.deletion_units = v2.deletion_units;
    r.target_strata = v2.target_strata;
    std::memcpy(out, &r, sizeof(r));
  });
}

int32_t vckss_rust_engine_preparation_receipt_v2(uint64_t generation, VckssEnginePreparationReceiptV2* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssEnginePreparationReceiptV2>(out, cap, "V2 preparation receipt");
    std::lock_guard<std::mutex> l(reg().mu);
    auto r = receipt_v4(generation).v3.v2;
    r.struct_size = sizeof(r);
    std::memcpy(out, &r, sizeof(r));
  });
}

int32_t vckss_rust_engine_preparation_receipt_v3(uint64_t generation, VckssEnginePreparationReceiptV3* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssEnginePreparationReceiptV3>(out, cap, "V3 preparation receipt");
    std::lock_guard<std::mutex> l(reg().mu);
    auto r = receipt_v4(generation).v3;
    r.v2.struct_size = sizeof(r);
    std::memcpy(out, &r, sizeof(r));
  });
}

int32_t vckss_rust_engine_preparation_receipt_v4(uint64_t generation, VckssEnginePreparationReceiptV4* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssEnginePreparationReceiptV4>(out, cap, "V4 preparation receipt");
    std::lock_guard<std::mutex> l(reg().mu);
    auto r = receipt_v4(generation);
    r.v3.v2.struct_size = sizeof(r);
    std::memcpy(out, &r, sizeof(r));
  });
}

int32_t vckss_rust_engine_retained_mask_v1(uint64_t generation, uint8_t* out, uint64_t cap) {
  return status([&] {
    std::lock_guard<std::mutex> l(reg().mu);
    Prepared& p = reg().require(generation, "engine_retained");
    if (!out || cap < p.retained.size())
      fail(INVALID_INPUT, "engine_retained",
           "retained-mask capacity " + std::to_string(cap) + " is below required size " + std::to_string(p.retained.size()));
    std::memcpy(out, p.retained.data(), p.retained.size());
  });
}

static void fill_rhs_v1(const RhsReceipt& s, VckssEngineRhsReceiptV1& r, uint32_t route) {
  r.phase = s.phase;
  r.side = s.side;
  r.probe = s.probe;
  r.route = route;
  r.iterations = s.iterations;
  r.zero_rhs = s.zero_rhs;
  r.reserved = 0;
  r.reduced_residual = s.reduced_residual;
  r.complete_residual = s.complete_residual;
}

int32_t vckss_rust_engine_rhs_receipts_v1(uint64_t generation, VckssEngineRhsReceiptV1* out, uint64_t rows) {
  return status([&] {
    std::lock_guard<std::mutex> l(reg().mu);
    Prepared& p = reg().require(generation, "engine_rhs_receipts");
    if (reg().state != State::Solved) fail(STALE_CONTEXT, "engine_rhs_receipts", "generation has no solved result");
    const auto& rc = reg().result->receipts;
    if (!out || rows < rc.size())
      fail(INVALID_INPUT, "engine_rhs_receipts", "RHS receipt capacity is below " + std::to_string(rc.size()));
    uint32_t route = (p.last_options.preconditioner == 1 || p.last_options.preconditioner == 4)
                         ? VCKSS_ROUTE_DIAGONAL_PCG : VCKSS_ROUTE_CMG_PCG;
    for (size_t i = 0; i < rc.size(); ++i) fill_rhs_v1(rc[i], out[i], route);
  });
}

int32_t vckss_rust_engine_rhs_receipts_v2(uint64_t generation, VckssEngineRhsReceiptV2* out, uint64_t rows) {
  return status([&] {
    std::lock_guard<std::mutex> l(reg().mu);
    Prepared& p = reg().require(generation, "engine_rhs_receipts");
    if (reg().state != State::Solved) fail(STALE_CONTEXT, "engine_rhs_receipts", "generation has no solved result");
    const auto& rc = reg().result->receipts;
    if (!out || rows < rc.size())
      fail(INVALID_INPUT, "engine_rhs_receipts", "RHS receipt capacity is below " + std::to_string(rc.size()));
    uint32_t route = (p.last_options.preconditioner == 1 || p.last_options.preconditioner == 4)
                         ? VCKSS_ROUTE_DIAGONAL_PCG : VCKSS_ROUTE_CMG_PCG;
    double gate = std::max(10.0 * p.last_options.pcg_tolerance, 1e-11);
    for (size_t i = 0; i < rc.size(); ++i) {
      VckssEngineRhsReceiptV2 r{};
      fill_rhs_v1(rc[i], r.v1, route);
      r.status = rc[i].zero_rhs ? 1 : 2;
      r.operator_applications = rc[i].iterations + 1;
      r.preconditioner_applications = rc[i].iterations + 1;
      r.full_residual_tolerance = gate;
      // residual space and solver dimension by phase (reference
      // generic_rhs_receipt_value, vckss-plugin/src/ffi_engine.rs:8900-8960):
      // the generic joint fit and (joint nuisance) targets carry the control
      // block; leverage and control projections solve the firm system; the
      // no-control estimator solves the grounded quotient
      const uint64_t F = p.problem.firms, q = p.controls;
      const bool joint = rc[i].phase == 1 || (rc[i].phase == 3 && p.last_request.v3.v2.nuisance_mode == 1);
      r.residual_space = (p.plan.generic && joint) ? VCKSS_RESIDUAL_SPACE_WORKER_FIRM_CONTROL
                                                   : VCKSS_RESIDUAL_SPACE_WORKER_FIRM;
      r.solver_dimension = !p.plan.generic ? F - 1 : (joint ? F + q : F);
      out[i] = r;
    }
  });
}

int32_t vckss_rust_engine_release_v1(uint64_t generation) {
  return status([&] {
    std::lock_guard<std::mutex> l(reg().mu);
    Registry& r = reg();
    if (r.state != State::Empty && r.generation == generation) {
      r.state = State::Empty;
      r.prepared.reset();
      r.result.reset();
      r.last_released = std::max(r.last_released, generation);
      return;
    }
    if (r.state == State::Empty && generation <= r.last_released) return;
    fail(STALE_CONTEXT, "context_release", "generation " + std::to_string(generation) + " is not active");
  });
}

int32_t vckss_rust_engine_clear_abandoned_v1(void) {
  return status([&] {
    std::lock_guard<std::mutex> l(reg().mu);
    clear_abandoned(1);
  });
}

int32_t vckss_rust_engine_snapshot_v1(VckssEngineSnapshotV1* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssEngineSnapshotV1>(out, cap, "engine snapshot");
    std::lock_guard<std::mutex> l(reg().mu);
    VckssEngineSnapshotV1 s{};
    s.struct_size = sizeof(s);
    s.state = uint32_t(reg().state);
    s.generation = reg().state == State::Empty ? 0 : reg().generation;
    s.last_released_generation = reg().last_released;
    std::memcpy(out, &s, sizeof(s));
  });
}

// ---------------- B200 extensions ----------------

int32_t fevcb_device_count(void) { return device_count(); }

int32_t fevcb_set_stream(void* stream) {
  return status([&] { set_device_stream(stream); });
}

int32_t fevcb_engine_hybrid_check_v1(uint64_t generation, uint32_t* identical) {
  return status([&] {
    if (!identical) fail(INVALID_INPUT, "engine_hybrid_check", "output pointer is null");
    std::lock_guard<std::mutex> l(reg().mu);
    Prepared& p = reg().require(generation, "engine_hybrid_check");
    if (!p.device) fail(STALE_CONTEXT, "engine_hybrid_check", "generation has no device state; solve it first");
    *identical = device_hybrid_matches_host(*p.device, p.problem) ? 1u : 0u;
  });
}

int32_t fevcb_device_cache_trim_v1(uint64_t* freed_bytes, uint64_t* cached_bytes) {
  return status([&] {
    uint64_t freed = device_cache_trim();
    if (freed_bytes) *freed_bytes = freed;
    if (cached_bytes) *cached_bytes = device_cache_bytes();
  });
}

int32_t fevcb_engine_solve_options_v1(uint64_t generation, const FevcbSolveOptionsV1* options) {
  return status([&] {
    auto o = read_struct(options, "device solve options", 0);
    if (o.struct_size != sizeof(FevcbSolveOptionsV1) && o.struct_size != sizeof(FevcbSolveOptionsV2))
      fail(ABI_MISMATCH, "engine_ffi", "device solve options struct_size mismatch");
    FevcbSolveOptionsV2 o2{};
    std::memcpy(&o2, options, o.struct_size);
    if (o.block_columns != 0 && o.block_columns != 2 && o.block_columns != 8 && o.block_columns != 16 &&
        o.block_columns != 32 && o.block_columns != 64)
      fail(INVALID_INPUT, "engine_ffi", "block_columns must be 0, 2, 8, 16, 32 or 64");
    if (o.preconditioner > 4) fail(INVALID_INPUT, "engine_ffi", "preconditioner must be 0, 1, 2, 3 or 4");
    if (o2.precision > 2) fail(INVALID_INPUT, "engine_ffi", "precision must be 0 (double), 1 (mixed) or 2 (autotuned)");
    if (o2.reserved != 0) fail(INVALID_INPUT, "engine_ffi", "reserved fields must be zero");
    std::lock_guard<std::mutex> l(reg().mu);
    Prepared& p = reg().require(generation, "engine_solve_options");
    if (p.device && o.preconditioner != p.device_options.preconditioner) p.device.reset();
    p.device_options = o;
    p.precision = o2.precision;
  });
}

int32_t fevcb_engine_tuning_v1(uint64_t generation, FevcbTuningV1* out, uint32_t cap) {
  return status([&] {
    if (!out || cap < sizeof(FevcbTuningV1)) fail(INVALID_INPUT, "engine_ffi", "tuning output capacity is too small");
    std::lock_guard<std::mutex> l(reg().mu);
    Prepared& p = reg().require(generation, "engine_tuning");
    FevcbTuningV1 t{};
    t.struct_size = sizeof(FevcbTuningV1);
    t.chosen = -1;
    if (p.device) {
      int prec[3], pre[3], cand = 0;
      double ms[3];
      t.chosen = device_tuning(*p.device, prec, pre, ms, &cand);
      t.candidates = uint32_t(cand);
      for (int c = 0; c < 3; ++c) {
        t.precision[c] = uint32_t(prec[c]);
        t.preconditioner[c] = uint32_t(pre[c]);
        t.milliseconds[c] = ms[c];
      }
    }
    *out = t;
  });
}

int32_t fevcb_engine_prepare_timings_v1(uint64_t generation, FevcbPrepareTimingsV1* out, uint32_t cap) {
  return status([&] {
    if (!out || cap < sizeof(FevcbPrepareTimingsV1))
      fail(INVALID_INPUT, "engine_ffi", "prepare timings output capacity is too small");
    std::lock_guard<std::mutex> l(reg().mu);
    Prepared& p = reg().require(generation, "engine_prepare_timings");
    FevcbPrepareTimingsV1 t{};
    t.struct_size = sizeof(FevcbPrepareTimingsV1);
    t.threads = std::max(1u, std::thread::hardware_concurrency());
    t.ingest_ms = p.prepare_ms[0];
    t.canonical_ms = p.prepare_ms[1];
    t.graph_ms = p.prepare_ms[2];
    t.compression_ms = p.prepare_ms[3];
    t.plan_ms = p.prepare_ms[4];
    t.total_ms = t.ingest_ms + t.canonical_ms + t.graph_ms + t.compression_ms + t.plan_ms;
    *out = t;
  });
}

int32_t fevcb_engine_setup_timings_v1(uint64_t generation, FevcbSetupTimingsV1* out, uint32_t cap) {
  return status([&] {
    require_capacity<FevcbSetupTimingsV1>(out, cap, "setup timings");
    std::lock_guard<std::mutex> l(reg().mu);
    Prepared& p = reg().require(generation, "engine_setup_timings");
    if (!p.device) fail(STALE_CONTEXT, "engine_setup_timings", "the generation has no device engine yet");
    const DeviceStats st = device_stats(*p.device);
    FevcbSetupTimingsV1 t{};
    t.struct_size = sizeof(t);
    t.builders = uint32_t(st.builders);
    for (int i = 0; i < 16; ++i) t.builder_ms[i] = st.builder_ms[i];
    t.builders_span_ms = st.builders_span_ms;
    t.device_units_ms = st.device_units_ms;
    t.hybrid_ms = st.hybrid_ms;
    t.preconditioner_ms = st.preconditioner_ms;
    t.total_ms = st.setup_ms;
    *out = t;
  });
}

int32_t fevcb_engine_exact_limit_v1(uint64_t generation, uint64_t ceiling) {
  return status([&] {
    if (ceiling > 1000000) fail(INVALID_INPUT, "engine_ffi", "exact ceiling must lie in [0, 1000000]");
    std::lock_guard<std::mutex> l(reg().mu);
    Prepared& p = reg().require(generation, "engine_exact_limit");
    p.exact_ceiling = ceiling;
  });
}

int32_t fevcb_engine_timings_v1(uint64_t generation, FevcbSolveTimingsV1* out, uint32_t cap) {
  return status([&] {
    require_capacity<FevcbSolveTimingsV1>(out, cap, "device timings");
    std::lock_guard<std::mutex> l(reg().mu);
    Prepared& p = reg().require(generation, "engine_timings");
    if (reg().state != State::Solved) fail(STALE_CONTEXT, "engine_timings", "generation has no solved result");
    const SolveTimings& t = reg().result->timings;
    FevcbSolveTimingsV1 r{};
    r.struct_size = sizeof(r);
    r.total_ms = t.total_ms;
    r.fit_ms = t.fit_ms;
    r.leverage_ms = t.leverage_ms;
    r.target_ms = t.target_ms;
    r.block_iterations = t.pcg_iterations;
    r.column_iterations = t.column_iterations;
    r.rhs_columns = t.rhs_columns;
    r.kernel_launches = t.kernel_launches;
    r.fallbacks = uint32_t(t.fallbacks);
    if (p.device) {
      DeviceStats s = device_stats(*p.device);
      r.setup_ms = s.setup_ms;
      r.h2d_bytes = s.h2d_bytes;
      r.vertices = s.vertices;
      r.edges = s.edges;
      r.kept_workers = s.kept_workers;
      r.levels = s.levels;
    }
    std::memcpy(out, &r, sizeof(r));
  });
}

int32_t fevcb_engine_resolve_v1(uint64_t generation) {
  return status([&] {
    Registry& r = reg();
    std::lock_guard<std::mutex> l(r.mu);
    Prepared& p = r.require(generation, "engine_resolve");
    if (r.state != State::Solved || !p.solved_once || !p.device)
      fail(STALE_CONTEXT, "engine_resolve", "generation has no solved result to repeat");
    SolveOptions o = p.last_options;
    o.block_columns = int(p.device_options.block_columns);
    o.precision = int(p.precision);
    auto res = std::make_unique<SolveResult>(device_solve(*p.device, p.problem, p.plan, o, false));
    r.result = std::move(res);
  });
}

// Independent probe sets in one call: set 0 is a V5 solve with its seed and
// probe count (its result becomes the generation's result), every later set
// runs the leverage and target phases with its own seed and probes on the
// same device generation, keeping set 0's fit and the autotuned form.
int32_t fevcb_engine_solve_sets_v1(uint64_t generation, const VckssEngineSolveRequestV5* request,
                                   const FevcbProbeSetV1* sets, uint32_t count, FevcbProbeSetResultV1* results,
                                   uint32_t results_capacity_bytes) {
  return status([&] {
    auto q = read_struct(request, "V5 engine solve request");
    if (count == 0 || !sets) fail(INVALID_INPUT, "probe_sets", "at least one probe set is required");
    if (count > 4096) fail(RESOURCE_LIMIT, "probe_sets", "at most 4096 probe sets per call");
    if (!results || uint64_t(results_capacity_bytes) < uint64_t(count) * sizeof(FevcbProbeSetResultV1))
      fail(ABI_MISMATCH, "engine_ffi", "probe-set results destination is null or short");
    std::vector<FevcbProbeSetV1> set(sets, sets + count);
    for (const auto& st : set) {
      if (st.reserved != 0) fail(ABI_MISMATCH, "engine_ffi", "reserved probe-set fields must be zero");
      if (st.probes < 2) fail(INVALID_INPUT, "jla_validate", "JLA probe count must be at least two");
    }
    const SolveOptions base = options_from_v5(q);
    if (base.algorithm == 1) fail(UNSUPPORTED_FEATURE, "probe_sets", "probe sets need the JLA algorithm");
    auto put = [&](uint32_t i, const SolveResult& res) {
      FevcbProbeSetResultV1 v{};
      v.plugin = {res.plugin.worker, res.plugin.firm, res.plugin.covariance, res.plugin.total};
      v.correction = {res.correction.worker, res.correction.firm, res.correction.covariance, res.correction.total};
      v.corrected = {res.corrected.worker, res.corrected.firm, res.corrected.covariance, res.corrected.total};
      v.numerical_mcse = {res.mcse.worker, res.mcse.firm, res.mcse.covariance, res.mcse.total};
      std::memcpy(results + i, &v, sizeof(v));
    };
    SolveOptions first = base;
    first.seed = set[0].seed;
    first.probes = set[0].probes;
    solve_common(generation, first, Interrupt{}, true, &q.v4, 5);
    Registry& r = reg();
    std::lock_guard<std::mutex> l(r.mu);
    Prepared& p = r.require(generation, "probe_sets");
    if (p.projection)
      fail(UNSUPPORTED_FEATURE, "probe_sets", "probe sets do not carry a projection attachment");
    put(0, *r.result);
    for (uint32_t i = 1; i < count; ++i) {
      SolveOptions o = p.last_options;
      o.seed = set[i].seed;
      o.probes = set[i].probes;
      o.reuse_fit = true;
      SolveResult res = device_solve(*p.device, p.problem, p.plan, o, false);
      put(i, res);
    }
  });
}

int32_t fevcb_engine_unit_detail_v1(uint64_t generation, uint64_t units, double* projection_share,
                                    double* residual_share, double* finite_bias, double* finite_variance,
                                    double* residual_mass, double* deleted_mass, uint64_t cells, double* fitted_cell,
                                    double* cell_correction_weight, uint64_t probes, double* target_draws4) {
  return status([&] {
    std::lock_guard<std::mutex> l(reg().mu);
    Prepared& p = reg().require(generation, "engine_unit_detail");
    if (reg().state != State::Solved) fail(STALE_CONTEXT, "engine_unit_detail", "generation has no solved result");
    if (p.device && reg().result->unit_projection_share.empty()) device_unit_detail(*p.device, *reg().result);
    const SolveResult& s = *reg().result;
    if (s.unit_projection_share.empty()) fail(STALE_CONTEXT, "engine_unit_detail", "unit detail was not retained");
    if (units != s.unit_projection_share.size() || cells != s.fitted_cell.size() || probes != s.target_draws.size())
      fail(INVALID_INPUT, "engine_unit_detail", "detail dimensions differ from the solved generation");
    auto put = [&](double* dst, const std::vector<double>& v) {
      if (dst) std::memcpy(dst, v.data(), v.size() * sizeof(double));
    };
    put(projection_share, s.unit_projection_share);
    put(residual_share, s.unit_residual_share);
    put(finite_bias, s.unit_finite_bias);
    put(finite_variance, s.unit_finite_variance);
    put(residual_mass, s.unit_residual_mass);
    put(deleted_mass, s.unit_deleted_mass);
    put(fitted_cell, s.fitted_cell);
    put(cell_correction_weight, s.cell_correction_weight);
    if (target_draws4)
      for (size_t i = 0; i < s.target_draws.size(); ++i) {
        target_draws4[4 * i + 0] = s.target_draws[i].worker;
        target_draws4[4 * i + 1] = s.target_draws[i].firm;
        target_draws4[4 * i + 2] = s.target_draws[i].covariance;
        target_draws4[4 * i + 3] = s.target_draws[i].total;
      }
  });
}

int32_t fevcb_engine_problem_view_v1(uint64_t generation, FevcbProblemViewV1* out, uint32_t cap) {
  return status([&] {
    require_capacity<FevcbProblemViewV1>(out, cap, "problem view");
    std::lock_guard<std::mutex> l(reg().mu);
    Prepared& p = reg().require(generation, "engine_problem_view");
    if (!p.has_plan) fail(UNSUPPORTED_FEATURE, "engine_problem_view", "no compressed JLA plan was prepared");
    const Compressed& c = p.problem;
    const JlaPlan& j = p.plan;
    FevcbProblemViewV1 v{};
    v.struct_size = sizeof(v);
    v.rows = c.rows();
    v.workers = c.workers;
    v.firms = c.firms;
    v.cells = c.cells;
    v.units = j.del_cell.size();
    v.strata = j.tgt_cell.size();
    v.physical_total = c.physical_total;
    v.target_total = c.target_total;
    v.row_worker = c.row_worker.data();
    v.row_firm = c.row_firm.data();
    v.row_cell = c.row_cell.data();
    v.row_outcome = c.outcome.data();
    v.row_target = c.target.data();
    v.row_frequency = c.frequency.data();
    v.cell_worker = c.cell_worker.data();
    v.cell_firm = c.cell_firm.data();
    v.cell_weight = c.cell_weight.data();
    v.cell_outcome_sum = c.cell_outcome_sum.data();
    v.cell_target_sum = c.cell_target_sum.data();
    v.unit_cell = j.del_cell.data();
    v.unit_count = j.del_count.data();
    v.unit_rank = j.del_rank.data();
    v.unit_outcome_sum = j.del_outcome_sum.data();
    v.stratum_cell = j.tgt_cell.data();
    v.stratum_per_copy = j.tgt_per_copy.data();
    v.stratum_count = j.tgt_count.data();
    v.stratum_rank = j.tgt_rank.data();
    v.controls = c.controls.size();
    if (!c.controls.empty() && p.control_values.empty())
      for (auto& col : c.controls) p.control_values.insert(p.control_values.end(), col.begin(), col.end());
    v.control_values = p.control_values.empty() ? nullptr : p.control_values.data();
    v.group_ptr = j.generic ? j.group_ptr.data() : nullptr;
    v.group_rows = j.generic ? j.group_rows.data() : nullptr;
    v.row_rank = j.generic ? j.row_rank.data() : nullptr;
    v.row_copy_offset = j.observation ? j.row_copy_offset.data() : nullptr;
    v.deletion_mode = p.deletion_mode;
    std::memcpy(out, &v, sizeof(v));
  });
}

int32_t fevcb_engine_cmg_summary_v1(uint64_t generation, uint32_t eliminate_max_degree, FevcbCmgSummaryV1* out,
                                    uint32_t cap) {
  return status([&] {
    require_capacity<FevcbCmgSummaryV1>(out, cap, "CMG summary");
    std::lock_guard<std::mutex> l(reg().mu);
    Prepared& p = reg().require(generation, "engine_cmg_summary");
    uint32_t degree = eliminate_max_degree ? eliminate_max_degree : ELIMINATE_MAX_DEGREE;
    std::vector<uint32_t> kw, Lptr, Lcol;
    std::vector<int32_t> ki;
    std::vector<double> cs, wd, Lval, Ld;
    build_hybrid(p.problem, degree, kw, ki, cs, wd, Lptr, Lcol, Lval, Ld);
    MultigridReport rep;
    build_cmg_hierarchy(uint32_t(Ld.size()), Lptr, Lcol, Lval, Ld, MultigridOptions(), rep);
    FevcbCmgSummaryV1 v{};
    v.struct_size = sizeof(v);
    v.eliminate_max_degree = degree;
    v.vertices = Ld.size();
    v.edges = Lcol.size() / 2;
    v.hierarchy_levels = rep.vertices.size();
    v.terminal_vertices = rep.vertices.empty() ? 0 : rep.vertices.back();
    v.terminal_reason = uint32_t(rep.terminal_reason);
    for (size_t i = 0; i < rep.vertices.size() && i < 32; ++i) {
      v.level_vertices[i] = rep.vertices[i];
      v.level_edges[i] = rep.nonzeros[i] / 2;
    }
    for (size_t i = 0; i < rep.repeat.size() && i < 32; ++i) v.level_repeat[i] = uint32_t(rep.repeat[i]);
    std::memcpy(out, &v, sizeof(v));
  });
}

namespace {
// Shared preamble of the shard entries: options, device engine, checks.
SolveOptions shard_options(Prepared& p, const VckssEngineSolveRequestV5* request, uint32_t begin, uint32_t end) {
  auto q = read_struct(request, "V5 engine solve request");
  SolveOptions o = options_from_v5(q);
  if (p.has_plan && p.plan.generic && q.v4.v3.v2.algorithm == VCKSS_ALGORITHM_EXACT)
    fail(UNSUPPORTED_FEATURE, "shard", "the exact estimator is not sharded");
  if (!p.has_plan) fail(UNSUPPORTED_FEATURE, "shard", "no JLA plan was prepared");
  if (o.deletion_mode != p.deletion_mode)
    fail(INVALID_INPUT, "engine_solve", "solve deletion mode differs from the prepared graph mode");
  if (begin % 4 != 0 || begin >= end || end > o.probes)
    fail(INVALID_INPUT, "shard", "probe range must start on a multiple of four and lie inside the probes");
  o.centering = p.centering;
  o.block_columns = int(p.device_options.block_columns);
  o.precision = int(p.precision);
  o.preconditioner = int(p.device_options.preconditioner);
  if (o.preconditioner == 0) o.preconditioner = o.solver_route == VCKSS_ROUTE_CMG_PCG ? 2 : 1;
  if (p.device && p.device_preconditioner != o.preconditioner) p.device.reset();
  if (!p.device) {
    p.device = make_device_engine(p.problem, p.plan, o.preconditioner);
    p.device_preconditioner = o.preconditioner;
  }
  o.probe_begin = begin;
  o.probe_end = end;
  return o;
}
}  // namespace

int32_t fevcb_engine_shard_size_v1(uint64_t generation, uint64_t* count) {
  return status([&] {
    if (!count) fail(INVALID_INPUT, "shard", "null output");
    std::lock_guard<std::mutex> l(reg().mu);
    Prepared& p = reg().require(generation, "engine_shard");
    if (!p.has_plan) fail(UNSUPPORTED_FEATURE, "shard", "no JLA plan was prepared");
    *count = shard_accumulator_count(p.problem, p.plan);
  });
}

int32_t fevcb_engine_shard_leverage_v1(uint64_t generation, const VckssEngineSolveRequestV5* request,
                                       uint32_t begin, uint32_t end, double* acc, uint64_t count) {
  return status([&] {
    std::lock_guard<std::mutex> l(reg().mu);
    Prepared& p = reg().require(generation, "engine_shard");
    if (!acc || count != shard_accumulator_count(p.problem, p.plan))
      fail(INVALID_INPUT, "shard", "accumulator buffer has the wrong length");
    if (p.projection) fail(UNSUPPORTED_FEATURE, "shard", "probe shards do not carry a projection attachment");
    SolveOptions o = shard_options(p, request, begin, end);
    o.shard_phase = 1;
    o.shard_output = acc;  // host or device memory: copied by unified addressing
    SolveResult res = device_solve(*p.device, p.problem, p.plan, o, false);
    {
      SolveTimings& t = p.shard_timings;
      t.kernel_launches += res.timings.kernel_launches;
      t.rhs_columns += res.timings.rhs_columns;
      t.column_iterations += res.timings.column_iterations;
      t.pcg_iterations += res.timings.pcg_iterations;
      t.fit_ms += res.timings.fit_ms;
      t.leverage_ms += res.timings.leverage_ms;
      t.target_ms += res.timings.target_ms;
    }

  });
}

int32_t fevcb_engine_shard_target_v1(uint64_t generation, const VckssEngineSolveRequestV5* request, uint32_t begin,
                                     uint32_t end, const double* acc, uint64_t count, double* draws) {
  return status([&] {
    std::lock_guard<std::mutex> l(reg().mu);
    Prepared& p = reg().require(generation, "engine_shard");
    if (!acc || !draws || count != shard_accumulator_count(p.problem, p.plan))
      fail(INVALID_INPUT, "shard", "accumulator or draw buffer is missing or has the wrong length");
    if (!p.device) fail(STALE_CONTEXT, "shard", "run the leverage shard first");
    SolveOptions o = shard_options(p, request, begin, end);
    o.shard_phase = 2;
    o.shard_input = acc;
    SolveResult res = device_solve(*p.device, p.problem, p.plan, o, false);
    for (uint32_t j = begin; j < end; ++j) {
      const Components& d = res.target_draws[j];
      draws[size_t(j - begin) * 4 + 0] = d.worker;
      draws[size_t(j - begin) * 4 + 1] = d.firm;
      draws[size_t(j - begin) * 4 + 2] = d.covariance;
      draws[size_t(j - begin) * 4 + 3] = d.total;
    }
    p.shard_plugin = res.plugin;
    {
      SolveTimings& t = p.shard_timings;
      t.kernel_launches += res.timings.kernel_launches;
      t.rhs_columns += res.timings.rhs_columns;
      t.column_iterations += res.timings.column_iterations;
      t.pcg_iterations += res.timings.pcg_iterations;
      t.fit_ms += res.timings.fit_ms;
      t.leverage_ms += res.timings.leverage_ms;
      t.target_ms += res.timings.target_ms;
    }
  });
}

int32_t fevcb_engine_shard_finish_v1(uint64_t generation, const VckssEngineSolveRequestV5* request,
                                     const double* draws) {
  return status([&] {
    Registry& r = reg();
    std::lock_guard<std::mutex> l(r.mu);
    Prepared& p = r.require(generation, "engine_shard");
    if (!draws) fail(INVALID_INPUT, "shard", "draws are missing");
    auto q = read_struct(request, "V5 engine solve request");
    SolveOptions o = options_from_v5(q);
    if (!p.device) fail(STALE_CONTEXT, "shard", "no shard of this generation has run");
    auto res = std::make_unique<SolveResult>();
    res->plugin = p.shard_plugin;
    res->target_draws.resize(o.probes);
    for (uint32_t j = 0; j < o.probes; ++j) {
      const double* d = draws + size_t(j) * 4;
      if (!(std::isfinite(d[0]) && std::isfinite(d[1]) && std::isfinite(d[2]) && std::isfinite(d[3])))
        fail(CORRECTION_NONFINITE, "jla_target", "a target draw is nonfinite");
      res->target_draws[j] = Components{d[0], d[1], d[2], d[3]};
    }
    finish_draws(*res, o.probes);
    res->timings = p.shard_timings;
    res->timings.total_ms = res->timings.fit_ms + res->timings.leverage_ms + res->timings.target_ms;
    p.shard_timings = SolveTimings();
    o.centering = p.centering;
    p.last_options = o;
    r.result = std::move(res);
    r.state = State::Solved;
  });
}

namespace {
std::mutex g_learned_mu;
std::map<uint64_t, std::unique_ptr<GnnTrainer>> g_trainers;
std::map<uint64_t, GnnTrainer::Dump> g_dumps;
uint64_t g_next_trainer = 1;

GnnTrainer& trainer(uint64_t h) {
  auto it = g_trainers.find(h);
  if (it == g_trainers.end()) fail(STALE_CONTEXT, "learned_train", "unknown trainer handle");
  return *it->second;
}

void require_count(uint64_t count) {
  if (count != gnn_param_count())
    fail(INVALID_INPUT, "learned", "parameter count must be " + std::to_string(gnn_param_count()));
}
}  // namespace

int32_t fevcb_learned_param_count_v1(uint64_t* count) {
  return status([&] {
    if (!count) fail(INVALID_INPUT, "learned", "null output");
    *count = gnn_param_count();
  });
}

int32_t fevcb_learned_initial_params_v1(uint64_t seed, float* params, uint64_t count) {
  return status([&] {
    if (!params) fail(INVALID_INPUT, "learned", "null output");
    require_count(count);
    auto p = gnn_initial_params(seed);
    std::copy(p.begin(), p.end(), params);
  });
}

int32_t fevcb_learned_install_v1(const float* params, uint64_t count) {
  return status([&] {
    if (!params) fail(INVALID_INPUT, "learned", "null parameters");
    require_count(count);
    std::vector<float> p(params, params + count);
    for (float x : p)
      if (!std::isfinite(x)) fail(INVALID_INPUT, "learned", "parameters must be finite");
    set_learned_params(std::move(p));
  });
}

int32_t fevcb_learned_trainer_create_v1(uint64_t seed, uint64_t* handle) {
  return status([&] {
    if (!handle) fail(INVALID_INPUT, "learned_train", "null handle output");
    if (device_count() < 1) fail(UNSUPPORTED_FEATURE, "device", "no CUDA device is visible; training runs on a GPU");
    std::lock_guard<std::mutex> l(g_learned_mu);
    uint64_t h = g_next_trainer++;
    g_trainers[h] = make_gnn_trainer(seed);
    *handle = h;
  });
}

int32_t fevcb_learned_trainer_destroy_v1(uint64_t handle) {
  return status([&] {
    std::lock_guard<std::mutex> l(g_learned_mu);
    trainer(handle);
    g_trainers.erase(handle);
    g_dumps.erase(handle);
  });
}

int32_t fevcb_learned_trainer_add_panel_v1(uint64_t handle, uint64_t generation, uint32_t columns, uint64_t seed) {
  return status([&] {
    std::vector<uint32_t> kw, Lptr, Lcol;
    std::vector<int32_t> ki;
    std::vector<double> cs, wd, Lval, Ld;
    {
      std::lock_guard<std::mutex> l(reg().mu);
      Prepared& p = reg().require(generation, "learned_add_panel");
      build_hybrid(p.problem, ELIMINATE_MAX_DEGREE, kw, ki, cs, wd, Lptr, Lcol, Lval, Ld);
    }
    std::lock_guard<std::mutex> l(g_learned_mu);
    trainer(handle).add_graph(uint32_t(Ld.size()), Lptr, Lcol, Lval, Ld, int(columns), seed);
  });
}

int32_t fevcb_learned_trainer_train_v1(uint64_t handle, uint32_t steps, double lr, double* losses) {
  return status([&] {
    if (!(lr > 0.0 && lr < 1.0)) fail(INVALID_INPUT, "learned_train", "learning rate must lie in (0, 1)");
    std::lock_guard<std::mutex> l(g_learned_mu);
    auto out = trainer(handle).train(int(steps), lr);
    if (losses) std::copy(out.begin(), out.end(), losses);
  });
}

int32_t fevcb_learned_trainer_gradient_v1(uint64_t handle, uint32_t graph, double* loss, float* gradient,
                                          uint64_t count) {
  return status([&] {
    if (!loss || !gradient) fail(INVALID_INPUT, "learned_train", "null output");
    require_count(count);
    std::lock_guard<std::mutex> l(g_learned_mu);
    GnnTrainer& t = trainer(handle);
    if (graph >= uint32_t(t.graphs())) fail(INVALID_INPUT, "learned_train", "graph index out of range");
    std::vector<float> g;
    *loss = t.gradient(int(graph), g);
    std::copy(g.begin(), g.end(), gradient);
  });
}

int32_t fevcb_learned_trainer_params_v1(uint64_t handle, float* params, uint64_t count) {
  return status([&] {
    if (!params) fail(INVALID_INPUT, "learned_train", "null output");
    require_count(count);
    std::lock_guard<std::mutex> l(g_learned_mu);
    auto& p = trainer(handle).params();
    std::copy(p.begin(), p.end(), params);
  });
}

int32_t fevcb_learned_trainer_set_params_v1(uint64_t handle, const float* params, uint64_t count) {
  return status([&] {
    if (!params) fail(INVALID_INPUT, "learned_train", "null parameters");
    require_count(count);
    std::lock_guard<std::mutex> l(g_learned_mu);
    gnn_trainer_set_params(trainer(handle), std::vector<float>(params, params + count));
  });
}

int32_t fevcb_learned_trainer_dump_v1(uint64_t handle, uint32_t graph, FevcbLearnedDumpV1* out, uint32_t cap) {
  return status([&] {
    require_capacity<FevcbLearnedDumpV1>(out, cap, "learned dump");
    std::lock_guard<std::mutex> l(g_learned_mu);
    GnnTrainer& t = trainer(handle);
    if (graph >= uint32_t(t.graphs())) fail(INVALID_INPUT, "learned_train", "graph index out of range");
    GnnTrainer::Dump& d = g_dumps[handle] = t.dump(int(graph));
    FevcbLearnedDumpV1 v{};
    v.struct_size = sizeof(v);
    v.pairs = d.pairs;
    v.vertices = d.n;
    v.row_ptr = d.ptr.data();
    v.col = d.col.data();
    v.weight = d.val.data();
    v.diagonal = d.diag.data();
    v.features = d.X.data();
    v.basis = d.Y.data();
    v.error = d.E.data();
    v.energy = d.ELE.data();
    std::memcpy(out, &v, sizeof(v));
  });
}

int32_t fevcb_cmg_aggregate_v1(uint32_t n, const uint32_t* ptr, const uint32_t* col, const double* val,
                               double threshold, uint32_t* labels, uint32_t* aggregates) {
  return status([&] {
    if (!ptr || !labels || !aggregates || (n > 0 && ptr[n] > 0 && (!col || !val)))
      fail(INVALID_INPUT, "cmg_aggregate", "null graph or output pointer");
    if (!(threshold >= 0.0 && threshold <= 1.0))
      fail(INVALID_INPUT, "cmg_aggregate", "low effective degree threshold must lie in [0, 1]");
    std::vector<uint32_t> P(ptr, ptr + n + 1), Cc(col, col + ptr[n]);
    std::vector<double> V(val, val + ptr[n]), D(n, 0.0);
    for (uint32_t v = 0; v < n; ++v)
      for (uint32_t e = P[v]; e < P[v + 1]; ++e) {
        if (Cc[e] >= n || !(V[e] > 0.0)) fail(INVALID_INPUT, "cmg_aggregate", "invalid edge");
        D[v] += V[e];
      }
    std::vector<uint32_t> out;
    *aggregates = forest_aggregation(n, P, Cc, V, D, threshold, out);
    std::copy(out.begin(), out.end(), labels);
  });
}

int32_t fevcb_engine_kernel_benchmark_v1(uint64_t generation, uint32_t kernel, uint32_t block_columns,
                                         uint32_t launches, double* ms, double* bytes) {
  return status([&] {
    if (!ms || !bytes) fail(INVALID_INPUT, "benchmark", "output pointers are null");
    std::lock_guard<std::mutex> l(reg().mu);
    Prepared& p = reg().require(generation, "engine_kernel_benchmark");
    if (!p.device) fail(STALE_CONTEXT, "engine_kernel_benchmark", "generation has no device state; solve it first");
    device_kernel_benchmark(*p.device, int(kernel), int(block_columns), int(launches), ms, bytes);
  });
}

int32_t fevcb_counter_atoms_v1(uint64_t seed, uint64_t domain_tag, uint64_t first_probe, uint32_t columns,
                               const uint64_t* entity, const uint64_t* trials, uint64_t count, int64_t* out) {
  return status([&] {
    if (!entity || !trials || !out || columns == 0 || count == 0)
      fail(INVALID_INPUT, "counter_rng", "semantic atom request has incompatible dimensions");
    device_atoms(seed, domain_tag, first_probe, columns, entity, trials, count, out);
  });
}

}  // extern "C"

// ---- fixed-effect projection attachment (reference ffi_engine.rs:2413-2418,
// 2883-2899, 3679-3835, 6030-6110, 9766-9846; session_retained.rs:443-613)

namespace {

const ProjectionResult& projection_of(uint64_t g, const char* phase) {
  reg().require(g, phase);
  if (reg().state != State::Solved || !reg().result)
    fail(CONTEXT_POISONED, "context_export", "generation " + std::to_string(g) + " has no solved result");
  const ProjectionResult& r = reg().result->projection;
  if (!r.present) fail(UNSUPPORTED_FEATURE, phase, "the solved generation has no projection result");
  return r;
}

VckssProjectionResultReceiptV1 projection_receipt(uint64_t g, const ProjectionResult& r) {
  VckssProjectionResultReceiptV1 v{};
  v.struct_size = sizeof(v);
  v.schema_version = VCKSS_PROJECTION_SCHEMA_V1;
  v.generation = g;
  v.columns = r.columns;
  v.effect = uint32_t(r.effect);
  v.weight = uint32_t(r.weight);
  v.gram_rcond = r.gram_rcond;
  v.gram_relres = r.gram_relres;
  v.gram_original_relres = r.gram_original_relres;
  v.covariance_smallest_eigenvalue = r.covariance_smallest_eigenvalue;
  v.covariance_largest_eigenvalue = r.covariance_largest_eigenvalue;
  v.psd_cleanup = r.psd_cleanup;
  v.proxy_minimum = r.proxy_minimum;
  v.proxy_maximum = r.proxy_maximum;
  v.maximum_iterations = r.maximum_iterations;
  v.maximum_reduced_residual = r.maximum_reduced_residual;
  v.maximum_complete_residual = r.maximum_complete_residual;
  v.full_residual_tolerance = r.full_residual_tolerance;
  v.projection_peak_forecast_bytes = r.projection_peak_forecast_bytes;
  v.persistent_bytes = r.persistent_bytes;
  v.result_bytes = r.result_bytes;
  return v;
}

}  // namespace

extern "C" {

uint32_t vckss_rust_projection_centering_schema_v1(void) { return 1; }

int32_t vckss_rust_engine_default_projection_augmentation_request_interrupt_v1(
    VckssProjectionAugmentationRequestInterruptV1* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssProjectionAugmentationRequestInterruptV1>(out, cap, "projection augmentation request");
    VckssProjectionAugmentationRequestInterruptV1 v{};
    v.options.abi_version = VCKSS_RUST_ABI_VERSION_V1;
    v.options.struct_size = sizeof(VckssProjectionAugmentationRequestInterruptV1);
    v.options.effect = VCKSS_PROJECTION_EFFECT_WORKER;
    v.options.weight = VCKSS_PROJECTION_WEIGHT_FREQUENCY;
    v.options.rank_tolerance = 1e-10;
    std::memcpy(out, &v, sizeof(v));
  });
}

int32_t vckss_rust_engine_augment_projection_interrupt_v1(uint64_t generation,
                                                           const VckssProjectionAugmentationRequestInterruptV1* request,
                                                           const VckssProjectionColumnsV1* columns) {
  return status([&] {
    auto q = read_struct(request, "projection augmentation request");
    Interrupt intr(q.interrupt_poll, q.interrupt_context, q.checkpoint_interval, q.reserved, "projection_augmentation");
    intr.check("engine_projection_augmentation_entry");
    const VckssProjectionAugmentationRequestV1& o = q.options;
    require_abi(o.abi_version);
    if (o.struct_size < sizeof(VckssProjectionAugmentationRequestV1) || o.reserved != 0 || o.rows == 0 ||
        o.project_count == 0 || !std::isfinite(o.rank_tolerance) || o.rank_tolerance < 1e-14 ||
        o.rank_tolerance >= 0.1)
      fail(INVALID_INPUT, "engine_projection_augmentation", "projection augmentation request is malformed");
    auto c = read_struct(columns, "projection column descriptor", 0);
    if (c.reserved != 0 || c.reserved_2 != 0 || c.rows != o.rows || c.project_count != o.project_count)
      fail(INVALID_INPUT, "engine_projection_augmentation", "projection request and column descriptor disagree");
    if (o.rows > (uint64_t(1) << 40) || o.caller_copy_bytes != o.rows * uint64_t(o.project_count) * 8)
      fail(INVALID_INPUT, "engine_projection_augmentation",
           "projection caller-copy bytes do not match the supplied dimensions");
    if (!c.project)
      fail(INVALID_INPUT, "engine_projection_augmentation", "positive projection count and pointer array are required");
    std::vector<std::vector<double>> project(o.project_count);
    for (uint32_t k = 0; k < o.project_count; ++k) {
      intr.check("engine_copy_projection_descriptors");
      const double* src = c.project[k];
      if (!src) fail(INVALID_INPUT, "engine_projection_augmentation", "projection column pointer is null");
      project[k].assign(src, src + o.rows);
      for (double v : project[k])
        if (!std::isfinite(v)) fail(INVALID_INPUT, "engine_projection_augmentation", "projection column has a nonfinite value");
    }
    if (o.effect != VCKSS_PROJECTION_EFFECT_WORKER && o.effect != VCKSS_PROJECTION_EFFECT_FIRM)
      fail(INVALID_INPUT, "engine_projection_augmentation", "unknown projection effect");
    if (o.weight != VCKSS_PROJECTION_WEIGHT_FREQUENCY && o.weight != VCKSS_PROJECTION_WEIGHT_TARGET)
      fail(INVALID_INPUT, "engine_projection_augmentation", "unknown projection weight");
    std::lock_guard<std::mutex> l(reg().mu);
    Prepared& p = reg().require(generation, "engine_projection_augmentation");
    if (reg().state != State::Prepared)
      fail(CONTEXT_POISONED, "context_augment",
           "generation " + std::to_string(generation) + " is not in the prepared state");
    // a refusal from here on fails the generation, as the reference's
    // registry does for a failed augmentation (session_retained.rs:443-613)
    struct Poison {
      bool armed = true;
      ~Poison() {
        if (armed) reg().state = State::Failed;
      }
    } poison;
    if (p.problem.rows() != o.rows)
      fail(INVALID_INPUT, "engine_projection_augmentation", "projection rows differ from the prepared retained sample");
    if (p.projection)
      fail(CONTEXT_POISONED, "session_projection_augmentation", "the prepared generation already owns a projection");
    if (o.project_count + 1 > PROJECTION_MAX_COLUMNS)
      fail(RESOURCE_LIMIT, "session_projection_augmentation", "the device projection handles at most 31 covariates");
    auto pp = std::make_shared<PreparedProjection>(prepare_projection(
        p.problem, project, ProjectionEffect(o.effect), ProjectionWeight(o.weight), o.rank_tolerance));
    // this library's resident accounting with the reference's augmentation
    // formula: two caller-sized copies, four persistent blocks, eight
    // q-square blocks and a header (session_retained.rs:532-553)
    const uint64_t resident = p.problem.rows() * (4 * 6 + 8 * 3) + p.problem.cells * (4 * 2 + 8 * 3);
    const uint64_t cols = pp->columns;
    pp->rows = o.rows;
    pp->caller_copy_bytes = o.caller_copy_bytes;
    pp->augmentation_peak_forecast_bytes =
        resident + 2 * o.caller_copy_bytes + 4 * pp->persistent_bytes + 8 * cols * cols * 8 + 4096;
    pp->total_prepared_resident_bytes = resident + pp->persistent_bytes;
    intr.check("session_projection_augmentation_final");
    p.projection = std::move(pp);
    poison.armed = false;
  });
}

int32_t vckss_rust_engine_projection_augmentation_receipt_v1(uint64_t generation,
                                                             VckssProjectionAugmentationReceiptV1* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssProjectionAugmentationReceiptV1>(out, cap, "projection augmentation receipt");
    std::lock_guard<std::mutex> l(reg().mu);
    Prepared& p = reg().require(generation, "engine_projection_augmentation_receipt");
    if (reg().state != State::Prepared)
      fail(CONTEXT_POISONED, "engine_projection_augmentation_receipt",
           "projection augmentation receipt must be read before solve");
    if (!p.projection)
      fail(UNSUPPORTED_FEATURE, "engine_projection_augmentation_receipt",
           "the prepared generation has no projection attachment");
    const PreparedProjection& pp = *p.projection;
    VckssProjectionAugmentationReceiptV1 v{};
    v.struct_size = sizeof(v);
    v.schema_version = VCKSS_PROJECTION_SCHEMA_V1;
    v.generation = generation;
    v.rows = pp.rows;
    v.columns = pp.columns;
    v.effect = uint32_t(pp.effect);
    v.weight = uint32_t(pp.weight);
    v.caller_copy_bytes = pp.caller_copy_bytes;
    v.augmentation_peak_forecast_bytes = pp.augmentation_peak_forecast_bytes;
    v.projection_persistent_bytes = pp.persistent_bytes;
    v.total_prepared_resident_bytes = pp.total_prepared_resident_bytes;
    v.gram_rcond = pp.gram_rcond;
    v.gram_relres = pp.gram_relres;
    v.gram_original_relres = pp.gram_original_relres;
    std::memcpy(out, &v, sizeof(v));
  });
}

int32_t vckss_rust_engine_projection_result_v1(uint64_t generation, double* coefficients,
                                               uint64_t coefficients_capacity, double* covariance,
                                               uint64_t covariance_capacity, double* naive_covariance,
                                               uint64_t naive_covariance_capacity,
                                               VckssProjectionResultReceiptV1* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssProjectionResultReceiptV1>(out, cap, "projection result receipt");
    std::lock_guard<std::mutex> l(reg().mu);
    const ProjectionResult& r = projection_of(generation, "engine_projection_result");
    auto put = [](double* dst, uint64_t capacity, const std::vector<double>& v, const char* label) {
      if (!dst || capacity < v.size())
        fail(INVALID_INPUT, "engine_projection_result", std::string(label) + " destination is null or short");
      std::memcpy(dst, v.data(), v.size() * sizeof(double));
    };
    put(coefficients, coefficients_capacity, r.coefficients, "projection coefficients");
    put(covariance, covariance_capacity, r.covariance, "projection covariance");
    put(naive_covariance, naive_covariance_capacity, r.naive_covariance, "naive projection covariance");
    VckssProjectionResultReceiptV1 v = projection_receipt(generation, r);
    std::memcpy(out, &v, sizeof(v));
  });
}

int32_t vckss_rust_engine_projection_result_receipt_v1(uint64_t generation, VckssProjectionResultReceiptV1* out,
                                                       uint32_t cap) {
  return status([&] {
    require_capacity<VckssProjectionResultReceiptV1>(out, cap, "projection result receipt");
    std::lock_guard<std::mutex> l(reg().mu);
    VckssProjectionResultReceiptV1 v =
        projection_receipt(generation, projection_of(generation, "engine_projection_result_receipt"));
    std::memcpy(out, &v, sizeof(v));
  });
}

}  // extern "C"

// ---- numerical MCSE attachment (reference vckss-plugin/src/numerical_api.rs)

namespace {

// validate_point with point_only (numerical_api.rs:113-203): schema, reserved
// fields, JLA with Counter-V1 on the automatic / diagonal / CMG route, no
// projection or component attachment, and a point request that reconciles
// with its planned capability for the request's control count.
void numerical_validate(const VckssNumericalRequestV1& q) {
  require_abi(q.abi_version);
  require_abi(q.point.v3.v2.v1.abi_version);
  if (q.schema_version != 1 || q.reserved != 0 || q.reserved_2 != 0 || q.tolerance_supplied > 1 ||
      q.projection_requested > 1 || q.component_requested > 1)
    fail(ABI_MISMATCH, "engine_ffi", "invalid numerical V1 schema or reserved fields");
  const VckssEngineSolveRequestV4& pt = q.point;
  if (pt.v3.v2.v1.struct_size < sizeof(VckssEngineSolveRequestV4))
    fail(ABI_MISMATCH, "engine_ffi", "numerical point prefix reports a short structure size");
  if (pt.v3.reserved_3 != 0 || pt.reserved_4 != 0)
    fail(ABI_MISMATCH, "engine_ffi", "reserved numerical point prefix fields must be zero");
  if (q.threads == 0 || pt.v3.v2.v1.probes < 2)
    fail(INVALID_INPUT, "numerical_preflight", "positive threads and at least two probes required");
  const uint32_t alg = pt.v3.v2.algorithm, eng = pt.v3.engine, route = pt.v3.v2.v1.solver_route;
  if (q.projection_requested != 0 || q.component_requested != 0 ||
      (alg != VCKSS_ALGORITHM_JLA && alg != VCKSS_ALGORITHM_AUTO) ||
      (eng != VCKSS_ENGINE_AUTO_OR_UNSPECIFIED && eng != VCKSS_ENGINE_GENERIC && eng != VCKSS_ENGINE_COMPRESSED) ||
      (route != VCKSS_ROUTE_AUTO && route != VCKSS_ROUTE_DIAGONAL_PCG && route != VCKSS_ROUTE_CMG_PCG) ||
      pt.v3.v2.v1.rng_contract != VCKSS_RNG_COUNTER_V1)
    fail(UNSUPPORTED_FEATURE, "numerical_preflight",
         "numerical V1 requires Counter-V1 JLA with no projection or component-inference attachment");
  VckssEngineSolveRequestV1 v1 = pt.v3.v2.v1;  // the point's option gates (automatic widths allowed)
  if (v1.leverage_batch_width == 0) v1.leverage_batch_width = 8;
  if (v1.target_batch_width == 0) v1.target_batch_width = 8;
  (void)options_from_v1(v1, true);
  auto c = capability_request_for_solve(pt, q.controls_count);
  const uint32_t reason = capability_reason(c);
  if (pt.v3.capability_schema != VCKSS_REQUEST_CAPABILITY_SCHEMA_V3 ||
      pt.v3.capability_profile != VCKSS_REQUEST_PROFILE_PLANNED_V1 || reason != VCKSS_REQUEST_REASON_SUPPORTED ||
      capability_signature(c) != pt.v3.request_signature)
    fail(UNSUPPORTED_FEATURE, "numerical_preflight",
         "numerical point request does not reconcile with its planned capability");
}

void numerical_solve(uint64_t g, const VckssNumericalRequestV1& q, const Interrupt& intr) {
  numerical_validate(q);
  SolveOptions o = options_from_v4(q.point);
  {
    std::lock_guard<std::mutex> l(reg().mu);
    Prepared& p = reg().require(g, "context_solve");
    if (p.projection)  // ffi_engine.rs:4926-4934
      fail(UNSUPPORTED_FEATURE, "numerical_preflight",
           "numerical V1 does not support projection or component-inference intersections");
    // algorithm(auto) resolves once the retained dimensions are known
    // (vckss-core/src/engine_plan.rs:179-240): exact within the exact limit
    const uint64_t complexity = uint64_t(p.problem.workers) + p.problem.firms - 1 + p.problem.controls.size();
    if (q.point.v3.v2.algorithm == VCKSS_ALGORITHM_AUTO && complexity <= q.point.v3.v2.exact_estimator_limit) {
      o.algorithm = 1;
      o.exact_limit = q.point.v3.v2.exact_estimator_limit;
      o.blocksize_limit = q.point.v3.v2.blocksize_limit ? q.point.v3.v2.blocksize_limit : 5000;
    }
  }
  o.numerical = true;
  solve_common(g, o, intr, true, &q.point, 4);
}

const NumericalAttachment& numerical_of(uint64_t g, const char* phase) {
  reg().require(g, phase);
  if (reg().state != State::Solved || !reg().result) fail(STALE_CONTEXT, phase, "generation has no solved result");
  const NumericalAttachment& a = reg().result->numerical;
  if (!a.present) fail(UNSUPPORTED_FEATURE, "numerical_preflight", "result has no numerical V1 attachment");
  return a;
}

}  // namespace

extern "C" {

uint32_t vckss_rust_numerical_schema_v1(void) { return 1; }

int32_t vckss_rust_engine_numerical_preflight_v1(const VckssNumericalRequestV1* request) {
  return status([&] { numerical_validate(read_struct(request, "numerical preflight")); });
}

int32_t vckss_rust_engine_solve_numerical_v1(uint64_t generation, const VckssNumericalRequestV1* request) {
  return status([&] { numerical_solve(generation, read_struct(request, "numerical solve"), Interrupt{}); });
}

int32_t vckss_rust_engine_solve_numerical_interrupt_v1(uint64_t generation, const VckssNumericalRequestV1* request,
                                                      VckssInterruptPollV1 poll, void* context, uint32_t interval) {
  return status([&] {
    auto q = read_struct(request, "numerical interrupt solve");
    numerical_solve(generation, q, Interrupt(poll, context, interval, 0, "numerical"));
  });
}

int32_t vckss_rust_engine_numerical_result_v1(uint64_t generation, VckssNumericalResultV1* out, uint32_t cap) {
  return status([&] {
    require_capacity<VckssNumericalResultV1>(out, cap, "numerical result");
    std::lock_guard<std::mutex> l(reg().mu);
    const NumericalAttachment& a = numerical_of(generation, "numerical_result");
    const SolveResult& s = *reg().result;
    VckssNumericalResultV1 v{};
    v.struct_size = sizeof(v);
    v.schema_version = 1;
    v.generation = generation;
    v.status = a.status;
    v.engine = a.exact ? 3u : a.engine;
    v.failed_replay_probe = 0xffffffffu;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        v.conditional[i][j] = a.conditional[i][j];
        v.leverage[i][j] = a.leverage[i][j];
        v.raw[i][j] = a.raw[i][j];
        v.usable[i][j] = a.usable[i][j];
      }
    for (int k = 0; k < 4; ++k) v.mcse[k] = a.mcse[k];
    v.psd_adjustment = a.psd_adjustment;
    if (!a.exact) {
      v.leverage_probes = a.leverage_probes;
      v.target_probes = a.target_probes;
      v.target_fold_a = a.folds[0];
      v.target_fold_b = a.folds[1];
      v.certified_replay_rhs = a.replay_probe.size();
      v.executed_replay_rhs = a.replay_probe.size();
      v.attempted_replay_rhs = a.attempted_replay_rhs;
      v.replay_generator_words = a.generator_words;
      v.allocation_bound_bytes = a.allocation_bound_bytes;
      v.failed_replay_probe = a.failed_replay_probe;
      v.replay_error_code = a.replay_error_code;
      for (int f = 0; f < 2; ++f)
        for (int j = 0; j < 3; ++j) v.score_means[f][j] = a.score_means[f][j];
      v.minimum_constrained = a.minimum_constrained;
      v.minimum_residual_margin = a.minimum_residual_margin;
      v.maximum_sensitivity_ratio = a.maximum_sensitivity_ratio;
      double mx = 0.0;
      for (double r : a.replay_residual) mx = std::max(mx, r);
      v.maximum_replay_complete_residual = mx;
      v.point_rhs = s.receipts.size();
      v.maximum_point_complete_residual = s.max_complete_residual;
    }
    std::memcpy(out, &v, sizeof(v));
  });
}

// The attachment's host covariance algebra on given conditional and leverage
// matrices (row-major 3 x 3): fills status, conditional, leverage, raw,
// usable, mcse and psd_adjustment of *out and zeroes the rest.
int32_t fevcb_numerical_finalize_v1(const double* conditional, const double* leverage, VckssNumericalResultV1* out,
                                    uint32_t cap) {
  return status([&] {
    require_capacity<VckssNumericalResultV1>(out, cap, "numerical finalize");
    if (!conditional || !leverage) fail(INVALID_INPUT, "numerical_mc", "null covariance input");
    Matrix3 c{}, l{};
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        c[i][j] = conditional[3 * i + j];
        l[i][j] = leverage[3 * i + j];
      }
    NumericalAttachment a;
    finalize_covariance(c, l, a);
    VckssNumericalResultV1 v{};
    v.struct_size = sizeof(v);
    v.schema_version = 1;
    v.status = a.status;
    v.failed_replay_probe = 0xffffffffu;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        v.conditional[i][j] = a.conditional[i][j];
        v.leverage[i][j] = a.leverage[i][j];
        v.raw[i][j] = a.raw[i][j];
        v.usable[i][j] = a.usable[i][j];
      }
    for (int k = 0; k < 4; ++k) v.mcse[k] = a.mcse[k];
    v.psd_adjustment = a.psd_adjustment;
    std::memcpy(out, &v, sizeof(v));
  });
}

int32_t vckss_rust_engine_numerical_rhs_v1(uint64_t generation, VckssNumericalRhsV1* out, uint64_t capacity,
                                          uint64_t* written) {
  return status([&] {
    if (!written) fail(ABI_MISMATCH, "engine_ffi", "numerical RHS count destination is null");
    std::lock_guard<std::mutex> l(reg().mu);
    const NumericalAttachment& a = numerical_of(generation, "numerical_rhs");
    const uint64_t n = a.exact ? 0 : a.replay_probe.size();
    if (capacity > uint64_t(INT64_MAX) / sizeof(VckssNumericalRhsV1) || capacity < n || (n != 0 && !out))
      fail(ABI_MISMATCH, "engine_ffi", "invalid or short numerical RHS destination");
    const uintptr_t start = reinterpret_cast<uintptr_t>(out), stop = start + n * sizeof(VckssNumericalRhsV1);
    const uintptr_t cs = reinterpret_cast<uintptr_t>(written), ce = cs + sizeof(uint64_t);
    if (n != 0 && start < ce && cs < stop)
      fail(ABI_MISMATCH, "engine_ffi", "numerical RHS and count destinations overlap");
    for (uint64_t i = 0; i < n; ++i) {
      VckssNumericalRhsV1 r{};
      r.schema_version = 1;
      r.phase = 1;
      r.probe = a.replay_probe[i];
      r.complete_residual = a.replay_residual[i];
      std::memcpy(out + i, &r, sizeof(r));
    }
    *written = n;
  });
}

}  // extern "C"


extern "C" int32_t fevcb_counter_atoms_noalloc_v1(uint64_t seed, uint64_t domain_tag, uint64_t first_probe,
                                                  uint32_t columns, const uint64_t* entity, const uint64_t* trials,
                                                  uint64_t count, int64_t* out) {
  return status([&] {
    if (!entity || !trials || !out || columns == 0 || count == 0)
      fail(INVALID_INPUT, "counter_rng", "semantic atom request has incompatible dimensions");
    device_atoms_noalloc(seed, domain_tag, first_probe, columns, entity, trials, count, out);
  });
}
