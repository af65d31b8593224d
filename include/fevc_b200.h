/* fevc-b200: B200-native leave-out leverage engine, C ABI.
 *
 * The library exports the plugin entry points of fevc's Rust backend for the
 * JLA solve path with the same names, struct layouts and status codes, so a
 * caller written against rust/stata_backend/include/vckss_rust.h (the Stata C
 * shim rust/stata_backend/cshim/stata_entry.c, or a C harness) links or
 * dlopens this library unchanged.  Each declaration cites the reference
 * function it replaces (paths inside the reference project).
 *
 * Lifecycle: prepare (host ingest, graph pruning, compression, semantic plan)
 * -> optional centering -> solve (device) -> result / receipts -> release.
 * One generation is active at a time; the caller owns all memory; every output
 * is capacity-checked.  Status codes: 0 OK, 1 USER_BREAK, 10 ABI_MISMATCH,
 * 11 UNSUPPORTED_FEATURE, 20..23 invalid input, 30..32 graph, 40/41 resources,
 * 60..64 solver, 70..79 estimator, 80..82 context, 90 invariant, 99 panic
 * (reference rust/crates/vckss-core/src/error.rs:8-48).
 *
 * Entry points prefixed fevcb_ are B200 extensions with no reference
 * counterpart (device selection, stream binding, timings, raw device atoms).
 */
#ifndef FEVC_B200_H
#define FEVC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VCKSS_RUST_ABI_VERSION_V1 1u
#define VCKSS_DELETION_MATCH 1u
#define VCKSS_DELETION_OBSERVATION 2u
#define VCKSS_RNG_COUNTER_V1 1u
#define VCKSS_ROUTE_AUTO 0u
#define VCKSS_ROUTE_EXACT 1u
#define VCKSS_ROUTE_DIAGONAL_PCG 2u
#define VCKSS_ROUTE_CMG_PCG 3u
#define VCKSS_RESIDUAL_SPACE_WORKER_FIRM 1u
#define VCKSS_RESIDUAL_SPACE_WORKER_FIRM_CONTROL 2u
#define VCKSS_REQUEST_CAPABILITY_SCHEMA_V3 3u
#define VCKSS_REQUEST_FREQUENCY_UNIT 0u
#define VCKSS_REQUEST_FREQUENCY_LITERAL 1u
#define VCKSS_REQUEST_PROFILE_NONE 0u
#define VCKSS_REQUEST_PROFILE_PLANNED_V1 4u
#define VCKSS_ALGORITHM_AUTO 0u
#define VCKSS_ALGORITHM_EXACT 1u
#define VCKSS_ALGORITHM_JLA 2u
#define VCKSS_NUISANCE_JOINT 1u
#define VCKSS_NUISANCE_FIXED_OFFSET 2u
#define VCKSS_RNG_NONE 0u
#define VCKSS_ENGINE_AUTO_OR_UNSPECIFIED 0u
#define VCKSS_ENGINE_COMPRESSED 1u
#define VCKSS_ENGINE_GENERIC 2u
#define VCKSS_BATCH_MODE_AUTO 0u
#define VCKSS_BATCH_MODE_EXPLICIT 1u
#define VCKSS_BATCH_MODE_INDEPENDENT 2u
#define VCKSS_STAYERS_MOVERS 1u
#define VCKSS_STAYERS_ALL 2u
#define VCKSS_TARGET_WEIGHT_FREQUENCY_DEFAULT 0u
#define VCKSS_TARGET_WEIGHT_STORED_ROW_EXPLICIT 1u
#define VCKSS_DELETION_SOURCE_CELL_DEFAULT 1u
#define VCKSS_DELETION_SOURCE_MATCH_ID_EXPLICIT 2u
#define VCKSS_DELETION_SOURCE_OBSERVATION_ROW 3u
/* request capability reason codes (reference vckss_rust.h:89-124) */
#define VCKSS_REQUEST_REASON_SUPPORTED 0u
#define VCKSS_REQUEST_REASON_UNKNOWN_SCHEMA 1u
#define VCKSS_REQUEST_REASON_UNKNOWN_ALGORITHM 2u
#define VCKSS_REQUEST_REASON_UNKNOWN_DELETION 4u
#define VCKSS_REQUEST_REASON_UNKNOWN_NUISANCE 5u
#define VCKSS_REQUEST_REASON_UNKNOWN_SOLVER_ROUTE 6u
#define VCKSS_REQUEST_REASON_UNKNOWN_RNG_CONTRACT 7u
#define VCKSS_REQUEST_REASON_UNKNOWN_FREQUENCY_USE 8u
#define VCKSS_REQUEST_REASON_CONTROLS_LIMIT 9u
#define VCKSS_REQUEST_REASON_EXACT_RNG 10u
#define VCKSS_REQUEST_REASON_EXACT_SOLVER_ROUTE 11u
#define VCKSS_REQUEST_REASON_JLA_RNG 15u
#define VCKSS_REQUEST_REASON_UNKNOWN_ENGINE 16u
#define VCKSS_REQUEST_REASON_EXACT_ENGINE 17u
#define VCKSS_REQUEST_REASON_JLA_GENERIC_SOLVER_ROUTE 19u
#define VCKSS_REQUEST_REASON_UNKNOWN_BATCH_MODE 20u
#define VCKSS_REQUEST_REASON_UNKNOWN_STAYERS_MODE 21u
#define VCKSS_REQUEST_REASON_UNKNOWN_TARGET_WEIGHT_MODE 22u
#define VCKSS_REQUEST_REASON_UNKNOWN_DELETION_UNIT_SOURCE 23u
#define VCKSS_REQUEST_REASON_PROBEORDER_UNSUPPORTED 24u
#define VCKSS_REQUEST_REASON_WALLSECONDS_UNSUPPORTED 25u
#define VCKSS_REQUEST_REASON_PHYSICAL_LIMIT 26u
#define VCKSS_REQUEST_REASON_DELETION_UNIT_SOURCE_MISMATCH 27u
#define VCKSS_REQUEST_REASON_STAYERS_MODE_UNSUPPORTED 29u
#define VCKSS_REQUEST_REASON_BATCH_SUMMARY_MISMATCH 30u
#define VCKSS_REQUEST_REASON_WALLSECONDS_VALUE 31u
#define VCKSS_REQUEST_REASON_FALLBACK_ROUTE_MISMATCH 32u
#define VCKSS_REQUEST_REASON_AUTO_RNG 33u
#define VCKSS_REQUEST_REASON_AUTO_ENGINE_COMPRESSED 34u
#define VCKSS_REQUEST_REASON_COMPRESSED_SCIENTIFIC_INELIGIBILITY 35u
#define VCKSS_INTERRUPT_CONTINUE 0
#define VCKSS_INTERRUPT_USER_BREAK 1

typedef int32_t (*VckssInterruptPollV1)(void *context);

/* ---- preparation requests (reference vckss_rust.h:261-290) ---- */
typedef struct VckssEnginePrepareRequestV1 {
  uint32_t abi_version;
  uint32_t struct_size;
  uint64_t rows;
  uint32_t cleanup_abandoned;
  uint32_t reserved;
} VckssEnginePrepareRequestV1;

typedef struct VckssEnginePrepareRequestV2 {
  uint32_t abi_version;
  uint32_t struct_size;
  uint64_t rows;
  uint32_t cleanup_abandoned;
  uint32_t reserved;
  uint64_t memory_limit_bytes;
  uint64_t caller_copy_bytes;
} VckssEnginePrepareRequestV2;

typedef struct VckssEnginePrepareRequestV3 {
  VckssEnginePrepareRequestV2 v2;
  uint32_t deletion_mode;
  uint32_t controls_count;
  uint64_t reserved_2;
} VckssEnginePrepareRequestV3;

typedef struct VckssEnginePrepareRequestV4 {
  VckssEnginePrepareRequestV3 v3;
  uint32_t implicit_match;
  uint32_t reserved_3;
} VckssEnginePrepareRequestV4;

typedef struct VckssEnginePrepareRequestInterruptV1 {
  VckssEnginePrepareRequestV2 options;
  VckssInterruptPollV1 interrupt_poll;
  void *interrupt_context;
  uint32_t checkpoint_interval;
  uint32_t reserved;
} VckssEnginePrepareRequestInterruptV1;

typedef struct VckssEnginePrepareRequestInterruptV2 {
  VckssEnginePrepareRequestV3 options;
  VckssInterruptPollV1 interrupt_poll;
  void *interrupt_context;
  uint32_t checkpoint_interval;
  uint32_t reserved;
} VckssEnginePrepareRequestInterruptV2;

typedef struct VckssEnginePrepareRequestInterruptV3 {
  VckssEnginePrepareRequestV4 options;
  VckssInterruptPollV1 interrupt_poll;
  void *interrupt_context;
  uint32_t checkpoint_interval;
  uint32_t reserved;
} VckssEnginePrepareRequestInterruptV3;

/* ---- caller columns, binary64 (reference vckss_rust.h:343-367) ---- */
typedef struct VckssEngineColumnsV1 {
  uint32_t struct_size;
  uint32_t reserved;
  uint64_t rows;
  const double *worker;
  const double *firm;
  const double *deletion;
  const double *outcome;
  const double *frequency;
  const double *target_weight;
} VckssEngineColumnsV1;

typedef struct VckssEngineColumnsV2 {
  VckssEngineColumnsV1 v1;
  const double *const *controls;
  uint32_t controls_count;
  uint32_t reserved_2;
} VckssEngineColumnsV2;

typedef struct VckssEngineColumnsV3 {
  VckssEngineColumnsV2 v2;
  const double *probe_order;
  uint32_t probeorder_supplied;
  uint32_t reserved_3;
} VckssEngineColumnsV3;

/* ---- solve requests (reference vckss_rust.h:501-571) ---- */
typedef struct VckssEngineSolveRequestV1 {
  uint32_t abi_version;
  uint32_t struct_size;
  uint64_t seed;
  uint32_t probes;
  uint32_t leverage_batch_width;
  uint32_t target_batch_width;
  uint32_t deletion_mode;
  uint32_t rng_contract;
  uint32_t solver_route;
  uint32_t allow_automatic_cmg_setup_fallback;
  uint64_t exact_dimension_limit;
  uint64_t cmg_minimum_dimension;
  double pcg_tolerance;
  uint32_t maximum_iterations;
  uint32_t residual_replacement_interval;
  double rank_tolerance;
  double block_tolerance;
  uint64_t cmg_terminal_vertices;
  uint64_t cmg_dense_vertex_cap;
  uint64_t cmg_maximum_levels;
  uint64_t cmg_aggregate_cap;
  double cmg_minimum_reduction;
  double cmg_jacobi_weight;
  uint32_t cmg_pre_sweeps;
  uint32_t cmg_post_sweeps;
  double cmg_maximum_edge_complexity;
  double cmg_maximum_vertex_complexity;
  uint64_t cmg_memory_limit_bytes;
} VckssEngineSolveRequestV1;

typedef struct VckssEngineSolveRequestV2 {
  VckssEngineSolveRequestV1 v1;
  uint32_t algorithm;
  uint32_t nuisance_mode;
  uint64_t exact_estimator_limit;
  uint64_t blocksize_limit;
} VckssEngineSolveRequestV2;

typedef struct VckssEngineSolveRequestV3 {
  VckssEngineSolveRequestV2 v2;
  uint32_t engine;
  uint32_t batch_mode;
  uint32_t stayers_mode;
  uint32_t target_weight_mode;
  uint32_t deletion_unit_source;
  uint32_t probeorder_supplied;
  uint32_t wallseconds_supplied;
  uint32_t capability_schema;
  uint32_t capability_profile;
  uint32_t frequency_use;
  uint64_t physical_limit;
  uint64_t request_signature;
  uint64_t reserved_3;
} VckssEngineSolveRequestV3;

typedef struct VckssEngineSolveRequestV4 {
  VckssEngineSolveRequestV3 v3;
  uint32_t leverage_batch_mode;
  uint32_t target_batch_mode;
  double wallseconds;
  uint64_t reserved_4;
} VckssEngineSolveRequestV4;

typedef struct VckssEngineSolveRequestV5 {
  VckssEngineSolveRequestV4 v4;
  uint32_t threads;
  uint32_t tolerance_supplied;
  uint32_t full_cmg_v2;
  uint32_t reserved_5;
} VckssEngineSolveRequestV5;

typedef struct VckssEngineSolveRequestInterruptV1 {
  VckssEngineSolveRequestV1 options;
  VckssInterruptPollV1 interrupt_poll;
  void *interrupt_context;
  uint32_t checkpoint_interval;
  uint32_t reserved;
} VckssEngineSolveRequestInterruptV1;

typedef struct VckssEngineSolveRequestInterruptV5 {
  VckssEngineSolveRequestV5 options;
  VckssInterruptPollV1 interrupt_poll;
  void *interrupt_context;
  uint32_t checkpoint_interval;
  uint32_t reserved;
} VckssEngineSolveRequestInterruptV5;

typedef struct VckssEngineSolveRequestInterruptV4 {
  VckssEngineSolveRequestV4 options;
  VckssInterruptPollV1 interrupt_poll;
  void *interrupt_context;
  uint32_t checkpoint_interval;
  uint32_t reserved;
} VckssEngineSolveRequestInterruptV4;

/* V6-V8 extend V4 (reference vckss_rust.h:577-660). */
typedef struct VckssEngineSolveRequestV6 {
  VckssEngineSolveRequestV4 v4;
  uint32_t execution_mode;
  uint32_t threads;
  uint64_t reserved_6;
} VckssEngineSolveRequestV6;

typedef struct VckssEngineSolveRequestV7 {
  VckssEngineSolveRequestV6 v6;
  uint32_t component_batch_mode;
  uint32_t reserved_7;
} VckssEngineSolveRequestV7;

typedef struct VckssEngineSolveRequestV8 {
  VckssEngineSolveRequestV7 v7;
  uint32_t resolved_execution_mode;
  uint32_t tolerance_supplied;
} VckssEngineSolveRequestV8;

/* Numerical MCSE attachment (reference vckss_rust.h:2335-2388,
 * vckss-plugin/src/numerical_api.rs:17-100): a V4 point request, and the
 * covariance of the (worker, firm, covariance) corrections from the target
 * draws (conditional) and from a replay of the leverage probes (leverage). */
typedef struct VckssNumericalRequestV1 {
  uint32_t abi_version, struct_size, schema_version, threads;
  uint32_t tolerance_supplied, projection_requested, component_requested, reserved;
  uint32_t controls_count, reserved_2;
  VckssEngineSolveRequestV4 point;
} VckssNumericalRequestV1;

typedef struct VckssNumericalRequestV2 {
  VckssNumericalRequestV1 v1;
  uint32_t execution_mode, component_batch_mode, full_cmg, reserved;
} VckssNumericalRequestV2;

typedef struct VckssNumericalResultV1 {
  uint32_t struct_size, schema_version;
  uint64_t generation;
  /* 1 exact zero, 2 local, 3 local after PSD adjustment, 4 unstable (not PSD),
   * 5 nonsmooth adjustment, 6 nonfinite derivative, 7 replay failed */
  uint32_t status, engine, leverage_probes, target_probes, target_fold_a, target_fold_b;
  uint64_t certified_replay_rhs, executed_replay_rhs, attempted_replay_rhs, replay_generator_words,
      allocation_bound_bytes;
  uint32_t failed_replay_probe, replay_error_code;
  double psd_adjustment, minimum_constrained, minimum_residual_margin, maximum_sensitivity_ratio;
  double score_means[2][3];
  double conditional[3][3], leverage[3][3], raw[3][3], usable[3][3], mcse[4];
  uint64_t point_rhs;
  double maximum_point_complete_residual, maximum_replay_complete_residual;
} VckssNumericalResultV1;

typedef struct VckssNumericalRhsV1 {
  uint32_t schema_version, phase, probe, reserved;
  double complete_residual;
} VckssNumericalRhsV1;

typedef struct VckssEngineSolveRequestInterruptV8 {
  VckssEngineSolveRequestV8 options;
  VckssInterruptPollV1 interrupt_poll;
  void *interrupt_context;
  uint32_t checkpoint_interval;
  uint32_t reserved;
} VckssEngineSolveRequestInterruptV8;

/* ---- request capability (reference vckss_rust.h:177-259) ---- */
typedef struct VckssBackendRequestCapabilityRequestV1 {
  uint32_t abi_version;
  uint32_t struct_size;
  uint32_t request_schema;
  uint32_t algorithm;
  uint32_t deletion_mode;
  uint32_t nuisance_mode;
  uint32_t solver_route;
  uint32_t rng_contract;
  uint32_t controls_count;
  uint32_t frequency_use;
  uint64_t reserved;
} VckssBackendRequestCapabilityRequestV1;

typedef struct VckssBackendRequestCapabilityReceiptV1 {
  uint32_t struct_size;
  uint32_t abi_version;
  uint32_t request_schema;
  uint32_t supported;
  uint32_t reason_code;
  uint32_t profile_code;
  uint32_t algorithm;
  uint32_t deletion_mode;
  uint32_t nuisance_mode;
  uint32_t solver_route;
  uint32_t rng_contract;
  uint32_t controls_count;
  uint32_t frequency_use;
  uint32_t reserved;
  uint64_t request_signature;
} VckssBackendRequestCapabilityReceiptV1;

typedef struct VckssBackendRequestCapabilityRequestV2 {
  VckssBackendRequestCapabilityRequestV1 v1;
  uint32_t engine;
  uint32_t batch_mode;
  uint32_t stayers_mode;
  uint32_t target_weight_mode;
  uint32_t deletion_unit_source;
  uint32_t probeorder_supplied;
  uint32_t wallseconds_supplied;
  uint32_t reserved_2;
  uint64_t physical_limit;
} VckssBackendRequestCapabilityRequestV2;

typedef struct VckssBackendRequestCapabilityReceiptV2 {
  VckssBackendRequestCapabilityReceiptV1 v1;
  uint32_t engine;
  uint32_t batch_mode;
  uint32_t stayers_mode;
  uint32_t target_weight_mode;
  uint32_t deletion_unit_source;
  uint32_t probeorder_supplied;
  uint32_t wallseconds_supplied;
  uint32_t reserved_2;
  uint64_t physical_limit;
} VckssBackendRequestCapabilityReceiptV2;

typedef struct VckssBackendRequestCapabilityRequestV3 {
  VckssBackendRequestCapabilityRequestV2 v2;
  uint32_t leverage_batch_mode;
  uint32_t target_batch_mode;
  uint32_t allow_automatic_cmg_setup_fallback;
  uint32_t reserved_3;
  double wallseconds;
  uint64_t reserved_4;
} VckssBackendRequestCapabilityRequestV3;

typedef struct VckssBackendRequestCapabilityReceiptV3 {
  VckssBackendRequestCapabilityReceiptV2 v2;
  uint32_t leverage_batch_mode;
  uint32_t target_batch_mode;
  uint32_t allow_automatic_cmg_setup_fallback;
  uint32_t reserved_3;
  double wallseconds;
  uint32_t algorithm_resolution_deferred;
  uint32_t engine_resolution_deferred;
  uint32_t route_resolution_deferred;
  uint32_t leverage_batch_resolution_deferred;
  uint32_t target_batch_resolution_deferred;
  uint32_t wall_advisory_only;
  uint64_t reserved_4;
} VckssBackendRequestCapabilityReceiptV3;

/* ---- full-CMG receipt (reference vckss_rust.h:1458-1509): this library
 * fills it from the device solve (hybrid graph, hierarchy when the CMG route
 * ran, right-hand-side and iteration totals, residual maxima). ---- */
typedef struct VckssFullCmgReceiptV1 {
  uint32_t struct_size;
  uint32_t schema_version;
  uint64_t generation;
  uint32_t backend_identity;
  uint32_t platform_os;
  uint32_t platform_arch;
  uint32_t batch_strategy_mask;
  uint8_t cmg_source_commit[40];
  uint32_t threads_requested;
  uint32_t threads_used;
  uint64_t maximum_concurrency;
  uint64_t vertices;
  uint64_t edges;
  uint64_t hierarchy_levels;
  uint64_t terminal_vertices;
  uint64_t graph_copy_bytes;
  uint64_t hierarchy_bytes;
  uint64_t plan_bytes;
  uint64_t workspace_bytes_each;
  uint64_t workspace_pool_bytes;
  uint64_t admitted_peak_bytes;
  double fit_effective_tolerance;
  double probe_effective_tolerance;
  double fit_initial_inner_tolerance;
  double probe_initial_inner_tolerance;
  uint64_t refinement_attempts;
  uint64_t refined_columns;
  uint64_t batch_calls;
  uint64_t rhs_count;
  uint64_t serial_batches;
  uint64_t planned_batches;
  uint64_t across_rhs_batches;
  uint64_t total_iterations;
  uint64_t total_operator_applications;
  uint64_t total_preconditioner_applications;
  double maximum_reduced_residual;
  double maximum_complete_residual;
  uint64_t graph_ns;
  uint64_t hierarchy_plan_ns;
  uint64_t rhs_ns;
  uint64_t solve_ns;
  uint64_t extraction_ns;
  uint64_t preparation_peak_bytes;
  uint64_t prepared_persistent_bytes;
  uint64_t non_cmg_command_peak_bytes;
  uint64_t pre_rng_forecast_bytes;
  uint64_t actual_retained_bytes;
  uint64_t allocator_allowance_bytes;
  uint64_t maximum_batch_rhs;
  uint64_t workspace_count;
} VckssFullCmgReceiptV1;

/* ---- results and receipts (reference vckss_rust.h:711-768, 1037-1052, 1611-1634) ---- */
typedef struct VckssComponentVectorV1 {
  double worker;
  double firm;
  double covariance;
  double total;
} VckssComponentVectorV1;

typedef struct VckssEngineResultV1 {
  uint32_t struct_size;
  uint32_t reserved;
  uint64_t generation;
  VckssComponentVectorV1 plugin;
  VckssComponentVectorV1 correction;
  VckssComponentVectorV1 corrected;
  VckssComponentVectorV1 numerical_mcse;
} VckssEngineResultV1;

typedef struct VckssEnginePreparationReceiptV1 {
  uint32_t struct_size;
  uint32_t reserved;
  uint64_t generation;
  uint64_t input_rows;
  uint64_t retained_rows;
  uint64_t workers;
  uint64_t firms;
  uint64_t cells;
  uint64_t deletion_units;
  uint64_t target_strata;
} VckssEnginePreparationReceiptV1;

typedef struct VckssEnginePreparationReceiptV2 {
  uint32_t struct_size;
  uint32_t reserved;
  uint64_t generation;
  uint64_t input_rows;
  uint64_t retained_rows;
  uint64_t workers;
  uint64_t firms;
  uint64_t cells;
  uint64_t deletion_units;
  uint64_t target_strata;
  uint64_t memory_limit_bytes;
  uint64_t caller_copy_bytes;
  uint64_t preparation_peak_forecast_bytes;
  uint64_t prepared_resident_bytes;
  uint64_t graph_input_rows;
  uint64_t graph_retained_rows;
  uint64_t graph_input_physical_mass;
  uint64_t graph_retained_physical_mass;
  uint64_t graph_initial_components;
  uint64_t graph_maximum_components;
  uint64_t graph_initial_component_rows;
  uint64_t graph_mover_input_rows;
  uint64_t graph_initial_deletion_edges;
  uint64_t graph_retained_deletion_edges;
  uint64_t graph_insufficient_workers_removed;
  uint64_t graph_articulation_workers_removed;
  uint64_t graph_bridge_units_removed;
  uint64_t graph_bridge_rows_removed;
  uint64_t graph_degree_iterations;
  uint64_t graph_articulation_iterations;
  uint64_t graph_bridge_iterations;
  uint64_t graph_fixed_point_iterations;
} VckssEnginePreparationReceiptV2;

typedef struct VckssEnginePreparationReceiptV3 {
  VckssEnginePreparationReceiptV2 v2;
  double target_weight_sum;
} VckssEnginePreparationReceiptV3;

typedef struct VckssEnginePreparationReceiptV4 {
  VckssEnginePreparationReceiptV3 v3;
  uint32_t controls_count;
  uint32_t deletion_mode;
} VckssEnginePreparationReceiptV4;

typedef struct VckssEngineRhsReceiptV1 {
  uint32_t phase;
  uint32_t side;
  int64_t probe;
  uint32_t route;
  uint32_t iterations;
  uint32_t zero_rhs;
  uint32_t reserved;
  double reduced_residual;
  double complete_residual;
} VckssEngineRhsReceiptV1;

typedef struct VckssEngineRhsReceiptV2 {
  VckssEngineRhsReceiptV1 v1;
  uint32_t status;
  uint32_t residual_replacements;
  uint64_t operator_applications;
  uint64_t preconditioner_applications;
  double full_residual_tolerance;
  uint32_t residual_space;
  uint32_t reserved_2;
  uint64_t solver_dimension;
} VckssEngineRhsReceiptV2;

typedef struct VckssEngineSnapshotV1 {
  uint32_t struct_size;
  uint32_t state;
  uint64_t generation;
  uint64_t last_released_generation;
} VckssEngineSnapshotV1;

typedef struct VckssBackendCapabilitiesV1 {
  uint32_t struct_size;
  uint32_t abi_version;
  uint64_t core_ready_flags;
  uint64_t support_flags;
  uint32_t deterministic_parallelism;
  uint32_t reserved;
} VckssBackendCapabilitiesV1;

/* ---- library identity (reference ffi_engine.rs / vckss_rust.h:1642-1650) ---- */
uint32_t vckss_rust_abi_version(void);
const char *vckss_rust_backend_version(void);
const char *vckss_rust_capabilities_json(void);
const char *vckss_rust_last_error(void);
int32_t vckss_rust_selftest(void);
int32_t vckss_rust_backend_capabilities_v1(VckssBackendCapabilitiesV1 *output, uint32_t output_capacity_bytes);

/* ---- defaults (reference ffi_engine.rs:1094-1276, 2723-2800) ---- */
int32_t vckss_rust_engine_default_solve_request_v1(VckssEngineSolveRequestV1 *output, uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_default_solve_request_v2(VckssEngineSolveRequestV2 *output, uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_default_solve_request_v3(VckssEngineSolveRequestV3 *output, uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_default_solve_request_v4(VckssEngineSolveRequestV4 *output, uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_default_solve_request_v5(VckssEngineSolveRequestV5 *output, uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_default_solve_request_interrupt_v1(VckssEngineSolveRequestInterruptV1 *output,
                                                             uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_default_solve_request_interrupt_v5(VckssEngineSolveRequestInterruptV5 *output,
                                                             uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_default_prepare_request_v3(VckssEnginePrepareRequestV3 *output, uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_default_prepare_request_interrupt_v1(VckssEnginePrepareRequestInterruptV1 *output,
                                                               uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_default_prepare_request_interrupt_v2(VckssEnginePrepareRequestInterruptV2 *output,
                                                               uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_default_prepare_request_interrupt_v3(VckssEnginePrepareRequestInterruptV3 *output,
                                                               uint32_t output_capacity_bytes);

/* ---- preparation (reference ffi_engine.rs:3270-3316 prepare_v1; 3318-3470 V2/V3; V4 implicit match) ---- */
int32_t vckss_rust_engine_prepare_v1(const VckssEnginePrepareRequestV1 *request, const VckssEngineColumnsV1 *columns,
                                     uint64_t *output_handle, uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_prepare_v2(const VckssEnginePrepareRequestV2 *request, const VckssEngineColumnsV1 *columns,
                                     uint64_t *output_handle, uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_prepare_v3(const VckssEnginePrepareRequestV3 *request, const VckssEngineColumnsV2 *columns,
                                     uint64_t *output_handle, uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_prepare_interrupt_v1(const VckssEnginePrepareRequestInterruptV1 *request,
                                               const VckssEngineColumnsV1 *columns, uint64_t *output_handle,
                                               uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_prepare_interrupt_v2(const VckssEnginePrepareRequestInterruptV2 *request,
                                               const VckssEngineColumnsV2 *columns, uint64_t *output_handle,
                                               uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_prepare_interrupt_v4(const VckssEnginePrepareRequestInterruptV3 *request,
                                               const VckssEngineColumnsV3 *columns, uint64_t *output_handle,
                                               uint32_t output_capacity_bytes);

/* centering mode 0 None, 1 Mean (2 Corrected is refused) (reference ffi_engine.rs:2446-2467) */
int32_t vckss_rust_engine_centering_v1(uint64_t generation, uint32_t mode);

/* ---- solve (reference ffi_engine.rs:4474-4500 V1, 4629-4690 V5; body 5892-6000) ---- */
int32_t vckss_rust_engine_solve_v1(uint64_t generation, const VckssEngineSolveRequestV1 *request);
int32_t vckss_rust_engine_solve_interrupt_v1(uint64_t generation, const VckssEngineSolveRequestInterruptV1 *request);
int32_t vckss_rust_engine_solve_v5(uint64_t generation, const VckssEngineSolveRequestV5 *request);
int32_t vckss_rust_engine_solve_interrupt_v5(uint64_t generation, const VckssEngineSolveRequestInterruptV5 *request);
/* V4 and V8 solves (reference vckss_rust.h:1603-1609, 1945-1950): V4 and
 * later requests must carry the request signature and profile that
 * vckss_rust_backend_request_capability_v3 reports for them. */
int32_t vckss_rust_engine_solve_v4(uint64_t generation, const VckssEngineSolveRequestV4 *request);
int32_t vckss_rust_engine_solve_interrupt_v4(uint64_t generation, const VckssEngineSolveRequestInterruptV4 *request);
int32_t vckss_rust_engine_default_solve_request_v8(VckssEngineSolveRequestV8 *output, uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_default_solve_request_interrupt_v8(VckssEngineSolveRequestInterruptV8 *output,
                                                            uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_solve_v8(uint64_t generation, const VckssEngineSolveRequestV8 *request);
int32_t vckss_rust_engine_solve_interrupt_v8(uint64_t generation, const VckssEngineSolveRequestInterruptV8 *request);
/* Classify a request and compute its signature (reference vckss_rust.h:1661-1665;
 * vckss-plugin/src/ffi_engine.rs:2629-2719, 9304-9532). */
int32_t vckss_rust_backend_request_capability_v3(const VckssBackendRequestCapabilityRequestV3 *request,
                                                 VckssBackendRequestCapabilityReceiptV3 *output,
                                                 uint32_t output_capacity_bytes);
/* Reference vckss_rust.h:2121-2125. */
int32_t vckss_rust_engine_full_cmg_receipt_v1(uint64_t generation, VckssFullCmgReceiptV1 *output,
                                              uint32_t output_capacity_bytes);

/* ---- results and receipts (reference ffi_engine.rs:5992-6040 result_v1; 4370-4470 receipts, retained mask) ---- */
int32_t vckss_rust_engine_result_v1(uint64_t generation, VckssEngineResultV1 *output, uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_preparation_receipt_v1(uint64_t generation, VckssEnginePreparationReceiptV1 *output,
                                                 uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_preparation_receipt_v2(uint64_t generation, VckssEnginePreparationReceiptV2 *output,
                                                 uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_preparation_receipt_v3(uint64_t generation, VckssEnginePreparationReceiptV3 *output,
                                                 uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_preparation_receipt_v4(uint64_t generation, VckssEnginePreparationReceiptV4 *output,
                                                 uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_retained_mask_v1(uint64_t generation, uint8_t *output, uint64_t output_capacity_bytes);
int32_t vckss_rust_engine_rhs_receipts_v1(uint64_t generation, VckssEngineRhsReceiptV1 *output,
                                          uint64_t output_capacity_rows);
int32_t vckss_rust_engine_rhs_receipts_v2(uint64_t generation, VckssEngineRhsReceiptV2 *output,
                                          uint64_t output_capacity_rows);

/* ---- cleanup (reference ffi_engine.rs:7146-7200, 2470) ---- */
int32_t vckss_rust_engine_release_v1(uint64_t generation);
int32_t vckss_rust_engine_clear_abandoned_v1(void);
int32_t vckss_rust_engine_snapshot_v1(VckssEngineSnapshotV1 *output, uint32_t output_capacity_bytes);
const char *vckss_rust_engine_last_error(void);

/* ================= B200 extensions (no reference counterpart) ================= */

/* Device options applied to the next solve of a generation. */
typedef struct FevcbSolveOptionsV1 {
  uint32_t struct_size;
  uint32_t block_columns;   /* right-hand sides per blocked PCG: 0 auto, 2 (one target probe per solve), 8, 16, 32, 64 */
  uint32_t preconditioner;  /* 0 auto, 1 Jacobi, 2 aggregation multigrid, 3 learned (flexible PCG),
                               4 degree-1 polynomial stage with uniform weights z = (a r + s A (s r / d)) / d */
  uint32_t keep_unit_detail;/* 1: keep per-unit leverage arrays for fevcb_engine_unit_detail_v1 */
} FevcbSolveOptionsV1;

/* Prefix-extended options (struct_size 24), accepted by the same entry. */
typedef struct FevcbSolveOptionsV2 {
  FevcbSolveOptionsV1 v1;
  uint32_t precision;       /* 0 double; 1 single-precision residual, direction and products with a double
                               solution, double reductions and double residual replacement; 2 autotuned:
                               the fastest of those forms on the generation's first leverage block
                               (fevcb_engine_tuning_v1) */
  uint32_t reserved;
} FevcbSolveOptionsV2;

/* Wall and device timings of the last solve. */
typedef struct FevcbSolveTimingsV1 {
  uint32_t struct_size;
  uint32_t fallbacks;       /* learned-preconditioner blocks finished by the Jacobi fallback */
  double total_ms;
  double fit_ms;
  double leverage_ms;
  double target_ms;
  double setup_ms;
  uint64_t block_iterations;
  uint64_t column_iterations;
  uint64_t rhs_columns;
  uint64_t kernel_launches;
  uint64_t h2d_bytes;
  uint64_t vertices;
  uint64_t edges;
  uint64_t kept_workers;
  uint64_t levels;
} FevcbSolveTimingsV1;

int32_t fevcb_device_count(void);
/* Bind the CUDA stream (a cudaStream_t) used by generations prepared afterwards; NULL = library-owned stream. */
int32_t fevcb_set_stream(void *stream);
/* Whether the hybrid Laplacian the device assembled for a solved generation
 * (with its row segments and worker reconstruction arrays) equals the host
 * builder's bit for bit: *identical = 1 or 0. */
int32_t fevcb_engine_hybrid_check_v1(uint64_t generation, uint32_t *identical);
/* Device buffers of released generations stay cached (at most 16 GiB per
 * device) for the next generation, and so do the pinned host blocks that
 * stage uploads (at most 8 GiB per process); this returns the current
 * device's cached blocks and the pinned blocks to the driver (freed_bytes
 * counts both).  Either pointer may be NULL. */
int32_t fevcb_device_cache_trim_v1(uint64_t *freed_bytes, uint64_t *cached_bytes);
int32_t fevcb_engine_solve_options_v1(uint64_t generation, const FevcbSolveOptionsV1 *options);
int32_t fevcb_engine_timings_v1(uint64_t generation, FevcbSolveTimingsV1 *output, uint32_t output_capacity_bytes);
/* Re-run the solve of a solved generation with the same request (device-resident inputs). */
int32_t fevcb_engine_resolve_v1(uint64_t generation);
/* Per-unit and per-probe detail of the last solve (units in plan order). Arrays may be NULL. */
int32_t fevcb_engine_unit_detail_v1(uint64_t generation, uint64_t units, double *projection_share,
                                    double *residual_share, double *finite_bias, double *finite_variance,
                                    double *residual_mass, double *deleted_mass, uint64_t cells, double *fitted_cell,
                                    double *cell_correction_weight, uint64_t probes, double *target_draws4);
/* Read-only view of a prepared generation's compressed problem and semantic
 * plan (host arrays owned by the library, valid until release). */
typedef struct FevcbProblemViewV1 {
  uint32_t struct_size;
  uint32_t reserved;
  uint64_t rows, workers, firms, cells, units, strata;
  uint64_t physical_total;
  double target_total;
  const uint32_t *row_worker, *row_firm, *row_cell;
  const double *row_outcome, *row_target;
  const uint64_t *row_frequency;
  const uint32_t *cell_worker, *cell_firm;
  const double *cell_weight, *cell_outcome_sum, *cell_target_sum;
  const uint32_t *unit_cell;
  const uint64_t *unit_count, *unit_rank;
  const double *unit_outcome_sum;
  const uint32_t *stratum_cell;
  const double *stratum_per_copy;
  const uint64_t *stratum_count, *stratum_rank;
  uint64_t controls;                 /* control columns (generic plan) */
  const double *control_values;      /* rows x controls, column-major */
  const uint64_t *group_ptr;         /* generic plan: rows of each deletion unit ... */
  const uint32_t *group_rows;        /* ... in semantic-rank order (observation: class rows in row order) */
  const uint64_t *row_rank;          /* generic plan: semantic rank of every row */
  const uint64_t *row_copy_offset;   /* observation plan: number of the row's first copy in its class */
  uint64_t deletion_mode;            /* VCKSS_DELETION_MATCH or VCKSS_DELETION_OBSERVATION */
} FevcbProblemViewV1;
int32_t fevcb_engine_problem_view_v1(uint64_t generation, FevcbProblemViewV1 *output, uint32_t output_capacity_bytes);

/* The combinatorial aggregation hierarchy of a prepared generation, built on
 * the host only (no GPU needed): the hybrid Laplacian with workers of at most
 * `eliminate_max_degree` cells eliminated (0: the device engine's 16; 4: the
 * reference's rule, whose vertex and edge counts and hierarchy the plugin's
 * VckssFullCmgReceiptV1 reports) and its CMG levels. */
typedef struct FevcbCmgSummaryV1 {
  uint32_t struct_size;
  uint32_t eliminate_max_degree;
  uint64_t vertices;          /* hybrid vertices (firms + kept workers) */
  uint64_t edges;             /* undirected hybrid edges */
  uint64_t hierarchy_levels;
  uint64_t terminal_vertices;
  uint32_t terminal_reason;   /* 1 direct, 2 full contraction, 3 stagnated vertices, 4 fill, 5 level cap */
  uint32_t reserved;
  uint64_t level_vertices[32];
  uint64_t level_edges[32];
  uint32_t level_repeat[32];
} FevcbCmgSummaryV1;
int32_t fevcb_engine_cmg_summary_v1(uint64_t generation, uint32_t eliminate_max_degree, FevcbCmgSummaryV1 *output,
                                    uint32_t output_capacity_bytes);

/* Probe sharding across devices (no counterpart in the reference: its
 * plugin runs on one host).  Every device prepares the same panel; each solves
 * a contiguous range of the request's probes (ranges start on multiples of
 * four, one Counter-V1 block):
 *   1. fevcb_engine_shard_leverage_v1: the fit and the range's leverage probes;
 *      writes the leverage accumulators (fevcb_engine_shard_size_v1 doubles);
 *   2. the caller sums the accumulators over all devices (an all-reduce);
 *   3. fevcb_engine_shard_target_v1: the adjustment from the summed
 *      accumulators and the range's target probes; writes 4 doubles per probe
 *      (worker, firm, covariance, total draws);
 *   4. the caller gathers all probes' draws; fevcb_engine_shard_finish_v1
 *      publishes the components as the generation's result (result_v1).
 * The result equals the single-device solve of the same request.  The
 * accumulator buffers of steps 1 and 3 may be host or device memory (copies
 * use unified addressing), so a device buffer can go straight to a device
 * all-reduce without passing through the host. */
int32_t fevcb_engine_shard_size_v1(uint64_t generation, uint64_t *accumulators);
int32_t fevcb_engine_shard_leverage_v1(uint64_t generation, const VckssEngineSolveRequestV5 *request,
                                       uint32_t probe_begin, uint32_t probe_end, double *accumulators,
                                       uint64_t count);
int32_t fevcb_engine_shard_target_v1(uint64_t generation, const VckssEngineSolveRequestV5 *request,
                                     uint32_t probe_begin, uint32_t probe_end, const double *accumulators,
                                     uint64_t count, double *draws);
int32_t fevcb_engine_shard_finish_v1(uint64_t generation, const VckssEngineSolveRequestV5 *request,
                                     const double *draws);

/* Learned preconditioner (no counterpart in the reference).  A trainer holds
 * training graphs (the hybrid Laplacians of prepared generations) with
 * residual/error pairs that CMG-PCG generates on the device, and trains the
 * graph network with the library's own forward and backward kernels.
 * fevcb_learned_install_v1 makes a parameter vector the network of
 * preconditioner 3 (device solve option) for later solves. */
int32_t fevcb_learned_param_count_v1(uint64_t *count);
int32_t fevcb_learned_initial_params_v1(uint64_t seed, float *params, uint64_t count);
int32_t fevcb_learned_install_v1(const float *params, uint64_t count);
int32_t fevcb_learned_trainer_create_v1(uint64_t seed, uint64_t *handle);
int32_t fevcb_learned_trainer_destroy_v1(uint64_t handle);
int32_t fevcb_learned_trainer_add_panel_v1(uint64_t handle, uint64_t generation, uint32_t columns, uint64_t seed);
int32_t fevcb_learned_trainer_train_v1(uint64_t handle, uint32_t steps, double learning_rate, double *losses);
int32_t fevcb_learned_trainer_gradient_v1(uint64_t handle, uint32_t graph, double *loss, float *gradient,
                                          uint64_t count);
int32_t fevcb_learned_trainer_params_v1(uint64_t handle, float *params, uint64_t count);
int32_t fevcb_learned_trainer_set_params_v1(uint64_t handle, const float *params, uint64_t count);
/* Host copies of one training graph (valid until the next call on the trainer). */
typedef struct FevcbLearnedDumpV1 {
  uint32_t struct_size;
  uint32_t pairs;
  uint64_t vertices;
  const uint32_t *row_ptr, *col;
  const double *weight, *diagonal;
  const float *features;  /* vertices x 8 */
  const float *basis;     /* 4 x vertices x pairs */
  const float *error;     /* vertices x pairs */
  const float *energy;    /* pairs: e' L e */
} FevcbLearnedDumpV1;
int32_t fevcb_learned_trainer_dump_v1(uint64_t handle, uint32_t graph, FevcbLearnedDumpV1 *output,
                                      uint32_t output_capacity_bytes);

/* One CMG forest-aggregation step on a Laplacian given as CSR of positive
 * off-diagonal conductances (both directions, diagonal = row sums), host only:
 * labels[v] is the aggregate of vertex v (first-occurrence numbering). */
int32_t fevcb_cmg_aggregate_v1(uint32_t vertices, const uint32_t *row_ptr, const uint32_t *col, const double *weight,
                               double low_degree_threshold, uint32_t *labels, uint32_t *aggregates);

/* Time standalone launches of one hot kernel of a solved generation with CUDA
 * events, L2 flushed before each launch.  kernel: 1 the persistent blocked
 * PCG form the solver uses at this block width (20 iterations per launch),
 * 3 leverage atoms + cell sums, 4 leverage moments, 5 the three-barrier and
 * 6 the two-barrier persistent PCG, 7 the three-barrier form with per-lane
 * index loads in its gather, 8 the three-barrier form without the pipelined
 * product phase (20 iterations per launch), 9 the single-kernel mixed-precision
 * Jacobi solve and 10 the same with the degree-1 polynomial stage (FP32
 * storage, FP64 residual replacement; 20 iterations per launch, blocks of 32
 * or 64 columns).
 * Outputs the median milliseconds per launch and algorithmic bytes per launch. */
int32_t fevcb_engine_kernel_benchmark_v1(uint64_t generation, uint32_t kernel, uint32_t block_columns,
                                         uint32_t launches, double *ms_per_launch, double *bytes_per_launch);

/* The solver-form autotuner of a generation solved with precision 2 (no
 * counterpart in the reference): the candidates timed on the first leverage
 * block (precision 0/1 and preconditioner 1 Jacobi, 3 learned or 4 uniform
 * degree-1 stage), their milliseconds, and the index of the one kept
 * (-1 before the first such solve). */
typedef struct FevcbTuningV1 {
  uint32_t struct_size;
  int32_t chosen;
  uint32_t candidates;
  uint32_t precision[3];
  uint32_t preconditioner[3];
  uint32_t reserved;
  double milliseconds[3];
} FevcbTuningV1;
int32_t fevcb_engine_tuning_v1(uint64_t generation, FevcbTuningV1 *output, uint32_t output_capacity_bytes);

/* Wall time of the host preparation of a generation, by phase (the split of
 * the reference's preparation timings): ingest copy of the caller's columns,
 * canonical ids and validation (vckss-core/src/problem.rs:102-173), graph
 * fixed point (graph.rs:82-511), compression (problem.rs:194-606) and the
 * JLA plan with semantic ranks (jla.rs:21-790).  threads = host threads the
 * preparation may use. */
typedef struct FevcbPrepareTimingsV1 {
  uint32_t struct_size;
  uint32_t threads;
  double ingest_ms;
  double canonical_ms;
  double graph_ms;
  double compression_ms;
  double plan_ms;
  double total_ms;
} FevcbPrepareTimingsV1;
int32_t fevcb_engine_prepare_timings_v1(uint64_t generation, FevcbPrepareTimingsV1 *output,
                                        uint32_t output_capacity_bytes);

/* Wall milliseconds of the device engine's setup for the generation (built
 * on its first solve): the host builders, each on its own thread with its
 * uploads (cells and firm segments; deletion units; target strata offsets,
 * scales and keys; row data; match groups; then one per control column),
 * their parallel span, the
 * device steps after them (controls transposed, the rows of every cell
 * sorted, the leave-observation-out unit arrays derived), the hybrid
 * Laplacian's assembly, the preconditioner's setup, and the whole setup.
 * Builders a plan does not use report 0.  STALE_CONTEXT before a solve. */
typedef struct FevcbSetupTimingsV1 {
  uint32_t struct_size;
  uint32_t builders;
  double builder_ms[16];
  double builders_span_ms;
  double device_units_ms;
  double hybrid_ms;
  double preconditioner_ms;
  double total_ms;
} FevcbSetupTimingsV1;
int32_t fevcb_engine_setup_timings_v1(uint64_t generation, FevcbSetupTimingsV1 *output,
                                      uint32_t output_capacity_bytes);

/* Independent probe sets on one prepared generation in one call (no
 * counterpart in the reference, which draws one seed per solve): set 0 is the
 * V5 request solved with that set's seed and probe count, and its result
 * becomes the generation's result (engine_result_v1, receipts); each later
 * set runs the leverage and target probes of its own seed and count on the
 * same device generation, keeping set 0's fit (which no seed changes) and
 * the solver form chosen for the generation.  results[i] equals what a
 * separate V5 solve of set i returns.  At most 4096 sets per call. */
typedef struct FevcbProbeSetV1 {
  uint64_t seed;
  uint32_t probes;
  uint32_t reserved;
} FevcbProbeSetV1;
typedef struct FevcbProbeSetResultV1 {
  VckssComponentVectorV1 plugin;
  VckssComponentVectorV1 correction;
  VckssComponentVectorV1 corrected;
  VckssComponentVectorV1 numerical_mcse;
} FevcbProbeSetResultV1;
int32_t fevcb_engine_solve_sets_v1(uint64_t generation, const VckssEngineSolveRequestV5 *request,
                                   const FevcbProbeSetV1 *sets, uint32_t count, FevcbProbeSetResultV1 *results,
                                   uint32_t results_capacity_bytes);

/* The numerical MCSE attachment's covariance algebra on given matrices (no
 * solve; host only): conditional and leverage are row-major 3 x 3 in the
 * order worker, firm, covariance.  Fills status, conditional, leverage, raw,
 * usable, mcse and psd_adjustment of *output as vckss_rust_engine_numerical_
 * result_v1 reports them (reference numerical_mc.rs:234-354 `finalize`); the
 * replay fields stay zero. */
int32_t fevcb_numerical_finalize_v1(const double *conditional, const double *leverage,
                                    VckssNumericalResultV1 *output, uint32_t output_capacity_bytes);

/* Ceiling on the identified dimension (W + F - 1) of an exact-estimator solve
 * of this generation (no counterpart in the reference, whose dense estimator
 * refuses limits above 2,000: vckss-core/src/exact_estimator.rs:104-108).
 * The device computes exact leverages by blocked solves instead of a dense
 * inverse, so panels such as 20,000 workers x 1,000 firms (about 8,000
 * parameters) fit.  0 restores the request's own limit; at most 1,000,000. */
int32_t fevcb_engine_exact_limit_v1(uint64_t generation, uint64_t ceiling);

/* Counter-V1 atoms computed on the device: out[e*columns + j] for probe first_probe + j. */
int32_t fevcb_counter_atoms_v1(uint64_t seed, uint64_t domain_tag, uint64_t first_probe, uint32_t columns,
                               const uint64_t *entity, const uint64_t *trials, uint64_t count, int64_t *out);

/* Same result as fevcb_counter_atoms_v1, for callers that cannot allocate
 * device memory (no counterpart in the reference): a process whose own
 * framework already holds nearly all device memory, or one that fixes its
 * device-memory plan at start-up.  Inputs and outputs stay host arrays; the
 * call stages them in one file-scope 8 MiB device array instead of allocating,
 * so it calls no cudaMalloc/cudaFree.  Requests needing more than 8 MiB
 * (2 x count x 8 bytes + count x columns x 8 bytes, each part rounded up to
 * 256 bytes) are refused with RESOURCE_LIMIT (40); without a visible device
 * the call returns UNSUPPORTED_FEATURE (11), as fevcb_counter_atoms_v1 does.
 * The copies and the kernel run on the stream bound by fevcb_set_stream (the
 * legacy default stream when none is bound) and the call returns after that
 * stream has finished them.  The first call on a device looks up the array's
 * device address and keeps it for the life of the process: make that first
 * call before any stream capture, and do not call again on a device after
 * cudaDeviceReset.  Every call shares the array: calls that overlap on the GPU
 * race and must be serialised by the caller. */
int32_t fevcb_counter_atoms_noalloc_v1(uint64_t seed, uint64_t domain_tag, uint64_t first_probe, uint32_t columns,
                                       const uint64_t *entity, const uint64_t *trials, uint64_t count, int64_t *out);


/* Detailed receipts V1-V7 (vckss_rust.h:1084-1439): the same layouts; the fields
 * this engine fills are listed at fevcb::fill_detailed_receipt (abi.cpp). */
typedef struct VckssEngineDetailedReceiptV1 {
  uint32_t struct_size;
  uint32_t reserved;
  uint64_t generation;
  uint64_t seed;
  uint32_t probes_requested;
  uint32_t leverage_probes_accepted;
  uint32_t target_probes_accepted;
  uint32_t solver_requested;
  uint32_t solver_selected;
  uint32_t solver_fallback;
  int32_t solver_fallback_error;
  uint64_t solver_dimension;
  uint64_t leverage_batch_width;
  uint64_t target_batch_width;
  double rank_tolerance;
  double block_tolerance;
  double full_residual_tolerance;
  uint32_t full_fit_route;
  uint32_t full_fit_iterations;
  double full_fit_reduced_residual;
  double full_fit_complete_residual;
  uint32_t full_fit_zero_rhs;
  uint32_t reserved_1;
  uint64_t leverage_rhs_count;
  uint64_t target_rhs_count;
  double max_reduced_residual;
  double max_complete_residual;
  double max_leverage;
  double max_reciprocal_residual;
  double accounting_residual;
  uint64_t topology_checksum;
  uint64_t cmg_levels;
  uint64_t cmg_fine_vertices;
  uint64_t cmg_fine_edges;
  uint64_t cmg_terminal_vertices;
  double cmg_edge_complexity;
  double cmg_vertex_complexity;
  uint64_t cmg_structural_bytes;
  uint64_t cmg_workspace_bytes;
  uint64_t cmg_dense_factor_bytes;
} VckssEngineDetailedReceiptV1;

typedef struct VckssEngineDetailedReceiptV2 {
  uint32_t struct_size;
  uint32_t reserved;
  uint64_t generation;
  uint64_t seed;
  uint32_t probes_requested;
  uint32_t leverage_probes_accepted;
  uint32_t target_probes_accepted;
  uint32_t solver_requested;
  uint32_t solver_selected;
  uint32_t solver_fallback;
  int32_t solver_fallback_error;
  uint64_t solver_dimension;
  uint64_t leverage_batch_width;
  uint64_t target_batch_width;
  double rank_tolerance;
  double block_tolerance;
  double full_residual_tolerance;
  uint32_t full_fit_route;
  uint32_t full_fit_iterations;
  double full_fit_reduced_residual;
  double full_fit_complete_residual;
  uint32_t full_fit_zero_rhs;
  uint32_t reserved_1;
  uint64_t leverage_rhs_count;
  uint64_t target_rhs_count;
  double max_reduced_residual;
  double max_complete_residual;
  double max_leverage;
  double max_reciprocal_residual;
  double accounting_residual;
  uint64_t topology_checksum;
  uint64_t cmg_levels;
  uint64_t cmg_fine_vertices;
  uint64_t cmg_fine_edges;
  uint64_t cmg_terminal_vertices;
  double cmg_edge_complexity;
  double cmg_vertex_complexity;
  uint64_t cmg_structural_bytes;
  uint64_t cmg_workspace_bytes;
  uint64_t cmg_dense_factor_bytes;
  double full_fit_weighted_rss;
  uint64_t memory_limit_bytes;
  uint64_t caller_copy_bytes;
  uint64_t preparation_peak_forecast_bytes;
  uint64_t prepared_resident_bytes;
  uint64_t solver_setup_forecast_bytes;
  uint64_t leverage_phase_forecast_bytes;
  uint64_t target_phase_forecast_bytes;
  uint64_t result_forecast_bytes;
  uint64_t solve_peak_forecast_bytes;
  uint64_t command_peak_forecast_bytes;
} VckssEngineDetailedReceiptV2;

typedef struct VckssEngineDetailedReceiptV3 {
  VckssEngineDetailedReceiptV2 v2;
  uint32_t rng_contract;
  uint32_t reserved_2;
  uint64_t rhs_receipt_rows;
  uint64_t caller_result_copy_bytes;
} VckssEngineDetailedReceiptV3;

typedef struct VckssEngineDetailedReceiptV4 {
  VckssEngineDetailedReceiptV3 v3;
  uint32_t algorithm_requested;
  uint32_t algorithm_selected;
  uint32_t deletion_mode;
  uint32_t nuisance_mode;
  uint64_t parameters;
  uint64_t full_parameters;
  uint64_t correction_parameters;
  double information_rcond;
  double inverse_relres;
  uint64_t exact_peak_forecast_bytes;
} VckssEngineDetailedReceiptV4;

typedef struct VckssEngineDetailedReceiptV5 {
  VckssEngineDetailedReceiptV4 v4;
  uint64_t applicability_flags;
  double working_fit_complete_residual;
  double inverse_sqrt_relres;
  double maker_relres;
  double control_basis_relres;
  double control_basis_forward_error;
  double deletion_rank_gap;
  double firm_zero_sum_residual;
  uint64_t fit_peak_forecast_bytes;
  uint64_t correction_peak_forecast_bytes;
  double actual_accounting_residual;
} VckssEngineDetailedReceiptV5;

typedef struct VckssEngineDetailedReceiptV6 {
  VckssEngineDetailedReceiptV5 v5;
  uint32_t engine_requested;
  uint32_t engine_selected;
  uint64_t generic_applicability_flags;
  uint32_t controls_count;
  uint32_t rhs_receipt_schema;
  uint64_t control_projection_rhs_count;
  double control_rank_rcond;
  double control_rank_smallest_generalized_eigenvalue_lower;
  double control_rank_largest_generalized_eigenvalue_upper;
  double control_rank_projection_error_bound;
  double control_rank_normalization_error_bound;
  double control_rank_fe_information_eigenvalue_lower_bound;
  double control_rank_maximum_projection_residual;
  double control_rank_effective_tolerance;
  double control_rank_projection_pcg_tolerance;
  double control_rank_projection_residual_gate;
  double generic_control_basis_relres;
  double generic_control_basis_forward_error;
  double generic_control_schur_rcond;
  double generic_control_schur_relres;
  double generic_deletion_rank_gap;
  double full_joint_fit_complete_residual;
  double generic_working_fit_complete_residual;
  double generic_maker_relres;
  uint64_t canonicalization_peak_forecast_bytes;
  uint64_t generic_fit_peak_forecast_bytes;
  uint64_t geometry_peak_forecast_bytes;
  uint64_t generic_leverage_peak_forecast_bytes;
  uint64_t generic_target_peak_forecast_bytes;
  uint64_t maker_peak_forecast_bytes;
  uint64_t generic_result_forecast_bytes;
  uint64_t generic_peak_forecast_bytes;
  uint64_t rhs_v2_caller_copy_bytes;
  uint32_t capability_schema;
  uint32_t capability_profile;
  uint32_t batch_mode;
  uint32_t stayers_mode;
  uint32_t target_weight_mode;
  uint32_t deletion_unit_source;
  uint32_t probeorder_supplied;
  uint32_t wallseconds_supplied;
  uint32_t frequency_use;
  uint32_t reserved_6;
  uint64_t physical_limit;
  uint64_t request_signature;
} VckssEngineDetailedReceiptV6;

typedef struct VckssEstimatorResolutionReceiptV1 {
  uint32_t algorithm_schema;
  uint32_t algorithm_requested;
  uint32_t algorithm_selected;
  uint32_t algorithm_reason;
  uint32_t engine_schema;
  uint32_t engine_requested;
  uint32_t engine_selected;
  uint32_t engine_reason;
  uint32_t compressed_eligibility;
  uint32_t resolved_before_rng;
  uint32_t opportunistic_engine_fallback_allowed;
  uint32_t reserved;
  uint64_t identified_complexity;
  uint64_t exact_limit;
  uint64_t rng_draws_before_resolution;
  uint64_t counter_atoms_before_resolution;
} VckssEstimatorResolutionReceiptV1;

typedef struct VckssSolverExecutionReceiptV1 {
  uint32_t schema_version;
  uint32_t requested_route;
  uint32_t selected_route;
  uint32_t fallback_used;
  int32_t fallback_error;
  uint32_t full_setup_complete;
  uint32_t fe_setup_complete;
  uint32_t fe_hierarchy_reused;
  uint32_t plan_frozen_before_rng;
  uint32_t auto_route_contract;
  uint32_t threads_requested;
  uint32_t threads_used;
  uint32_t parallel_regions;
  uint32_t applicability;
  uint32_t reserved_1;
  uint32_t reserved_2;
  uint64_t planned_rhs;
  uint64_t auto_firm_threshold;
  uint64_t auto_rhs_threshold;
  uint64_t full_solver_dimension;
  uint64_t fe_solver_dimension;
  uint64_t logical_atoms_before_plan_freeze;
  uint64_t unique_words_before_plan_freeze;
  uint64_t physical_trials_before_plan_freeze;
} VckssSolverExecutionReceiptV1;

typedef struct VckssBatchPhasePlanReceiptV1 {
  uint32_t request_mode;
  uint32_t selection_reason;
  uint32_t applicability;
  uint32_t reserved;
  uint64_t requested_width;
  uint64_t selected_width;
  uint64_t probe_width_cap;
  uint64_t declared_threads;
  uint64_t thread_width_cap;
  uint64_t route_width_cap;
  uint64_t effective_width_cap;
  uint64_t hard_memory_bytes;
  uint64_t width_one_forecast_bytes;
  uint64_t selected_forecast_bytes;
} VckssBatchPhasePlanReceiptV1;

typedef struct VckssBatchExecutionReceiptV1 {
  uint32_t schema_version;
  uint32_t deterministic;
  uint32_t width_invariance_required;
  uint32_t arithmetic_contract;
  uint32_t whole_command_admitted;
  uint32_t applicability;
  uint64_t non_batched_peak_bytes;
  uint64_t selected_command_peak_bytes;
  VckssBatchPhasePlanReceiptV1 leverage;
  VckssBatchPhasePlanReceiptV1 target;
} VckssBatchExecutionReceiptV1;

typedef struct VckssWallExecutionReceiptV1 {
  uint32_t schema_version;
  uint32_t model_code;
  uint32_t status;
  uint32_t routing_effect;
  uint32_t requested_applicable;
  uint32_t forecast_applicable;
  uint32_t advisory_applicable;
  uint32_t margin_applicable;
  double requested_seconds;
  double forecast_seconds;
  double advisory_seconds;
  double advisory_margin_fraction;
  uint64_t preparation_work;
  uint64_t engine_setup_work;
  uint64_t full_fit_work;
  uint64_t leverage_work;
  uint64_t target_work;
  uint64_t result_export_work;
  uint64_t total_work;
} VckssWallExecutionReceiptV1;

typedef struct VckssCounterPhaseExecutionReceiptV1 {
  uint64_t planned_logical_atoms;
  uint64_t actual_logical_atoms;
  uint64_t planned_unique_packed_words;
  uint64_t actual_unique_packed_words;
  uint64_t planned_physical_trials;
  uint64_t actual_physical_trials;
  uint64_t planned_generator_work;
  uint64_t actual_generator_work;
} VckssCounterPhaseExecutionReceiptV1;

typedef struct VckssCounterExecutionReceiptV1 {
  uint32_t schema_version;
  uint32_t rng_contract;
  uint32_t generator_work_applicable;
  uint32_t completed;
  VckssCounterPhaseExecutionReceiptV1 leverage;
  VckssCounterPhaseExecutionReceiptV1 target;
  VckssCounterPhaseExecutionReceiptV1 total;
  uint64_t logical_atoms_before_plan_freeze;
  uint64_t unique_words_before_plan_freeze;
  uint64_t physical_trials_before_plan_freeze;
} VckssCounterExecutionReceiptV1;

typedef struct VckssExecutionMemoryReceiptV1 {
  uint32_t schema_version;
  uint32_t applicability;
  uint32_t peak_phase;
  uint32_t reserved;
  uint64_t hard_limit_bytes;
  uint64_t prepared_persistent_bytes;
  uint64_t setup_peak_bytes;
  uint64_t fit_peak_bytes;
  uint64_t correction_peak_bytes;
  uint64_t leverage_peak_bytes;
  uint64_t target_peak_bytes;
  uint64_t result_peak_bytes;
  uint64_t non_batched_peak_bytes;
  uint64_t command_peak_bytes;
  uint64_t shared_cmg_persistent_bytes;
  uint64_t full_control_block_persistent_bytes;
  uint64_t setup_transient_bytes;
  uint64_t cmg_preconditioner_workspace_bytes;
  uint64_t cmg_aggregated_cell_capacity_bytes;
  uint64_t cmg_group_index_bytes;
  uint64_t cmg_hybrid_graph_bytes;
  uint64_t retained_nq_bytes;
  uint64_t retained_q2_bytes;
} VckssExecutionMemoryReceiptV1;

typedef struct VckssExecutionPlanReceiptV1 {
  uint32_t struct_size;
  uint32_t schema_version;
  uint64_t generation;
  uint64_t applicability_flags;
  uint64_t contract_flags;
  uint64_t request_signature;
  VckssEstimatorResolutionReceiptV1 resolution;
  VckssSolverExecutionReceiptV1 solver;
  VckssBatchExecutionReceiptV1 batch;
  VckssWallExecutionReceiptV1 wall;
  VckssCounterExecutionReceiptV1 counter;
  VckssExecutionMemoryReceiptV1 memory;
} VckssExecutionPlanReceiptV1;

typedef struct VckssEngineDetailedReceiptV7 {
  VckssEngineDetailedReceiptV6 v6;
  VckssExecutionPlanReceiptV1 execution;
} VckssEngineDetailedReceiptV7;

/* Detailed receipts of the last solve (vckss_rust.h:2093-2116).  V1 needs a
 * no-control match solve; V7 a V5 or V8 solve (its execution plan).  Fields
 * of the reference's CPU memory and thread model this engine has no
 * counterpart for are zero. */
int32_t vckss_rust_engine_detailed_receipt_v1(uint64_t generation, VckssEngineDetailedReceiptV1 *output,
                                              uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_detailed_receipt_v2(uint64_t generation, VckssEngineDetailedReceiptV2 *output,
                                              uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_detailed_receipt_v3(uint64_t generation, VckssEngineDetailedReceiptV3 *output,
                                              uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_detailed_receipt_v4(uint64_t generation, VckssEngineDetailedReceiptV4 *output,
                                              uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_detailed_receipt_v5(uint64_t generation, VckssEngineDetailedReceiptV5 *output,
                                              uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_detailed_receipt_v6(uint64_t generation, VckssEngineDetailedReceiptV6 *output,
                                              uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_detailed_receipt_v7(uint64_t generation, VckssEngineDetailedReceiptV7 *output,
                                              uint32_t output_capacity_bytes);

/* ---------------------------------------------------------------------------
 * Fixed-effect projection attachment (reference vckss_rust.h:400-427,
 * 798-838, 1721, 1820-1829, 1983-1998; ffi_engine.rs:2413-2418, 3679-3835,
 * 6030-6110).  A prepared generation whose solve runs the generic JLA engine
 * (controls, or leave-observation-out) takes one projection of a worker or
 * firm effect on caller covariates (plus the automatic constant): the host
 * builds the coefficient-space loadings at augmentation; the solve runs the
 * loadings' model solves on the GPU after the target phase and streams the
 * KSS covariance over the deletion units.  At most 31 covariates (32
 * columns with the constant) on the device. */
#define VCKSS_PROJECTION_EFFECT_WORKER 1u
#define VCKSS_PROJECTION_EFFECT_FIRM 2u
#define VCKSS_PROJECTION_WEIGHT_FREQUENCY 1u
#define VCKSS_PROJECTION_WEIGHT_TARGET 2u
#define VCKSS_PROJECTION_SCHEMA_V1 1u

typedef struct VckssProjectionAugmentationRequestV1 {
  uint32_t abi_version;
  uint32_t struct_size;
  uint64_t rows;
  uint32_t project_count;
  uint32_t effect;
  uint32_t weight;
  uint32_t reserved;
  double rank_tolerance;
  uint64_t caller_copy_bytes;
} VckssProjectionAugmentationRequestV1;

typedef struct VckssProjectionAugmentationRequestInterruptV1 {
  VckssProjectionAugmentationRequestV1 options;
  VckssInterruptPollV1 interrupt_poll;
  void *interrupt_context;
  uint32_t checkpoint_interval;
  uint32_t reserved;
} VckssProjectionAugmentationRequestInterruptV1;

typedef struct VckssProjectionColumnsV1 {
  uint32_t struct_size;
  uint32_t reserved;
  uint64_t rows;
  const double *const *project;
  uint32_t project_count;
  uint32_t reserved_2;
} VckssProjectionColumnsV1;

typedef struct VckssProjectionAugmentationReceiptV1 {
  uint32_t struct_size;
  uint32_t schema_version;
  uint64_t generation;
  uint64_t rows;
  uint64_t columns;
  uint32_t effect;
  uint32_t weight;
  uint64_t caller_copy_bytes;
  uint64_t augmentation_peak_forecast_bytes;
  uint64_t projection_persistent_bytes;
  uint64_t total_prepared_resident_bytes;
  double gram_rcond;
  double gram_relres;
  double gram_original_relres;
} VckssProjectionAugmentationReceiptV1;

typedef struct VckssProjectionResultReceiptV1 {
  uint32_t struct_size;
  uint32_t schema_version;
  uint64_t generation;
  uint64_t columns;
  uint32_t effect;
  uint32_t weight;
  double gram_rcond;
  double gram_relres;
  double gram_original_relres;
  double covariance_smallest_eigenvalue;
  double covariance_largest_eigenvalue;
  double psd_cleanup;
  double proxy_minimum;
  double proxy_maximum;
  uint32_t maximum_iterations;
  uint32_t reserved;
  double maximum_reduced_residual;
  double maximum_complete_residual;
  double full_residual_tolerance;
  uint64_t projection_peak_forecast_bytes;
  uint64_t persistent_bytes;
  uint64_t result_bytes;
} VckssProjectionResultReceiptV1;

#if defined(__cplusplus)
static_assert(sizeof(VckssProjectionAugmentationRequestV1) == 48, "projection augmentation request size");
static_assert(sizeof(VckssProjectionAugmentationRequestInterruptV1) == 72, "interrupt projection request size");
static_assert(sizeof(VckssProjectionColumnsV1) == 32, "projection column descriptor size");
static_assert(sizeof(VckssProjectionAugmentationReceiptV1) == 96, "projection augmentation receipt size");
static_assert(sizeof(VckssProjectionResultReceiptV1) == 152, "projection result receipt size");
#endif

/* 1: Mean-centred projection covariance is available. */
uint32_t vckss_rust_projection_centering_schema_v1(void);
/* Defaults: worker effect, frequency weight, rank tolerance 1e-10. */
int32_t vckss_rust_engine_default_projection_augmentation_request_interrupt_v1(
    VckssProjectionAugmentationRequestInterruptV1 *output, uint32_t output_capacity_bytes);
/* Attach to a prepared (unsolved) generation: columns copied synchronously;
 * INVALID_INPUT for malformed requests or nonfinite columns, SINGULAR_INFORMATION
 * for an unidentified covariate Gram, CONTEXT_POISONED for a second projection. */
int32_t vckss_rust_engine_augment_projection_interrupt_v1(uint64_t generation,
                                                           const VckssProjectionAugmentationRequestInterruptV1 *request,
                                                           const VckssProjectionColumnsV1 *columns);
int32_t vckss_rust_engine_projection_augmentation_receipt_v1(uint64_t generation,
                                                             VckssProjectionAugmentationReceiptV1 *output,
                                                             uint32_t output_capacity_bytes);
/* After a solve: the columns' coefficients, the KSS covariance (PSD-cleaned)
 * and the naive covariance, each columns x columns row-major. */
int32_t vckss_rust_engine_projection_result_v1(uint64_t generation, double *coefficients,
                                               uint64_t coefficients_capacity, double *covariance,
                                               uint64_t covariance_capacity, double *naive_covariance,
                                               uint64_t naive_covariance_capacity,
                                               VckssProjectionResultReceiptV1 *output, uint32_t output_capacity_bytes);
int32_t vckss_rust_engine_projection_result_receipt_v1(uint64_t generation, VckssProjectionResultReceiptV1 *output,
                                                       uint32_t output_capacity_bytes);

/* ---------------------------------------------------------------------------
 * The rest of the reference ABI (rust/stata_backend/include/vckss_rust.h).
 * These entry points sit outside the solve path this library replaces: the
 * schema probes report what is available (centering 1; exact execution and
 * component inference 0, i.e. absent), session
 * last-error text is the engine's, and every other call returns
 * VCKSS_UNSUPPORTED_FEATURE (11) with its name in the last-error text.
 * Their argument structs are only passed through, so they are declared
 * incomplete here. */
typedef struct VckssColumnsV1 VckssColumnsV1;
typedef struct VckssComponentBatchReceiptV1 VckssComponentBatchReceiptV1;
typedef struct VckssComponentInferenceAugmentationReceiptV1 VckssComponentInferenceAugmentationReceiptV1;
typedef struct VckssComponentInferenceAugmentationRequestInterruptV1 VckssComponentInferenceAugmentationRequestInterruptV1;
typedef struct VckssComponentInferenceResultReceiptV2 VckssComponentInferenceResultReceiptV2;
typedef struct VckssComponentInferenceResultReceiptV3 VckssComponentInferenceResultReceiptV3;
typedef struct VckssComponentInferenceResultReceiptV4 VckssComponentInferenceResultReceiptV4;
typedef struct VckssComponentInferenceResultReceiptV5 VckssComponentInferenceResultReceiptV5;
typedef struct VckssComponentInferenceUnitReceiptV1 VckssComponentInferenceUnitReceiptV1;
typedef struct VckssComponentInferenceUnitReceiptV2 VckssComponentInferenceUnitReceiptV2;
typedef struct VckssEnginePerformanceReceiptV1 VckssEnginePerformanceReceiptV1;
typedef struct VckssEngineSolveRequestInterruptV2 VckssEngineSolveRequestInterruptV2;
typedef struct VckssEngineSolveRequestInterruptV3 VckssEngineSolveRequestInterruptV3;
typedef struct VckssEngineSolveRequestInterruptV6 VckssEngineSolveRequestInterruptV6;
typedef struct VckssEngineSolveRequestInterruptV7 VckssEngineSolveRequestInterruptV7;
typedef struct VckssExactExecutionReceiptV1 VckssExactExecutionReceiptV1;
typedef struct VckssExactExecutionRequestInterruptV1 VckssExactExecutionRequestInterruptV1;
typedef struct VckssExactExecutionRequestV1 VckssExactExecutionRequestV1;
typedef struct VckssExecutionPlanReceiptV1 VckssExecutionPlanReceiptV1;
typedef struct VckssFullCmgModelReceiptV1 VckssFullCmgModelReceiptV1;
typedef struct VckssGenericExecutionReceiptV1 VckssGenericExecutionReceiptV1;
typedef struct VckssGenericExecutionReceiptV2 VckssGenericExecutionReceiptV2;
typedef struct VckssLeaveoutResidualDiagnosticV1 VckssLeaveoutResidualDiagnosticV1;
typedef struct VckssMemoryForecastV1 VckssMemoryForecastV1;
typedef struct VckssMemoryPolicyV1 VckssMemoryPolicyV1;
typedef struct VckssPreparationReceiptV1 VckssPreparationReceiptV1;
typedef struct VckssPrepareRequestV1 VckssPrepareRequestV1;
typedef int32_t (*VckssProgressOperationV1)(void *);
typedef struct VckssProgressOptionsV1 VckssProgressOptionsV1;
typedef struct VckssRepeatMeasurementDiagnosticV1 VckssRepeatMeasurementDiagnosticV1;
typedef struct VckssRepeatMeasurementLeadingV1 VckssRepeatMeasurementLeadingV1;
typedef struct VckssSessionSnapshotV1 VckssSessionSnapshotV1;
typedef struct VckssStayerAugmentationColumnsV1 VckssStayerAugmentationColumnsV1;
typedef struct VckssStayerAugmentationReceiptV1 VckssStayerAugmentationReceiptV1;
typedef struct VckssStayerAugmentationRequestInterruptV1 VckssStayerAugmentationRequestInterruptV1;
typedef struct VckssStayerAugmentationRequestV1 VckssStayerAugmentationRequestV1;
typedef struct VckssStayerHybridResultV1 VckssStayerHybridResultV1;

/* vckss_rust.h:1651 */
int32_t vckss_rust_backend_request_capability_v1(const VckssBackendRequestCapabilityRequestV1 *request, VckssBackendRequestCapabilityReceiptV1 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:1656 */
int32_t vckss_rust_backend_request_capability_v2(const VckssBackendRequestCapabilityRequestV2 *request, VckssBackendRequestCapabilityReceiptV2 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:12 */
uint32_t vckss_rust_centering_schema_v1(void);
/* vckss_rust.h:1864 */
uint32_t vckss_rust_component_inference_interface_version(void);
/* vckss_rust.h:2311 */
int32_t vckss_rust_engine_admit_prepare_memory_v1(const VckssEnginePrepareRequestV4 *, const VckssMemoryPolicyV1 *, uint32_t);
/* vckss_rust.h:1761 */
int32_t vckss_rust_engine_admit_prepare_probe_order_v1(const VckssEnginePrepareRequestV3 *request, uint32_t probeorder_supplied);
/* vckss_rust.h:1755 */
int32_t vckss_rust_engine_admit_prepare_v2(const VckssEnginePrepareRequestV2 *request);
/* vckss_rust.h:1758 */
int32_t vckss_rust_engine_admit_prepare_v3(const VckssEnginePrepareRequestV3 *request);
/* vckss_rust.h:1765 */
int32_t vckss_rust_engine_admit_prepare_v4(const VckssEnginePrepareRequestV4 *request, uint32_t probeorder_supplied);
/* vckss_rust.h:1830 */
int32_t vckss_rust_engine_augment_component_inference_interrupt_v1(uint64_t generation, const VckssComponentInferenceAugmentationRequestInterruptV1 *request);
/* vckss_rust.h:1865 */
int32_t vckss_rust_engine_augment_component_inference_interrupt_v2(uint64_t generation, const VckssComponentInferenceAugmentationRequestInterruptV1 *request);
/* vckss_rust.h:1874 */
int32_t vckss_rust_engine_augment_component_inference_interrupt_v3(uint64_t generation, const VckssComponentInferenceAugmentationRequestInterruptV1 *request);
/* vckss_rust.h:1883 */
int32_t vckss_rust_engine_augment_component_inference_interrupt_v4(uint64_t generation, const VckssComponentInferenceAugmentationRequestInterruptV1 *request, uint32_t gram_probes);
/* vckss_rust.h:1893 */
int32_t vckss_rust_engine_augment_component_inference_interrupt_v5(uint64_t generation, const VckssComponentInferenceAugmentationRequestInterruptV1 *request, uint32_t gram_probes);
/* vckss_rust.h:1834 */
int32_t vckss_rust_engine_augment_match_component_inference_interrupt_v1(uint64_t generation, const VckssComponentInferenceAugmentationRequestInterruptV1 *request);
/* vckss_rust.h:1869 */
int32_t vckss_rust_engine_augment_match_component_inference_interrupt_v2(uint64_t generation, const VckssComponentInferenceAugmentationRequestInterruptV1 *request);
/* vckss_rust.h:1878 */
int32_t vckss_rust_engine_augment_match_component_inference_interrupt_v3(uint64_t generation, const VckssComponentInferenceAugmentationRequestInterruptV1 *request);
/* vckss_rust.h:1888 */
int32_t vckss_rust_engine_augment_match_component_inference_interrupt_v4(uint64_t generation, const VckssComponentInferenceAugmentationRequestInterruptV1 *request, uint32_t gram_probes);
/* vckss_rust.h:1898 */
int32_t vckss_rust_engine_augment_match_component_inference_interrupt_v5(uint64_t generation, const VckssComponentInferenceAugmentationRequestInterruptV1 *request, uint32_t gram_probes);
/* vckss_rust.h:1810 */
int32_t vckss_rust_engine_augment_stayers_interrupt_v1(uint64_t generation, const VckssStayerAugmentationRequestInterruptV1 *request, const VckssStayerAugmentationColumnsV1 *columns);
/* vckss_rust.h:1805 */
int32_t vckss_rust_engine_augment_stayers_v1(uint64_t generation, const VckssStayerAugmentationRequestV1 *request, const VckssStayerAugmentationColumnsV1 *columns);
/* vckss_rust.h:1599 */
int32_t vckss_rust_engine_component_batch_receipt_v1(uint64_t generation, VckssComponentBatchReceiptV1 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:1903 */
int32_t vckss_rust_engine_component_inference_augmentation_receipt_v1(uint64_t generation, VckssComponentInferenceAugmentationReceiptV1 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:1999 */
int32_t vckss_rust_engine_component_inference_result_v2(uint64_t generation, double *primitive_covariance, uint64_t primitive_covariance_capacity, double *covariance, uint64_t covariance_capacity, double *trace_mcse, uint64_t trace_mcse_capacity, double *spectrum, uint64_t spectrum_capacity, double *q1, uint64_t q1_capacity, double *variance_summary, uint64_t variance_summary_capacity, double *fold_diagnostics, uint64_t fold_diagnostics_capacity, double *cv_diagnostics, uint64_t cv_diagnostics_capacity, VckssComponentInferenceResultReceiptV2 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:2020 */
int32_t vckss_rust_engine_component_inference_result_v3(uint64_t generation, double *primitive_covariance, uint64_t primitive_covariance_capacity, double *covariance, uint64_t covariance_capacity, double *trace_mcse, uint64_t trace_mcse_capacity, double *spectrum, uint64_t spectrum_capacity, double *q1, uint64_t q1_capacity, double *variance_summary, uint64_t variance_summary_capacity, double *fold_diagnostics, uint64_t fold_diagnostics_capacity, double *cv_diagnostics, uint64_t cv_diagnostics_capacity, VckssComponentInferenceResultReceiptV3 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:2041 */
int32_t vckss_rust_engine_component_inference_result_v4(uint64_t generation, double *primitive_covariance, uint64_t primitive_covariance_capacity, double *covariance, uint64_t covariance_capacity, double *trace_mcse, uint64_t trace_mcse_capacity, double *spectrum, uint64_t spectrum_capacity, double *q1, uint64_t q1_capacity, double *variance_summary, uint64_t variance_summary_capacity, double *fold_diagnostics, uint64_t fold_diagnostics_capacity, double *cv_diagnostics, uint64_t cv_diagnostics_capacity, VckssComponentInferenceResultReceiptV4 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:2062 */
int32_t vckss_rust_engine_component_inference_result_v5(uint64_t generation, double *primitive, uint64_t primitive_capacity, double *covariance, uint64_t covariance_capacity, double *mcse, uint64_t mcse_capacity, double *spectrum, uint64_t spectrum_capacity, double *q1, uint64_t q1_capacity, double *summaries, uint64_t summaries_capacity, double *folds, uint64_t folds_capacity, double *cv, uint64_t cv_capacity, double *targets, uint64_t targets_capacity, VckssComponentInferenceResultReceiptV5 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:1838 */
int32_t vckss_rust_engine_component_inference_unit_receipt_v1(uint64_t generation, VckssComponentInferenceUnitReceiptV1 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:1843 */
int32_t vckss_rust_engine_component_inference_unit_receipt_v2(uint64_t generation, VckssComponentInferenceUnitReceiptV2 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:1725 */
int32_t vckss_rust_engine_default_component_inference_augmentation_request_interrupt_v1(VckssComponentInferenceAugmentationRequestInterruptV1 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:1733 */
int32_t vckss_rust_engine_default_solve_request_interrupt_v2(VckssEngineSolveRequestInterruptV2 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:1737 */
int32_t vckss_rust_engine_default_solve_request_interrupt_v3(VckssEngineSolveRequestInterruptV3 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:1741 */
int32_t vckss_rust_engine_default_solve_request_interrupt_v4(VckssEngineSolveRequestInterruptV4 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:1586 */
int32_t vckss_rust_engine_default_solve_request_interrupt_v6(VckssEngineSolveRequestInterruptV6 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:1595 */
int32_t vckss_rust_engine_default_solve_request_interrupt_v7(VckssEngineSolveRequestInterruptV7 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:1584 */
int32_t vckss_rust_engine_default_solve_request_v6(VckssEngineSolveRequestV6 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:1717 */
int32_t vckss_rust_engine_default_stayer_augmentation_request_interrupt_v1(VckssStayerAugmentationRequestInterruptV1 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:707 */
int32_t vckss_rust_engine_exact_execution_receipt_v1(uint64_t generation, VckssExactExecutionReceiptV1 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:2106 */
int32_t vckss_rust_engine_execution_plan_receipt_v1(uint64_t generation, VckssExecutionPlanReceiptV1 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:1524 */
int32_t vckss_rust_engine_full_cmg_model_receipt_v1(uint64_t generation, VckssFullCmgModelReceiptV1 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:1592 */
int32_t vckss_rust_engine_generic_execution_receipt_v1(uint64_t generation, VckssGenericExecutionReceiptV1 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:1564 */
int32_t vckss_rust_engine_generic_execution_receipt_v2(uint64_t, VckssGenericExecutionReceiptV2 *, uint32_t);
/* vckss_rust.h:1848 */
int32_t vckss_rust_engine_leaveout_residual_diagnostic_v1(uint64_t generation, VckssLeaveoutResidualDiagnosticV1 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:2332 */
int32_t vckss_rust_engine_memory_forecast_v1(uint64_t, VckssMemoryForecastV1 *, uint32_t);
/* vckss_rust.h:2316 */
int32_t vckss_rust_engine_memory_policy_v1(uint64_t, VckssMemoryPolicyV1 *, uint32_t);
/* vckss_rust.h:2381 */
int32_t vckss_rust_engine_numerical_cmg_work_v1(uint64_t, VckssFullCmgModelReceiptV1 *, uint32_t);
/* vckss_rust.h:2376 */
int32_t vckss_rust_engine_numerical_preflight_v1(const VckssNumericalRequestV1 *);
/* vckss_rust.h:2355 */
int32_t vckss_rust_engine_numerical_preflight_v2(const VckssNumericalRequestV2 *);
/* vckss_rust.h:2380 */
int32_t vckss_rust_engine_numerical_result_v1(uint64_t, VckssNumericalResultV1 *, uint32_t);
/* vckss_rust.h:2382 */
int32_t vckss_rust_engine_numerical_rhs_v1(uint64_t, VckssNumericalRhsV1 *, uint64_t, uint64_t *);
/* vckss_rust.h:2116 */
int32_t vckss_rust_engine_performance_receipt_v1(uint64_t generation, VckssEnginePerformanceReceiptV1 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:1793 */
int32_t vckss_rust_engine_prepare_interrupt_v3(const VckssEnginePrepareRequestInterruptV2 *request, const VckssEngineColumnsV3 *columns, uint64_t *output_handle, uint32_t output_capacity_bytes);
/* vckss_rust.h:2313 */
int32_t vckss_rust_engine_prepare_memory_interrupt_v1(const VckssEnginePrepareRequestInterruptV3 *, const VckssEngineColumnsV3 *, const VckssMemoryPolicyV1 *, uint64_t *, uint32_t);
/* vckss_rust.h:1853 */
int32_t vckss_rust_engine_repeat_measurement_diagnostic_v1(uint64_t generation, VckssRepeatMeasurementDiagnosticV1 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:1858 */
int32_t vckss_rust_engine_repeat_measurement_leading_v1(uint64_t generation, VckssRepeatMeasurementLeadingV1 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:705 */
int32_t vckss_rust_engine_solve_exact_execution_interrupt_v1(uint64_t generation, const VckssExactExecutionRequestInterruptV1 *request);
/* vckss_rust.h:703 */
int32_t vckss_rust_engine_solve_exact_execution_v1(uint64_t generation, const VckssExactExecutionRequestV1 *request);
/* vckss_rust.h:693 */
int32_t vckss_rust_engine_solve_exact_legacy_execution_interrupt_v1(uint64_t generation, const VckssEngineSolveRequestInterruptV2 *request, uint32_t threads);
/* vckss_rust.h:701 */
int32_t vckss_rust_engine_solve_exact_resolved_execution_interrupt_v2(uint64_t generation, const VckssExactExecutionRequestInterruptV1 *request);
/* vckss_rust.h:699 */
int32_t vckss_rust_engine_solve_exact_resolved_execution_v2(uint64_t generation, const VckssExactExecutionRequestV1 *request);
/* vckss_rust.h:1957 */
int32_t vckss_rust_engine_solve_interrupt_v2(uint64_t generation, const VckssEngineSolveRequestInterruptV2 *request);
/* vckss_rust.h:1961 */
int32_t vckss_rust_engine_solve_interrupt_v3(uint64_t generation, const VckssEngineSolveRequestInterruptV3 *request);
/* vckss_rust.h:1590 */
int32_t vckss_rust_engine_solve_interrupt_v6(uint64_t generation, const VckssEngineSolveRequestInterruptV6 *request);
/* vckss_rust.h:1597 */
int32_t vckss_rust_engine_solve_interrupt_v7(uint64_t generation, const VckssEngineSolveRequestInterruptV7 *request);
/* vckss_rust.h:2352 */
int32_t vckss_rust_engine_solve_numerical_generic_legacy_v2(uint64_t generation, const VckssEngineSolveRequestInterruptV3 *request);
/* vckss_rust.h:2378 */
int32_t vckss_rust_engine_solve_numerical_interrupt_v1(uint64_t, const VckssNumericalRequestV1 *, VckssInterruptPollV1, void *, uint32_t);
/* vckss_rust.h:2356 */
int32_t vckss_rust_engine_solve_numerical_interrupt_v2(uint64_t, const VckssNumericalRequestV2 *, VckssInterruptPollV1, void *, uint32_t);
/* vckss_rust.h:2350 */
int32_t vckss_rust_engine_solve_numerical_legacy_v2(uint64_t generation, const VckssEngineSolveRequestInterruptV2 *request);
/* vckss_rust.h:2377 */
int32_t vckss_rust_engine_solve_numerical_v1(uint64_t, const VckssNumericalRequestV1 *);
/* vckss_rust.h:1937 */
int32_t vckss_rust_engine_solve_v2(uint64_t generation, const VckssEngineSolveRequestV2 *request);
/* vckss_rust.h:1941 */
int32_t vckss_rust_engine_solve_v3(uint64_t generation, const VckssEngineSolveRequestV3 *request);
/* vckss_rust.h:1588 */
int32_t vckss_rust_engine_solve_v6(uint64_t generation, const VckssEngineSolveRequestV6 *request);
/* vckss_rust.h:1815 */
int32_t vckss_rust_engine_stayer_augmentation_receipt_v1(uint64_t generation, VckssStayerAugmentationReceiptV1 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:1978 */
int32_t vckss_rust_engine_stayer_hybrid_result_v1(uint64_t generation, VckssStayerHybridResultV1 *output, uint32_t output_capacity_bytes);
/* vckss_rust.h:691 */
uint32_t vckss_rust_exact_execution_schema_v1(void);
/* vckss_rust.h:692 */
uint32_t vckss_rust_exact_legacy_execution_schema_v1(void);
/* vckss_rust.h:698 */
uint32_t vckss_rust_exact_resolved_execution_schema_v2(void);
/* vckss_rust.h:2375 */
uint32_t vckss_rust_numerical_schema_v1(void);
/* vckss_rust.h:2348 */
uint32_t vckss_rust_numerical_schema_v2(void);
/* vckss_rust.h:316 */
int32_t vckss_rust_report_call_v1(const VckssProgressOptionsV1 *, VckssProgressOperationV1, void *);
/* vckss_rust.h:1677 */
int32_t vckss_rust_session_clear_abandoned_v1(void);
/* vckss_rust.h:1679 */
const char *vckss_rust_session_last_error(void);
/* vckss_rust.h:1672 */
int32_t vckss_rust_session_preparation_receipt_v1(uint64_t generation, VckssPreparationReceiptV1 *output);
/* vckss_rust.h:1667 */
int32_t vckss_rust_session_prepare_v1(const VckssPrepareRequestV1 *request, const VckssColumnsV1 *columns, uint64_t *output_handle);
/* vckss_rust.h:1676 */
int32_t vckss_rust_session_release_v1(uint64_t generation);
/* vckss_rust.h:1678 */
int32_t vckss_rust_session_snapshot_v1(VckssSessionSnapshotV1 *output);

#ifdef __cplusplus
}
#endif

#if defined(__cplusplus)
static_assert(sizeof(VckssEnginePrepareRequestV1) == 24, "prepare request V1 layout");
static_assert(sizeof(VckssNumericalRequestV1) == 328, "numerical request layout");
static_assert(offsetof(VckssNumericalRequestV1, point) == 40, "numerical point offset");
static_assert(sizeof(VckssNumericalRequestV2) == 344, "numerical V2 request layout");
static_assert(sizeof(VckssNumericalResultV1) == 512, "numerical result layout");
static_assert(offsetof(VckssNumericalResultV1, conditional) == 168, "numerical covariance offset");
static_assert(sizeof(VckssNumericalRhsV1) == 24, "numerical RHS layout");
static_assert(sizeof(FevcbCmgSummaryV1) == 688, "CMG summary layout");
static_assert(sizeof(VckssEngineSolveRequestInterruptV4) == 312, "interrupt V4 solve layout");
static_assert(sizeof(VckssEngineSolveRequestV8) == 320, "V8 solve layout");
static_assert(sizeof(VckssEngineSolveRequestInterruptV8) == 344, "interrupt V8 solve layout");
static_assert(sizeof(VckssBackendRequestCapabilityRequestV3) == 120, "V3 capability request layout");
static_assert(sizeof(VckssBackendRequestCapabilityReceiptV3) == 160, "V3 capability receipt layout");
static_assert(sizeof(VckssFullCmgReceiptV1) == 400, "full-CMG receipt layout");
static_assert(sizeof(FevcbSolveOptionsV2) == 24, "device options V2 layout");
static_assert(sizeof(FevcbSetupTimingsV1) == 176, "setup timings layout");
static_assert(sizeof(FevcbLearnedDumpV1) == 80, "learned dump layout");
static_assert(sizeof(VckssEnginePrepareRequestV2) == 40, "prepare request V2 layout");
static_assert(sizeof(VckssEnginePrepareRequestV3) == 56, "prepare request V3 layout");
static_assert(sizeof(VckssEnginePrepareRequestV4) == 64, "prepare request V4 layout");
static_assert(sizeof(VckssEnginePrepareRequestInterruptV1) == 64, "interrupt prepare V1 layout");
static_assert(sizeof(VckssEnginePrepareRequestInterruptV2) == 80, "interrupt prepare V2 layout");
static_assert(sizeof(VckssEnginePrepareRequestInterruptV3) == 88, "interrupt prepare V3 layout");
static_assert(sizeof(VckssEngineColumnsV1) == 64, "columns V1 layout");
static_assert(sizeof(VckssEngineColumnsV2) == 80, "columns V2 layout");
static_assert(sizeof(VckssEngineColumnsV3) == 96, "columns V3 layout");
static_assert(sizeof(VckssEngineSolveRequestV1) == 176, "solve request V1 layout");
static_assert(sizeof(VckssEngineSolveRequestV2) == 200, "solve request V2 layout");
static_assert(sizeof(VckssEngineSolveRequestV3) == 264, "solve request V3 layout");
static_assert(sizeof(VckssEngineSolveRequestV4) == 288, "solve request V4 layout");
static_assert(sizeof(VckssEngineSolveRequestV5) == 304, "solve request V5 layout");
static_assert(sizeof(VckssEngineSolveRequestInterruptV1) == 200, "interrupt solve V1 layout");
static_assert(sizeof(VckssEngineSolveRequestInterruptV5) == 328, "interrupt solve V5 layout");
static_assert(sizeof(VckssEngineResultV1) == 144, "result layout");
static_assert(sizeof(VckssEnginePreparationReceiptV1) == 72, "preparation receipt V1 layout");
static_assert(sizeof(VckssEnginePreparationReceiptV2) == 248, "preparation receipt V2 layout");
static_assert(sizeof(VckssEnginePreparationReceiptV3) == 256, "preparation receipt V3 layout");
static_assert(sizeof(VckssEnginePreparationReceiptV4) == 264, "preparation receipt V4 layout");
static_assert(sizeof(VckssEngineRhsReceiptV1) == 48, "RHS receipt V1 layout");
static_assert(sizeof(VckssEngineRhsReceiptV2) == 96, "RHS receipt V2 layout");
static_assert(sizeof(VckssEngineSnapshotV1) == 24, "snapshot layout");
static_assert(sizeof(VckssBackendCapabilitiesV1) == 32, "capabilities layout");
static_assert(sizeof(VckssEngineDetailedReceiptV1) == 272, "detailed receipt V1 layout");
static_assert(sizeof(VckssEngineDetailedReceiptV2) == 360, "detailed receipt V2 layout");
static_assert(sizeof(VckssEngineDetailedReceiptV3) == 384, "detailed receipt V3 layout");
static_assert(sizeof(VckssEngineDetailedReceiptV4) == 448, "detailed receipt V4 layout");
static_assert(sizeof(VckssEngineDetailedReceiptV5) == 536, "detailed receipt V5 layout");
static_assert(sizeof(VckssEngineDetailedReceiptV6) == 840, "detailed receipt V6 layout");
static_assert(sizeof(VckssExecutionPlanReceiptV1) == 1000, "execution plan receipt layout");
static_assert(sizeof(VckssEngineDetailedReceiptV7) == 1840, "detailed receipt V7 layout");
static_assert(offsetof(VckssEngineDetailedReceiptV7, execution) == 840, "detailed receipt V7 extension offset");
#endif

#endif /* FEVC_B200_H */
