"""ctypes mirror of ``include/fevc_b200.h``.

The struct layouts are the plugin ABI's (``vckss_rust.h``), so the same
bindings drive this library and any binary exporting the reference plugin's
entry points.  ``Engine`` wraps the prepare -> solve -> result lifecycle in the
way the Stata shim calls it.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

u32, u64, i32, i64, f64 = C.c_uint32, C.c_uint64, C.c_int32, C.c_int64, C.c_double
dptr = C.POINTER(C.c_double)
InterruptPoll = C.CFUNCTYPE(C.c_int32, C.c_void_p)


class Struct(C.Structure):
    def as_dict(self):
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = v.as_dict() if isinstance(v, Struct) else v
        return out


class PrepareRequestV1(Struct):
    _fields_ = [("abi_version", u32), ("struct_size", u32), ("rows", u64), ("cleanup_abandoned", u32),
                ("reserved", u32)]


class PrepareRequestV2(Struct):
    _fields_ = PrepareRequestV1._fields_ + [("memory_limit_bytes", u64), ("caller_copy_bytes", u64)]


class PrepareRequestV3(Struct):
    _fields_ = [("v2", PrepareRequestV2), ("deletion_mode", u32), ("controls_count", u32), ("reserved_2", u64)]


class PrepareRequestV4(Struct):
    _fields_ = [("v3", PrepareRequestV3), ("implicit_match", u32), ("reserved_3", u32)]


class PrepareRequestInterruptV2(Struct):
    _fields_ = [("options", PrepareRequestV3), ("interrupt_poll", InterruptPoll), ("interrupt_context", C.c_void_p),
                ("checkpoint_interval", u32), ("reserved", u32)]


class PrepareRequestInterruptV3(Struct):
    _fields_ = [("options", PrepareRequestV4), ("interrupt_poll", InterruptPoll), ("interrupt_context", C.c_void_p),
                ("checkpoint_interval", u32), ("reserved", u32)]


class ColumnsV1(Struct):
    _fields_ = [("struct_size", u32), ("reserved", u32), ("rows", u64), ("worker", dptr), ("firm", dptr),
                ("deletion", dptr), ("outcome", dptr), ("frequency", dptr), ("target_weight", dptr)]


class ColumnsV2(Struct):
    _fields_ = [("v1", ColumnsV1), ("controls", C.POINTER(dptr)), ("controls_count", u32), ("reserved_2", u32)]


class ColumnsV3(Struct):
    _fields_ = [("v2", ColumnsV2), ("probe_order", dptr), ("probeorder_supplied", u32), ("reserved_3", u32)]


class SolveRequestV1(Struct):
    _fields_ = [("abi_version", u32), ("struct_size", u32), ("seed", u64), ("probes", u32),
                ("leverage_batch_width", u32), ("target_batch_width", u32), ("deletion_mode", u32),
                ("rng_contract", u32), ("solver_route", u32), ("allow_automatic_cmg_setup_fallback", u32),
                ("exact_dimension_limit", u64), ("cmg_minimum_dimension", u64), ("pcg_tolerance", f64),
                ("maximum_iterations", u32), ("residual_replacement_interval", u32), ("rank_tolerance", f64),
                ("block_tolerance", f64), ("cmg_terminal_vertices", u64), ("cmg_dense_vertex_cap", u64),
                ("cmg_maximum_levels", u64), ("cmg_aggregate_cap", u64), ("cmg_minimum_reduction", f64),
                ("cmg_jacobi_weight", f64), ("cmg_pre_sweeps", u32), ("cmg_post_sweeps", u32),
                ("cmg_maximum_edge_complexity", f64), ("cmg_maximum_vertex_complexity", f64),
                ("cmg_memory_limit_bytes", u64)]


class SolveRequestV2(Struct):
    _fields_ = [("v1", SolveRequestV1), ("algorithm", u32), ("nuisance_mode", u32), ("exact_estimator_limit", u64),
                ("blocksize_limit", u64)]


class SolveRequestV3(Struct):
    _fields_ = [("v2", SolveRequestV2), ("engine", u32), ("batch_mode", u32), ("stayers_mode", u32),
                ("target_weight_mode", u32), ("deletion_unit_source", u32), ("probeorder_supplied", u32),
                ("wallseconds_supplied", u32), ("capability_schema", u32), ("capability_profile", u32),
                ("frequency_use", u32), ("physical_limit", u64), ("request_signature", u64), ("reserved_3", u64)]


class SolveRequestV4(Struct):
    _fields_ = [("v3", SolveRequestV3), ("leverage_batch_mode", u32), ("target_batch_mode", u32),
                ("wallseconds", f64), ("reserved_4", u64)]


class SolveRequestV5(Struct):
    _fields_ = [("v4", SolveRequestV4), ("threads", u32), ("tolerance_supplied", u32), ("full_cmg_v2", u32),
                ("reserved_5", u32)]


class SolveRequestInterruptV4(Struct):
    _fields_ = [("options", SolveRequestV4), ("interrupt_poll", InterruptPoll), ("interrupt_context", C.c_void_p),
                ("checkpoint_interval", u32), ("reserved", u32)]


class SolveRequestV6(Struct):
    _fields_ = [("v4", SolveRequestV4), ("execution_mode", u32), ("threads", u32), ("reserved_6", u64)]


class SolveRequestV7(Struct):
    _fields_ = [("v6", SolveRequestV6), ("component_batch_mode", u32), ("reserved_7", u32)]


class SolveRequestV8(Struct):
    _fields_ = [("v7", SolveRequestV7), ("resolved_execution_mode", u32), ("tolerance_supplied", u32)]


class SolveRequestInterruptV8(Struct):
    _fields_ = [("options", SolveRequestV8), ("interrupt_poll", InterruptPoll), ("interrupt_context", C.c_void_p),
                ("checkpoint_interval", u32), ("reserved", u32)]


class CapabilityRequestV1(Struct):
    _fields_ = [(n, u32) for n in ("abi_version", "struct_size", "request_schema", "algorithm", "deletion_mode",
                                   "nuisance_mode", "solver_route", "rng_contract", "controls_count",
                                   "frequency_use")] + [("reserved", u64)]


class CapabilityRequestV2(Struct):
    _fields_ = [("v1", CapabilityRequestV1)] + [(n, u32) for n in (
        "engine", "batch_mode", "stayers_mode", "target_weight_mode", "deletion_unit_source", "probeorder_supplied",
        "wallseconds_supplied", "reserved_2")] + [("physical_limit", u64)]


class CapabilityRequestV3(Struct):
    _fields_ = [("v2", CapabilityRequestV2), ("leverage_batch_mode", u32), ("target_batch_mode", u32),
                ("allow_automatic_cmg_setup_fallback", u32), ("reserved_3", u32), ("wallseconds", f64),
                ("reserved_4", u64)]


class SolveRequestInterruptV1(Struct):
    _fields_ = [("options", SolveRequestV1), ("interrupt_poll", InterruptPoll), ("interrupt_context", C.c_void_p),
                ("checkpoint_interval", u32), ("reserved", u32)]


class Components(Struct):
    _fields_ = [("worker", f64), ("firm", f64), ("covariance", f64), ("total", f64)]

    def tuple(self):
        return (self.worker, self.firm, self.covariance, self.total)


class ResultV1(Struct):
    _fields_ = [("struct_size", u32), ("reserved", u32), ("generation", u64), ("plugin", Components),
                ("correction", Components), ("corrected", Components), ("numerical_mcse", Components)]


class NumericalRequestV1(Struct):
    """Numerical MCSE attachment request (reference vckss_rust.h
    VckssNumericalRequestV1, 328 bytes; the point request is a V4 solve)."""
    _fields_ = [(n, u32) for n in ("abi_version", "struct_size", "schema_version", "threads", "tolerance_supplied",
                                   "projection_requested", "component_requested", "reserved", "controls_count",
                                   "reserved_2")] + [("point", SolveRequestV4)]


class NumericalResultV1(Struct):
    """Numerical MCSE attachment result (VckssNumericalResultV1, 512 bytes)."""
    _fields_ = [("struct_size", u32), ("schema_version", u32), ("generation", u64)] + [
        (n, u32) for n in ("status", "engine", "leverage_probes", "target_probes", "target_fold_a",
                           "target_fold_b")] + [
        (n, u64) for n in ("certified_replay_rhs", "executed_replay_rhs", "attempted_replay_rhs",
                           "replay_generator_words", "allocation_bound_bytes")] + [
        ("failed_replay_probe", u32), ("replay_error_code", u32)] + [
        (n, f64) for n in ("psd_adjustment", "minimum_constrained", "minimum_residual_margin",
                           "maximum_sensitivity_ratio")] + [
        ("score_means", f64 * 6), ("conditional", f64 * 9), ("leverage", f64 * 9), ("raw", f64 * 9),
        ("usable", f64 * 9), ("mcse", f64 * 4), ("point_rhs", u64), ("maximum_point_complete_residual", f64),
        ("maximum_replay_complete_residual", f64)]


class ProbeSetV1(Struct):
    _fields_ = [("seed", u64), ("probes", u32), ("reserved", u32)]


class ProbeSetResultV1(Struct):
    _fields_ = [("plugin", Components), ("correction", Components), ("corrected", Components),
                ("numerical_mcse", Components)]


class NumericalRhsV1(Struct):
    _fields_ = [("schema_version", u32), ("phase", u32), ("probe", u32), ("reserved", u32),
                ("complete_residual", f64)]


class FevcbSetupTimingsV1(Struct):
    _fields_ = [("struct_size", u32), ("builders", u32), ("builder_ms", f64 * 16), ("builders_span_ms", f64),
                ("device_units_ms", f64), ("hybrid_ms", f64), ("preconditioner_ms", f64), ("total_ms", f64)]


class ProjectionAugmentationRequestV1(Struct):
    _fields_ = [("abi_version", u32), ("struct_size", u32), ("rows", u64), ("project_count", u32), ("effect", u32),
                ("weight", u32), ("reserved", u32), ("rank_tolerance", f64), ("caller_copy_bytes", u64)]


class ProjectionAugmentationRequestInterruptV1(Struct):
    _fields_ = [("options", ProjectionAugmentationRequestV1), ("interrupt_poll", C.c_void_p),
                ("interrupt_context", C.c_void_p), ("checkpoint_interval", u32), ("reserved", u32)]


class ProjectionColumnsV1(Struct):
    _fields_ = [("struct_size", u32), ("reserved", u32), ("rows", u64), ("project", C.POINTER(C.POINTER(f64))),
                ("project_count", u32), ("reserved_2", u32)]


class ProjectionAugmentationReceiptV1(Struct):
    _fields_ = [("struct_size", u32), ("schema_version", u32), ("generation", u64), ("rows", u64), ("columns", u64),
                ("effect", u32), ("weight", u32), ("caller_copy_bytes", u64),
                ("augmentation_peak_forecast_bytes", u64), ("projection_persistent_bytes", u64),
                ("total_prepared_resident_bytes", u64), ("gram_rcond", f64), ("gram_relres", f64),
                ("gram_original_relres", f64)]


class ProjectionResultReceiptV1(Struct):
    _fields_ = [("struct_size", u32), ("schema_version", u32), ("generation", u64), ("columns", u64),
                ("effect", u32), ("weight", u32), ("gram_rcond", f64), ("gram_relres", f64),
                ("gram_original_relres", f64), ("covariance_smallest_eigenvalue", f64),
                ("covariance_largest_eigenvalue", f64), ("psd_cleanup", f64), ("proxy_minimum", f64),
                ("proxy_maximum", f64), ("maximum_iterations", u32), ("reserved", u32),
                ("maximum_reduced_residual", f64), ("maximum_complete_residual", f64),
                ("full_residual_tolerance", f64), ("projection_peak_forecast_bytes", u64), ("persistent_bytes", u64),
                ("result_bytes", u64)]


class PreparationReceiptV2(Struct):
    _fields_ = [("struct_size", u32), ("reserved", u32)] + [(n, u64) for n in (
        "generation", "input_rows", "retained_rows", "workers", "firms", "cells", "deletion_units", "target_strata",
        "memory_limit_bytes", "caller_copy_bytes", "preparation_peak_forecast_bytes", "prepared_resident_bytes",
        "graph_input_rows", "graph_retained_rows", "graph_input_physical_mass", "graph_retained_physical_mass",
        "graph_initial_components", "graph_maximum_components", "graph_initial_component_rows",
        "graph_mover_input_rows", "graph_initial_deletion_edges", "graph_retained_deletion_edges",
        "graph_insufficient_workers_removed", "graph_articulation_workers_removed", "graph_bridge_units_removed",
        "graph_bridge_rows_removed", "graph_degree_iterations", "graph_articulation_iterations",
        "graph_bridge_iterations", "graph_fixed_point_iterations")]


class PreparationReceiptV3(Struct):
    _fields_ = [("v2", PreparationReceiptV2), ("target_weight_sum", f64)]


class PreparationReceiptV4(Struct):
    _fields_ = [("v3", PreparationReceiptV3), ("controls_count", u32), ("deletion_mode", u32)]


class RhsReceiptV1(Struct):
    _fields_ = [("phase", u32), ("side", u32), ("probe", i64), ("route", u32), ("iterations", u32),
                ("zero_rhs", u32), ("reserved", u32), ("reduced_residual", f64), ("complete_residual", f64)]


class SnapshotV1(Struct):
    _fields_ = [("struct_size", u32), ("state", u32), ("generation", u64), ("last_released_generation", u64)]


class FevcbSolveOptionsV1(Struct):
    _fields_ = [("struct_size", u32), ("block_columns", u32), ("preconditioner", u32), ("keep_unit_detail", u32)]


class FevcbSolveOptionsV2(Struct):
    _fields_ = [("v1", FevcbSolveOptionsV1), ("precision", u32), ("reserved", u32)]


class FevcbTuningV1(Struct):
    _fields_ = [("struct_size", u32), ("chosen", C.c_int32), ("candidates", u32), ("precision", u32 * 3),
                ("preconditioner", u32 * 3), ("reserved", u32), ("milliseconds", f64 * 3)]


class FevcbPrepareTimingsV1(Struct):
    _fields_ = [("struct_size", u32), ("threads", u32), ("ingest_ms", f64), ("canonical_ms", f64),
                ("graph_ms", f64), ("compression_ms", f64), ("plan_ms", f64), ("total_ms", f64)]


class FevcbSolveTimingsV1(Struct):
    _fields_ = [("struct_size", u32), ("fallbacks", u32), ("total_ms", f64), ("fit_ms", f64), ("leverage_ms", f64),
                ("target_ms", f64), ("setup_ms", f64)] + [(n, u64) for n in (
                    "block_iterations", "column_iterations", "rhs_columns", "kernel_launches", "h2d_bytes",
                    "vertices", "edges", "kept_workers", "levels")]


SIZES = {
    SolveRequestInterruptV4: 312, SolveRequestV8: 320, SolveRequestInterruptV8: 344, CapabilityRequestV3: 120,
    PrepareRequestV1: 24, PrepareRequestV2: 40, PrepareRequestV3: 56, PrepareRequestV4: 64,
    PrepareRequestInterruptV2: 80, PrepareRequestInterruptV3: 88, ColumnsV1: 64, ColumnsV2: 80, ColumnsV3: 96,
    SolveRequestV1: 176, SolveRequestV2: 200, SolveRequestV3: 264, SolveRequestV4: 288, SolveRequestV5: 304,
    SolveRequestInterruptV1: 200, ResultV1: 144, PreparationReceiptV2: 248, PreparationReceiptV3: 256,
    PreparationReceiptV4: 264, RhsReceiptV1: 48, SnapshotV1: 24,
}
for _cls, _size in SIZES.items():
    assert C.sizeof(_cls) == _size, (_cls.__name__, C.sizeof(_cls), _size)

TAG_LEVERAGE = 0x4C45564552414745
TAG_TARGET = 0x0054415247455401

# Every entry point the header declares, with its ctypes signature.
# Detailed receipts V1-V7 (vckss_rust.h:1084-1439); layouts as in include/fevc_b200.h.


class EngineDetailedReceiptV1(Struct):
    _fields_ = [
        ("struct_size", u32), ("reserved", u32), ("generation", u64), ("seed", u64), ("probes_requested", u32),
        ("leverage_probes_accepted", u32), ("target_probes_accepted", u32), ("solver_requested", u32),
        ("solver_selected", u32), ("solver_fallback", u32), ("solver_fallback_error", i32),
        ("solver_dimension", u64), ("leverage_batch_width", u64), ("target_batch_width", u64),
        ("rank_tolerance", f64), ("block_tolerance", f64), ("full_residual_tolerance", f64),
        ("full_fit_route", u32), ("full_fit_iterations", u32), ("full_fit_reduced_residual", f64),
        ("full_fit_complete_residual", f64), ("full_fit_zero_rhs", u32), ("reserved_1", u32),
        ("leverage_rhs_count", u64), ("target_rhs_count", u64), ("max_reduced_residual", f64),
        ("max_complete_residual", f64), ("max_leverage", f64), ("max_reciprocal_residual", f64),
        ("accounting_residual", f64), ("topology_checksum", u64), ("cmg_levels", u64), ("cmg_fine_vertices", u64),
        ("cmg_fine_edges", u64), ("cmg_terminal_vertices", u64), ("cmg_edge_complexity", f64),
        ("cmg_vertex_complexity", f64), ("cmg_structural_bytes", u64), ("cmg_workspace_bytes", u64),
        ("cmg_dense_factor_bytes", u64)
    ]


class EngineDetailedReceiptV2(Struct):
    _fields_ = [
        ("struct_size", u32), ("reserved", u32), ("generation", u64), ("seed", u64), ("probes_requested", u32),
        ("leverage_probes_accepted", u32), ("target_probes_accepted", u32), ("solver_requested", u32),
        ("solver_selected", u32), ("solver_fallback", u32), ("solver_fallback_error", i32),
        ("solver_dimension", u64), ("leverage_batch_width", u64), ("target_batch_width", u64),
        ("rank_tolerance", f64), ("block_tolerance", f64), ("full_residual_tolerance", f64),
        ("full_fit_route", u32), ("full_fit_iterations", u32), ("full_fit_reduced_residual", f64),
        ("full_fit_complete_residual", f64), ("full_fit_zero_rhs", u32), ("reserved_1", u32),
        ("leverage_rhs_count", u64), ("target_rhs_count", u64), ("max_reduced_residual", f64),
        ("max_complete_residual", f64), ("max_leverage", f64), ("max_reciprocal_residual", f64),
        ("accounting_residual", f64), ("topology_checksum", u64), ("cmg_levels", u64), ("cmg_fine_vertices", u64),
        ("cmg_fine_edges", u64), ("cmg_terminal_vertices", u64), ("cmg_edge_complexity", f64),
        ("cmg_vertex_complexity", f64), ("cmg_structural_bytes", u64), ("cmg_workspace_bytes", u64),
        ("cmg_dense_factor_bytes", u64), ("full_fit_weighted_rss", f64), ("memory_limit_bytes", u64),
        ("caller_copy_bytes", u64), ("preparation_peak_forecast_bytes", u64), ("prepared_resident_bytes", u64),
        ("solver_setup_forecast_bytes", u64), ("leverage_phase_forecast_bytes", u64),
        ("target_phase_forecast_bytes", u64), ("result_forecast_bytes", u64), ("solve_peak_forecast_bytes", u64),
        ("command_peak_forecast_bytes", u64)
    ]


class EngineDetailedReceiptV3(Struct):
    _fields_ = [
        ("v2", EngineDetailedReceiptV2), ("rng_contract", u32), ("reserved_2", u32), ("rhs_receipt_rows", u64),
        ("caller_result_copy_bytes", u64)
    ]


class EngineDetailedReceiptV4(Struct):
    _fields_ = [
        ("v3", EngineDetailedReceiptV3), ("algorithm_requested", u32), ("algorithm_selected", u32),
        ("deletion_mode", u32), ("nuisance_mode", u32), ("parameters", u64), ("full_parameters", u64),
        ("correction_parameters", u64), ("information_rcond", f64), ("inverse_relres", f64),
        ("exact_peak_forecast_bytes", u64)
    ]


class EngineDetailedReceiptV5(Struct):
    _fields_ = [
        ("v4", EngineDetailedReceiptV4), ("applicability_flags", u64), ("working_fit_complete_residual", f64),
        ("inverse_sqrt_relres", f64), ("maker_relres", f64), ("control_basis_relres", f64),
        ("control_basis_forward_error", f64), ("deletion_rank_gap", f64), ("firm_zero_sum_residual", f64),
        ("fit_peak_forecast_bytes", u64), ("correction_peak_forecast_bytes", u64),
        ("actual_accounting_residual", f64)
    ]


class EngineDetailedReceiptV6(Struct):
    _fields_ = [
        ("v5", EngineDetailedReceiptV5), ("engine_requested", u32), ("engine_selected", u32),
        ("generic_applicability_flags", u64), ("controls_count", u32), ("rhs_receipt_schema", u32),
        ("control_projection_rhs_count", u64), ("control_rank_rcond", f64),
        ("control_rank_smallest_generalized_eigenvalue_lower", f64),
        ("control_rank_largest_generalized_eigenvalue_upper", f64), ("control_rank_projection_error_bound", f64),
        ("control_rank_normalization_error_bound", f64),
        ("control_rank_fe_information_eigenvalue_lower_bound", f64),
        ("control_rank_maximum_projection_residual", f64), ("control_rank_effective_tolerance", f64),
        ("control_rank_projection_pcg_tolerance", f64), ("control_rank_projection_residual_gate", f64),
        ("generic_control_basis_relres", f64), ("generic_control_basis_forward_error", f64),
        ("generic_control_schur_rcond", f64), ("generic_control_schur_relres", f64),
        ("generic_deletion_rank_gap", f64), ("full_joint_fit_complete_residual", f64),
        ("generic_working_fit_complete_residual", f64), ("generic_maker_relres", f64),
        ("canonicalization_peak_forecast_bytes", u64), ("generic_fit_peak_forecast_bytes", u64),
        ("geometry_peak_forecast_bytes", u64), ("generic_leverage_peak_forecast_bytes", u64),
        ("generic_target_peak_forecast_bytes", u64), ("maker_peak_forecast_bytes", u64),
        ("generic_result_forecast_bytes", u64), ("generic_peak_forecast_bytes", u64),
        ("rhs_v2_caller_copy_bytes", u64), ("capability_schema", u32), ("capability_profile", u32),
        ("batch_mode", u32), ("stayers_mode", u32), ("target_weight_mode", u32), ("deletion_unit_source", u32),
        ("probeorder_supplied", u32), ("wallseconds_supplied", u32), ("frequency_use", u32), ("reserved_6", u32),
        ("physical_limit", u64), ("request_signature", u64)
    ]


class EstimatorResolutionReceiptV1(Struct):
    _fields_ = [
        ("algorithm_schema", u32), ("algorithm_requested", u32), ("algorithm_selected", u32),
        ("algorithm_reason", u32), ("engine_schema", u32), ("engine_requested", u32), ("engine_selected", u32),
        ("engine_reason", u32), ("compressed_eligibility", u32), ("resolved_before_rng", u32),
        ("opportunistic_engine_fallback_allowed", u32), ("reserved", u32), ("identified_complexity", u64),
        ("exact_limit", u64), ("rng_draws_before_resolution", u64), ("counter_atoms_before_resolution", u64)
    ]


class SolverExecutionReceiptV1(Struct):
    _fields_ = [
        ("schema_version", u32), ("requested_route", u32), ("selected_route", u32), ("fallback_used", u32),
        ("fallback_error", i32), ("full_setup_complete", u32), ("fe_setup_complete", u32),
        ("fe_hierarchy_reused", u32), ("plan_frozen_before_rng", u32), ("auto_route_contract", u32),
        ("threads_requested", u32), ("threads_used", u32), ("parallel_regions", u32), ("applicability", u32),
        ("reserved_1", u32), ("reserved_2", u32), ("planned_rhs", u64), ("auto_firm_threshold", u64),
        ("auto_rhs_threshold", u64), ("full_solver_dimension", u64), ("fe_solver_dimension", u64),
        ("logical_atoms_before_plan_freeze", u64), ("unique_words_before_plan_freeze", u64),
        ("physical_trials_before_plan_freeze", u64)
    ]


class BatchPhasePlanReceiptV1(Struct):
    _fields_ = [
        ("request_mode", u32), ("selection_reason", u32), ("applicability", u32), ("reserved", u32),
        ("requested_width", u64), ("selected_width", u64), ("probe_width_cap", u64), ("declared_threads", u64),
        ("thread_width_cap", u64), ("route_width_cap", u64), ("effective_width_cap", u64),
        ("hard_memory_bytes", u64), ("width_one_forecast_bytes", u64), ("selected_forecast_bytes", u64)
    ]


class BatchExecutionReceiptV1(Struct):
    _fields_ = [
        ("schema_version", u32), ("deterministic", u32), ("width_invariance_required", u32),
        ("arithmetic_contract", u32), ("whole_command_admitted", u32), ("applicability", u32),
        ("non_batched_peak_bytes", u64), ("selected_command_peak_bytes", u64),
        ("leverage", BatchPhasePlanReceiptV1), ("target", BatchPhasePlanReceiptV1)
    ]


class WallExecutionReceiptV1(Struct):
    _fields_ = [
        ("schema_version", u32), ("model_code", u32), ("status", u32), ("routing_effect", u32),
        ("requested_applicable", u32), ("forecast_applicable", u32), ("advisory_applicable", u32),
        ("margin_applicable", u32), ("requested_seconds", f64), ("forecast_seconds", f64),
        ("advisory_seconds", f64), ("advisory_margin_fraction", f64), ("preparation_work", u64),
        ("engine_setup_work", u64), ("full_fit_work", u64), ("leverage_work", u64), ("target_work", u64),
        ("result_export_work", u64), ("total_work", u64)
    ]


class CounterPhaseExecutionReceiptV1(Struct):
    _fields_ = [
        ("planned_logical_atoms", u64), ("actual_logical_atoms", u64), ("planned_unique_packed_words", u64),
        ("actual_unique_packed_words", u64), ("planned_physical_trials", u64), ("actual_physical_trials", u64),
        ("planned_generator_work", u64), ("actual_generator_work", u64)
    ]


class CounterExecutionReceiptV1(Struct):
    _fields_ = [
        ("schema_version", u32), ("rng_contract", u32), ("generator_work_applicable", u32), ("completed", u32),
        ("leverage", CounterPhaseExecutionReceiptV1), ("target", CounterPhaseExecutionReceiptV1),
        ("total", CounterPhaseExecutionReceiptV1), ("logical_atoms_before_plan_freeze", u64),
        ("unique_words_before_plan_freeze", u64), ("physical_trials_before_plan_freeze", u64)
    ]


class ExecutionMemoryReceiptV1(Struct):
    _fields_ = [
        ("schema_version", u32), ("applicability", u32), ("peak_phase", u32), ("reserved", u32),
        ("hard_limit_bytes", u64), ("prepared_persistent_bytes", u64), ("setup_peak_bytes", u64),
        ("fit_peak_bytes", u64), ("correction_peak_bytes", u64), ("leverage_peak_bytes", u64),
        ("target_peak_bytes", u64), ("result_peak_bytes", u64), ("non_batched_peak_bytes", u64),
        ("command_peak_bytes", u64), ("shared_cmg_persistent_bytes", u64),
        ("full_control_block_persistent_bytes", u64), ("setup_transient_bytes", u64),
        ("cmg_preconditioner_workspace_bytes", u64), ("cmg_aggregated_cell_capacity_bytes", u64),
        ("cmg_group_index_bytes", u64), ("cmg_hybrid_graph_bytes", u64), ("retained_nq_bytes", u64),
        ("retained_q2_bytes", u64)
    ]


class ExecutionPlanReceiptV1(Struct):
    _fields_ = [
        ("struct_size", u32), ("schema_version", u32), ("generation", u64), ("applicability_flags", u64),
        ("contract_flags", u64), ("request_signature", u64), ("resolution", EstimatorResolutionReceiptV1),
        ("solver", SolverExecutionReceiptV1), ("batch", BatchExecutionReceiptV1),
        ("wall", WallExecutionReceiptV1), ("counter", CounterExecutionReceiptV1),
        ("memory", ExecutionMemoryReceiptV1)
    ]


class EngineDetailedReceiptV7(Struct):
    _fields_ = [
        ("v6", EngineDetailedReceiptV6), ("execution", ExecutionPlanReceiptV1)
    ]

class FullCmgReceiptV1(C.Structure):
    """The plugin's VckssFullCmgReceiptV1 (vckss_rust.h:1458-1509, 400 bytes)."""
    _fields_ = ([("struct_size", u32), ("schema_version", u32), ("generation", u64), ("backend_identity", u32),
                 ("platform_os", u32), ("platform_arch", u32), ("batch_strategy_mask", u32),
                 ("cmg_source_commit", C.c_uint8 * 40), ("threads_requested", u32), ("threads_used", u32)]
                + [(n, u64) for n in ("maximum_concurrency", "vertices", "edges", "hierarchy_levels",
                                      "terminal_vertices", "graph_copy_bytes", "hierarchy_bytes", "plan_bytes",
                                      "workspace_bytes_each", "workspace_pool_bytes", "admitted_peak_bytes")]
                + [(n, f64) for n in ("fit_effective_tolerance", "probe_effective_tolerance",
                                      "fit_initial_inner_tolerance", "probe_initial_inner_tolerance")]
                + [(n, u64) for n in ("refinement_attempts", "refined_columns", "batch_calls", "rhs_count",
                                      "serial_batches", "planned_batches", "across_rhs_batches", "total_iterations",
                                      "total_operator_applications", "total_preconditioner_applications")]
                + [(n, f64) for n in ("maximum_reduced_residual", "maximum_complete_residual")]
                + [(n, u64) for n in ("graph_ns", "hierarchy_plan_ns", "rhs_ns", "solve_ns", "extraction_ns",
                                      "preparation_peak_bytes", "prepared_persistent_bytes",
                                      "non_cmg_command_peak_bytes", "pre_rng_forecast_bytes", "actual_retained_bytes",
                                      "allocator_allowance_bytes", "maximum_batch_rhs", "workspace_count")])


assert C.sizeof(FullCmgReceiptV1) == 400


class CmgSummaryV1(C.Structure):
    _fields_ = [("struct_size", u32), ("eliminate_max_degree", u32), ("vertices", u64), ("edges", u64),
                ("hierarchy_levels", u64), ("terminal_vertices", u64), ("terminal_reason", u32), ("reserved", u32),
                ("level_vertices", u64 * 32), ("level_edges", u64 * 32), ("level_repeat", u32 * 32)]


assert C.sizeof(CmgSummaryV1) == 688


def cmg_aggregate(lib, ptr: np.ndarray, col: np.ndarray, weight: np.ndarray, threshold: float = 0.125):
    """One CMG forest-aggregation step (host): (labels, aggregate count)."""
    n = len(ptr) - 1
    ptr = np.ascontiguousarray(ptr, dtype=np.uint32)
    col = np.ascontiguousarray(col, dtype=np.uint32)
    weight = np.ascontiguousarray(weight, dtype=np.float64)
    labels = np.zeros(n, dtype=np.uint32)
    count = u32(0)
    up = C.POINTER(u32)
    st = lib.fevcb_cmg_aggregate_v1(n, ptr.ctypes.data_as(up), col.ctypes.data_as(up), weight.ctypes.data_as(dptr),
                                    threshold, labels.ctypes.data_as(up), C.byref(count))
    if st != 0:
        raise EngineError(st, lib.vckss_rust_engine_last_error().decode())
    return labels, int(count.value)


SIGNATURES = {
    "fevcb_engine_setup_timings_v1": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_augment_projection_interrupt_v1": (i32, [u64, C.c_void_p, C.c_void_p]),
    "vckss_rust_engine_default_projection_augmentation_request_interrupt_v1": (i32, [C.c_void_p, u32]),
    "vckss_rust_engine_projection_augmentation_receipt_v1": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_projection_result_receipt_v1": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_projection_result_v1": (i32, [u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u32]),
    "vckss_rust_projection_centering_schema_v1": (u32, []),
    "vckss_rust_abi_version": (u32, []),
    "vckss_rust_backend_version": (C.c_char_p, []),
    "vckss_rust_capabilities_json": (C.c_char_p, []),
    "vckss_rust_last_error": (C.c_char_p, []),
    "vckss_rust_selftest": (i32, []),
    "vckss_rust_backend_capabilities_v1": (i32, [C.c_void_p, u32]),
    "vckss_rust_engine_default_solve_request_v1": (i32, [C.c_void_p, u32]),
    "vckss_rust_engine_default_solve_request_v2": (i32, [C.c_void_p, u32]),
    "vckss_rust_engine_default_solve_request_v3": (i32, [C.c_void_p, u32]),
    "vckss_rust_engine_default_solve_request_v4": (i32, [C.c_void_p, u32]),
    "vckss_rust_engine_default_solve_request_v5": (i32, [C.c_void_p, u32]),
    "vckss_rust_engine_default_solve_request_interrupt_v1": (i32, [C.c_void_p, u32]),
    "vckss_rust_engine_default_solve_request_interrupt_v5": (i32, [C.c_void_p, u32]),
    "vckss_rust_engine_default_prepare_request_v3": (i32, [C.c_void_p, u32]),
    "vckss_rust_engine_default_prepare_request_interrupt_v1": (i32, [C.c_void_p, u32]),
    "vckss_rust_engine_default_prepare_request_interrupt_v2": (i32, [C.c_void_p, u32]),
    "vckss_rust_engine_default_prepare_request_interrupt_v3": (i32, [C.c_void_p, u32]),
    "vckss_rust_engine_prepare_v1": (i32, [C.c_void_p, C.c_void_p, C.POINTER(u64), u32]),
    "vckss_rust_engine_prepare_v2": (i32, [C.c_void_p, C.c_void_p, C.POINTER(u64), u32]),
    "vckss_rust_engine_prepare_v3": (i32, [C.c_void_p, C.c_void_p, C.POINTER(u64), u32]),
    "vckss_rust_engine_prepare_interrupt_v1": (i32, [C.c_void_p, C.c_void_p, C.POINTER(u64), u32]),
    "vckss_rust_engine_prepare_interrupt_v2": (i32, [C.c_void_p, C.c_void_p, C.POINTER(u64), u32]),
    "vckss_rust_engine_prepare_interrupt_v4": (i32, [C.c_void_p, C.c_void_p, C.POINTER(u64), u32]),
    "vckss_rust_engine_centering_v1": (i32, [u64, u32]),
    "vckss_rust_engine_solve_v1": (i32, [u64, C.c_void_p]),
    "vckss_rust_engine_solve_interrupt_v1": (i32, [u64, C.c_void_p]),
    "vckss_rust_engine_solve_v5": (i32, [u64, C.c_void_p]),
    "vckss_rust_engine_solve_interrupt_v5": (i32, [u64, C.c_void_p]),
    "vckss_rust_engine_solve_v4": (i32, [u64, C.c_void_p]),
    "vckss_rust_engine_solve_interrupt_v4": (i32, [u64, C.c_void_p]),
    "vckss_rust_engine_default_solve_request_v8": (i32, [C.c_void_p, u32]),
    "vckss_rust_engine_default_solve_request_interrupt_v8": (i32, [C.c_void_p, u32]),
    "vckss_rust_engine_solve_v8": (i32, [u64, C.c_void_p]),
    "vckss_rust_engine_solve_interrupt_v8": (i32, [u64, C.c_void_p]),
    "vckss_rust_backend_request_capability_v3": (i32, [C.c_void_p, C.c_void_p, u32]),
    "vckss_rust_engine_full_cmg_receipt_v1": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_result_v1": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_preparation_receipt_v1": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_preparation_receipt_v2": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_preparation_receipt_v3": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_preparation_receipt_v4": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_retained_mask_v1": (i32, [u64, C.c_void_p, u64]),
    "vckss_rust_engine_rhs_receipts_v1": (i32, [u64, C.c_void_p, u64]),
    "vckss_rust_engine_rhs_receipts_v2": (i32, [u64, C.c_void_p, u64]),
    "vckss_rust_engine_release_v1": (i32, [u64]),
    "vckss_rust_engine_clear_abandoned_v1": (i32, []),
    "vckss_rust_engine_snapshot_v1": (i32, [C.c_void_p, u32]),
    "vckss_rust_engine_last_error": (C.c_char_p, []),
    "fevcb_device_count": (i32, []),
    "fevcb_set_stream": (i32, [C.c_void_p]),
    "fevcb_device_cache_trim_v1": (i32, [C.POINTER(u64), C.POINTER(u64)]),
    "fevcb_engine_hybrid_check_v1": (i32, [u64, C.POINTER(u32)]),
    "fevcb_engine_solve_options_v1": (i32, [u64, C.c_void_p]),
    "fevcb_engine_timings_v1": (i32, [u64, C.c_void_p, u32]),
    "fevcb_engine_resolve_v1": (i32, [u64]),
    "fevcb_engine_unit_detail_v1": (i32, [u64, u64] + [dptr] * 6 + [u64, dptr, dptr, u64, dptr]),
    "fevcb_engine_problem_view_v1": (i32, [u64, C.c_void_p, u32]),
    "fevcb_engine_kernel_benchmark_v1": (i32, [u64, u32, u32, u32, C.POINTER(f64), C.POINTER(f64)]),
    "fevcb_engine_cmg_summary_v1": (i32, [u64, u32, C.c_void_p, u32]),
    "fevcb_engine_shard_size_v1": (i32, [u64, C.POINTER(u64)]),
    "fevcb_engine_shard_leverage_v1": (i32, [u64, C.c_void_p, u32, u32, C.POINTER(f64), u64]),
    "fevcb_engine_shard_target_v1": (i32, [u64, C.c_void_p, u32, u32, C.POINTER(f64), u64, C.POINTER(f64)]),
    "fevcb_engine_shard_finish_v1": (i32, [u64, C.c_void_p, C.POINTER(f64)]),
    "fevcb_learned_param_count_v1": (i32, [C.POINTER(u64)]),
    "fevcb_learned_initial_params_v1": (i32, [u64, C.POINTER(C.c_float), u64]),
    "fevcb_learned_install_v1": (i32, [C.POINTER(C.c_float), u64]),
    "fevcb_learned_trainer_create_v1": (i32, [u64, C.POINTER(u64)]),
    "fevcb_learned_trainer_destroy_v1": (i32, [u64]),
    "fevcb_learned_trainer_add_panel_v1": (i32, [u64, u64, u32, u64]),
    "fevcb_learned_trainer_train_v1": (i32, [u64, u32, f64, C.POINTER(f64)]),
    "fevcb_learned_trainer_gradient_v1": (i32, [u64, u32, C.POINTER(f64), C.POINTER(C.c_float), u64]),
    "fevcb_learned_trainer_params_v1": (i32, [u64, C.POINTER(C.c_float), u64]),
    "fevcb_learned_trainer_set_params_v1": (i32, [u64, C.POINTER(C.c_float), u64]),
    "fevcb_learned_trainer_dump_v1": (i32, [u64, u32, C.c_void_p, u32]),
    "fevcb_cmg_aggregate_v1": (i32, [u32, C.POINTER(u32), C.POINTER(u32), C.POINTER(f64), f64, C.POINTER(u32),
                                     C.POINTER(u32)]),
    "fevcb_counter_atoms_v1": (i32, [u64, u64, u64, u32, C.POINTER(u64), C.POINTER(u64), u64, C.POINTER(i64)]),
    "fevcb_engine_exact_limit_v1": (i32, [u64, u64]),
    "fevcb_engine_tuning_v1": (i32, [u64, C.c_void_p, u32]),
    "fevcb_engine_prepare_timings_v1": (i32, [u64, C.c_void_p, u32]),
    "fevcb_numerical_finalize_v1": (i32, [C.c_void_p, C.c_void_p, C.c_void_p, u32]),
    "fevcb_engine_solve_sets_v1": (i32, [u64, C.c_void_p, C.c_void_p, u32, C.c_void_p, u32]),
    "vckss_rust_engine_numerical_preflight_v1": (i32, [C.c_void_p]),
    "vckss_rust_engine_numerical_result_v1": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_numerical_rhs_v1": (i32, [u64, C.c_void_p, u64, C.c_void_p]),
    "vckss_rust_engine_solve_numerical_interrupt_v1": (i32, [u64, C.c_void_p, C.c_void_p, C.c_void_p, u32]),
    "vckss_rust_engine_solve_numerical_v1": (i32, [u64, C.c_void_p]),
    "fevcb_counter_atoms_noalloc_v1": (i32, [u64, u64, u64, u32, C.POINTER(u64), C.POINTER(u64), u64,
                                             C.POINTER(i64)]),
}
SIGNATURES.update({f"vckss_rust_engine_detailed_receipt_v{k}": (i32, [u64, C.c_void_p, u32]) for k in range(1, 8)})

# Reference entry points outside the replaced solve path: schema probes,
# the session last-error alias and UNSUPPORTED_FEATURE returns (csrc/abi_unsupported.cpp).
UNSUPPORTED_SIGNATURES = {
    "vckss_rust_backend_request_capability_v1": (i32, [C.c_void_p, C.c_void_p, u32]),
    "vckss_rust_backend_request_capability_v2": (i32, [C.c_void_p, C.c_void_p, u32]),
    "vckss_rust_centering_schema_v1": (u32, []),
    "vckss_rust_component_inference_interface_version": (u32, []),
    "vckss_rust_engine_admit_prepare_memory_v1": (i32, [C.c_void_p, C.c_void_p, u32]),
    "vckss_rust_engine_admit_prepare_probe_order_v1": (i32, [C.c_void_p, u32]),
    "vckss_rust_engine_admit_prepare_v2": (i32, [C.c_void_p]),
    "vckss_rust_engine_admit_prepare_v3": (i32, [C.c_void_p]),
    "vckss_rust_engine_admit_prepare_v4": (i32, [C.c_void_p, u32]),
    "vckss_rust_engine_augment_component_inference_interrupt_v1": (i32, [u64, C.c_void_p]),
    "vckss_rust_engine_augment_component_inference_interrupt_v2": (i32, [u64, C.c_void_p]),
    "vckss_rust_engine_augment_component_inference_interrupt_v3": (i32, [u64, C.c_void_p]),
    "vckss_rust_engine_augment_component_inference_interrupt_v4": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_augment_component_inference_interrupt_v5": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_augment_match_component_inference_interrupt_v1": (i32, [u64, C.c_void_p]),
    "vckss_rust_engine_augment_match_component_inference_interrupt_v2": (i32, [u64, C.c_void_p]),
    "vckss_rust_engine_augment_match_component_inference_interrupt_v3": (i32, [u64, C.c_void_p]),
    "vckss_rust_engine_augment_match_component_inference_interrupt_v4": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_augment_match_component_inference_interrupt_v5": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_augment_stayers_interrupt_v1": (i32, [u64, C.c_void_p, C.c_void_p]),
    "vckss_rust_engine_augment_stayers_v1": (i32, [u64, C.c_void_p, C.c_void_p]),
    "vckss_rust_engine_component_batch_receipt_v1": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_component_inference_augmentation_receipt_v1": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_component_inference_result_v2": (i32, [u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u32]),
    "vckss_rust_engine_component_inference_result_v3": (i32, [u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u32]),
    "vckss_rust_engine_component_inference_result_v4": (i32, [u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u32]),
    "vckss_rust_engine_component_inference_result_v5": (i32, [u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u64, C.c_void_p, u32]),
    "vckss_rust_engine_component_inference_unit_receipt_v1": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_component_inference_unit_receipt_v2": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_default_component_inference_augmentation_request_interrupt_v1": (i32, [C.c_void_p, u32]),
    "vckss_rust_engine_default_solve_request_interrupt_v2": (i32, [C.c_void_p, u32]),
    "vckss_rust_engine_default_solve_request_interrupt_v3": (i32, [C.c_void_p, u32]),
    "vckss_rust_engine_default_solve_request_interrupt_v4": (i32, [C.c_void_p, u32]),
    "vckss_rust_engine_default_solve_request_interrupt_v6": (i32, [C.c_void_p, u32]),
    "vckss_rust_engine_default_solve_request_interrupt_v7": (i32, [C.c_void_p, u32]),
    "vckss_rust_engine_default_solve_request_v6": (i32, [C.c_void_p, u32]),
    "vckss_rust_engine_default_stayer_augmentation_request_interrupt_v1": (i32, [C.c_void_p, u32]),
    "vckss_rust_engine_exact_execution_receipt_v1": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_execution_plan_receipt_v1": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_full_cmg_model_receipt_v1": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_generic_execution_receipt_v1": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_generic_execution_receipt_v2": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_leaveout_residual_diagnostic_v1": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_memory_forecast_v1": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_memory_policy_v1": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_numerical_cmg_work_v1": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_numerical_preflight_v2": (i32, [C.c_void_p]),
    "vckss_rust_engine_performance_receipt_v1": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_prepare_interrupt_v3": (i32, [C.c_void_p, C.c_void_p, C.c_void_p, u32]),
    "vckss_rust_engine_prepare_memory_interrupt_v1": (i32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, u32]),
    "vckss_rust_engine_repeat_measurement_diagnostic_v1": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_repeat_measurement_leading_v1": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_solve_exact_execution_interrupt_v1": (i32, [u64, C.c_void_p]),
    "vckss_rust_engine_solve_exact_execution_v1": (i32, [u64, C.c_void_p]),
    "vckss_rust_engine_solve_exact_legacy_execution_interrupt_v1": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_solve_exact_resolved_execution_interrupt_v2": (i32, [u64, C.c_void_p]),
    "vckss_rust_engine_solve_exact_resolved_execution_v2": (i32, [u64, C.c_void_p]),
    "vckss_rust_engine_solve_interrupt_v2": (i32, [u64, C.c_void_p]),
    "vckss_rust_engine_solve_interrupt_v3": (i32, [u64, C.c_void_p]),
    "vckss_rust_engine_solve_interrupt_v6": (i32, [u64, C.c_void_p]),
    "vckss_rust_engine_solve_interrupt_v7": (i32, [u64, C.c_void_p]),
    "vckss_rust_engine_solve_numerical_generic_legacy_v2": (i32, [u64, C.c_void_p]),
    "vckss_rust_engine_solve_numerical_interrupt_v2": (i32, [u64, C.c_void_p, C.c_void_p, C.c_void_p, u32]),
    "vckss_rust_engine_solve_numerical_legacy_v2": (i32, [u64, C.c_void_p]),
    "vckss_rust_engine_solve_v2": (i32, [u64, C.c_void_p]),
    "vckss_rust_engine_solve_v3": (i32, [u64, C.c_void_p]),
    "vckss_rust_engine_solve_v6": (i32, [u64, C.c_void_p]),
    "vckss_rust_engine_stayer_augmentation_receipt_v1": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_engine_stayer_hybrid_result_v1": (i32, [u64, C.c_void_p, u32]),
    "vckss_rust_exact_execution_schema_v1": (u32, []),
    "vckss_rust_exact_legacy_execution_schema_v1": (u32, []),
    "vckss_rust_exact_resolved_execution_schema_v2": (u32, []),
    "vckss_rust_numerical_schema_v1": (u32, []),
    "vckss_rust_numerical_schema_v2": (u32, []),
    "vckss_rust_report_call_v1": (i32, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "vckss_rust_session_clear_abandoned_v1": (i32, []),
    "vckss_rust_session_last_error": (C.c_char_p, []),
    "vckss_rust_session_preparation_receipt_v1": (i32, [u64, C.c_void_p]),
    "vckss_rust_session_prepare_v1": (i32, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "vckss_rust_session_release_v1": (i32, [u64]),
    "vckss_rust_session_snapshot_v1": (i32, [C.c_void_p]),
}
SIGNATURES.update(UNSUPPORTED_SIGNATURES)

def capability_signature_v3(req: SolveRequestV4, controls_count: int) -> int:
    """Request signature that V4+ solves must carry: FNV-1a over the request's
    capability fields (reference vckss-plugin/src/ffi_engine.rs:9492-9532,
    field mapping ffi_engine.rs:10425-10460)."""
    h = 0xCBF29CE484222325

    def eat(data: bytes):
        nonlocal h
        for b in data:
            h ^= b
            h = (h * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF

    v3, v2, v1 = req.v3, req.v3.v2, req.v3.v2.v1
    eat(b"VCKSS-REQUEST-CAPABILITY-V3")
    for v in (v3.capability_schema, v2.algorithm, v1.deletion_mode, v2.nuisance_mode, v1.solver_route,
              v1.rng_contract, controls_count, v3.frequency_use, v3.engine, v3.batch_mode, v3.stayers_mode,
              v3.target_weight_mode, v3.deletion_unit_source, v3.probeorder_supplied, v3.wallseconds_supplied,
              req.leverage_batch_mode, req.target_batch_mode, v1.allow_automatic_cmg_setup_fallback):
        eat(int(v).to_bytes(4, "little"))
    eat(int(v3.physical_limit).to_bytes(8, "little"))
    eat(C.c_uint64.from_buffer_copy(C.c_double(req.wallseconds)).value.to_bytes(8, "little"))
    return h


LIBRARY_PATH = Path(__file__).resolve().parent / "libfevc_b200.so"


class EngineError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code
        self.message = message


def load(path: str | os.PathLike | None = None, *, bind_extensions: bool = True) -> C.CDLL:
    """Load a library exporting the plugin ABI (default: the in-tree build)."""
    path = Path(path) if path else LIBRARY_PATH
    if not path.exists():
        raise FileNotFoundError(f"{path} is missing; run fevc_b200/build.py (or __graft_entry__.build())")
    lib = C.CDLL(str(path), mode=os.RTLD_LOCAL | getattr(os, "RTLD_NOW", 2))
    for name, (res, args) in SIGNATURES.items():
        if name.startswith("fevcb_") and not bind_extensions:
            continue
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def _d(a: np.ndarray):
    return a.ctypes.data_as(dptr)


class Engine:
    """One prepare/solve/result/release cycle against a plugin-ABI library."""

    def __init__(self, lib: C.CDLL):
        self.lib = lib
        self.generation = 0
        self._keep = []

    def check(self, status: int) -> None:
        if status != 0:
            msg = self.lib.vckss_rust_engine_last_error()
            raise EngineError(status, msg.decode() if msg else "")

    # ---- preparation
    def prepare(self, panel, *, deletion_mode: int = 1, implicit_match: bool = False, cleanup: bool = True,
                use_v4: bool | None = None) -> int:
        cols = [np.ascontiguousarray(x, dtype=np.float64) for x in (
            panel.worker, panel.firm, panel.deletion, panel.outcome, panel.frequency, panel.target_weight)]
        controls = [np.ascontiguousarray(c, dtype=np.float64) for c in getattr(panel, "controls", [])]
        self._keep = cols + controls
        rows = cols[0].shape[0]
        c1 = ColumnsV1(C.sizeof(ColumnsV1), 0, rows, *[_d(x) for x in cols])
        handle = u64(0)
        if use_v4 is None:
            use_v4 = bool(controls) or deletion_mode != 1 or implicit_match
        if not use_v4:
            req = PrepareRequestV1(1, C.sizeof(PrepareRequestV1), rows, int(cleanup), 0)
            self.check(self.lib.vckss_rust_engine_prepare_v1(C.byref(req), C.byref(c1), C.byref(handle), 8))
        else:
            c1.struct_size = C.sizeof(ColumnsV3)
            ctl_array = (dptr * max(1, len(controls)))(*[_d(c) for c in controls])
            self._keep.append(ctl_array)
            c2 = ColumnsV2(c1, C.cast(ctl_array, C.POINTER(dptr)) if controls else None, len(controls), 0)
            c3 = ColumnsV3(c2, None, 0, 0)
            v2 = PrepareRequestV2(1, C.sizeof(PrepareRequestInterruptV3), rows, int(cleanup), 0, 1 << 40,
                                  rows * (6 + len(controls)) * 8)
            v3 = PrepareRequestV3(v2, deletion_mode, len(controls), 0)
            v4 = PrepareRequestV4(v3, int(implicit_match), 0)
            req = PrepareRequestInterruptV3(v4, InterruptPoll(0), None, 0, 0)
            self.check(self.lib.vckss_rust_engine_prepare_interrupt_v4(C.byref(req), C.byref(c3), C.byref(handle), 8))
        self.generation = handle.value
        return self.generation

    def centering(self, mode: int) -> None:
        self.check(self.lib.vckss_rust_engine_centering_v1(self.generation, mode))

    def receipt(self) -> dict:
        r = PreparationReceiptV4()
        self.check(self.lib.vckss_rust_engine_preparation_receipt_v4(self.generation, C.byref(r), C.sizeof(r)))
        d = r.v3.v2.as_dict()
        d["target_weight_sum"] = r.v3.target_weight_sum
        d["controls_count"] = r.controls_count
        d["deletion_mode"] = r.deletion_mode
        return d

    def retained_mask(self, rows: int) -> np.ndarray:
        out = np.zeros(rows, np.uint8)
        self.check(self.lib.vckss_rust_engine_retained_mask_v1(self.generation, out.ctypes.data_as(C.c_void_p), rows))
        return out

    # ---- solve
    def default_request(self) -> SolveRequestV1:
        req = SolveRequestV1()
        self.check(self.lib.vckss_rust_engine_default_solve_request_v1(C.byref(req), C.sizeof(req)))
        return req

    def solve(self, req: SolveRequestV1) -> None:
        self.check(self.lib.vckss_rust_engine_solve_v1(self.generation, C.byref(req)))

    def default_request_v5(self, deletion_mode: int = 1) -> SolveRequestV5:
        """The library's default V5 request; deletion_mode 2 also sets the
        observation-row deletion-unit source its capability check requires."""
        req = SolveRequestV5()
        self.check(self.lib.vckss_rust_engine_default_solve_request_v5(C.byref(req), C.sizeof(req)))
        if deletion_mode == 2:
            req.v4.v3.v2.v1.deletion_mode = 2
            req.v4.v3.deletion_unit_source = 3
        return req

    def exact_request_v5(self, limit: int = 2000) -> SolveRequestV5:
        """A V5 request for the exact estimator (algorithm EXACT, no RNG
        contract, automatic engine and route, identified-dimension limit)."""
        req = self.default_request_v5(1)
        req.v4.v3.v2.algorithm = 1
        req.v4.v3.v2.v1.rng_contract = 0
        req.v4.v3.v2.exact_estimator_limit = limit
        return req

    def exact_ceiling(self, ceiling: int) -> None:
        """Raise this generation's exact-estimator dimension ceiling above the
        request limit (fevcb_engine_exact_limit_v1)."""
        self.check(self.lib.fevcb_engine_exact_limit_v1(self.generation, ceiling))

    def solve_v5(self, req: SolveRequestV5, controls_count: int = 0) -> None:
        req.v4.v3.request_signature = capability_signature_v3(req.v4, controls_count)
        self.check(self.lib.vckss_rust_engine_solve_v5(self.generation, C.byref(req)))

    def solve_sets(self, req: SolveRequestV5, sets: list[tuple[int, int]], controls_count: int = 0) -> list[dict]:
        """Probe sets (seed, probes) in one call (fevcb_engine_solve_sets_v1);
        the first set's result becomes the generation's result."""
        req.v4.v3.request_signature = capability_signature_v3(req.v4, controls_count)
        arr = (ProbeSetV1 * len(sets))(*[ProbeSetV1(int(s), int(p), 0) for s, p in sets])
        out = (ProbeSetResultV1 * len(sets))()
        self.check(self.lib.fevcb_engine_solve_sets_v1(self.generation, C.byref(req), arr, len(sets), out,
                                                      C.sizeof(out)))
        return [{k: getattr(o, k).tuple() for k in ("plugin", "correction", "corrected", "numerical_mcse")}
                for o in out]

    def numerical_request(self, point: SolveRequestV5, controls_count: int = 0) -> NumericalRequestV1:
        """A numerical-attachment request around a V5 request's V4 point
        (signature reconciled for controls_count)."""
        point.v4.v3.request_signature = capability_signature_v3(point.v4, controls_count)
        return NumericalRequestV1(1, C.sizeof(NumericalRequestV1), 1, max(1, int(point.threads)),
                                  int(point.tolerance_supplied), 0, 0, 0, controls_count, 0, point.v4)

    def solve_numerical(self, req: NumericalRequestV1) -> None:
        self.check(self.lib.vckss_rust_engine_solve_numerical_v1(self.generation, C.byref(req)))

    def numerical_result(self) -> dict:
        r = NumericalResultV1()
        self.check(self.lib.vckss_rust_engine_numerical_result_v1(self.generation, C.byref(r), C.sizeof(r)))
        d = {}
        for name, _ in NumericalResultV1._fields_:
            v = getattr(r, name)
            d[name] = list(v) if hasattr(v, "__len__") else v
        return d

    def numerical_rhs(self, rows: int) -> tuple[int, list[dict]]:
        arr = (NumericalRhsV1 * max(rows, 1))()
        count = u64(0)
        self.check(self.lib.vckss_rust_engine_numerical_rhs_v1(self.generation, arr, rows, C.byref(count)))
        return count.value, [arr[i].as_dict() for i in range(min(rows, count.value))]

    # ---- fixed-effect projection attachment
    def augment_projection(self, columns, effect: int = 1, weight: int = 1, rank_tolerance: float = 1e-10) -> None:
        """Attach a projection of the worker (effect 1) or firm (2) effect on
        the given covariates (one float64 array per covariate, one value per
        retained row), weighted by frequency (1) or target weight (2)."""
        cols = [np.ascontiguousarray(c, dtype=np.float64) for c in columns]
        rows = len(cols[0])
        q = ProjectionAugmentationRequestInterruptV1()
        self.check(self.lib.vckss_rust_engine_default_projection_augmentation_request_interrupt_v1(
            C.byref(q), C.sizeof(q)))
        q.options.rows = rows
        q.options.project_count = len(cols)
        q.options.effect = effect
        q.options.weight = weight
        q.options.rank_tolerance = rank_tolerance
        q.options.caller_copy_bytes = rows * len(cols) * 8
        ptrs = (C.POINTER(f64) * len(cols))(*[c.ctypes.data_as(C.POINTER(f64)) for c in cols])
        d = ProjectionColumnsV1(C.sizeof(ProjectionColumnsV1), 0, rows, ptrs, len(cols), 0)
        self.check(self.lib.vckss_rust_engine_augment_projection_interrupt_v1(self.generation, C.byref(q), C.byref(d)))

    def projection_augmentation_receipt(self) -> dict:
        r = ProjectionAugmentationReceiptV1()
        self.check(self.lib.vckss_rust_engine_projection_augmentation_receipt_v1(self.generation, C.byref(r),
                                                                                C.sizeof(r)))
        return r.as_dict()

    def projection_result(self) -> dict:
        """Coefficients, KSS and naive covariances (columns x columns) and the
        result receipt of the last solve's projection."""
        r = ProjectionResultReceiptV1()
        self.check(self.lib.vckss_rust_engine_projection_result_receipt_v1(self.generation, C.byref(r), C.sizeof(r)))
        n = int(r.columns)
        coef, cov, naive = np.zeros(n), np.zeros(n * n), np.zeros(n * n)
        p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
        self.check(self.lib.vckss_rust_engine_projection_result_v1(self.generation, p(coef), n, p(cov), n * n,
                                                                   p(naive), n * n, C.byref(r), C.sizeof(r)))
        return {"coefficients": coef.tolist(), "covariance": cov.reshape(n, n).tolist(),
                "naive_covariance": naive.reshape(n, n).tolist(), "receipt": r.as_dict()}

    def result(self) -> dict:
        r = ResultV1()
        self.check(self.lib.vckss_rust_engine_result_v1(self.generation, C.byref(r), C.sizeof(r)))
        return {k: getattr(r, k).tuple() for k in ("plugin", "correction", "corrected", "numerical_mcse")}

    def rhs_receipts(self, count: int) -> list[dict]:
        arr = (RhsReceiptV1 * count)()
        self.check(self.lib.vckss_rust_engine_rhs_receipts_v1(self.generation, arr, count))
        return [a.as_dict() for a in arr]

    def release(self) -> None:
        if self.generation:
            self.check(self.lib.vckss_rust_engine_release_v1(self.generation))
            self.generation = 0

    # ---- B200 extensions
    def device_options(self, block_columns: int = 0, preconditioner: int = 0, precision: int = 0) -> None:
        """Device solve options: block width, preconditioner (1 Jacobi, 2 CMG,
        3 the learned per-vertex degree-1 stage, 4 the same stage with uniform
        weights) and precision (1: single-precision residual, direction and
        products with a double solution, double reductions and residual
        replacement)."""
        o = FevcbSolveOptionsV2(FevcbSolveOptionsV1(C.sizeof(FevcbSolveOptionsV2), block_columns, preconditioner, 1),
                                precision, 0)
        self.check(self.lib.fevcb_engine_solve_options_v1(self.generation, C.byref(o)))

    def detailed_receipt(self, version: int = 7):
        cls = globals()[f"EngineDetailedReceiptV{version}"]
        out = cls()
        self.check(getattr(self.lib, f"vckss_rust_engine_detailed_receipt_v{version}")(
            self.generation, C.byref(out), C.sizeof(out)))
        return out

    def setup_timings(self) -> dict:
        """Wall milliseconds of the device engine's setup (builders, device
        units, hybrid assembly, preconditioner, total)."""
        t = FevcbSetupTimingsV1()
        self.check(self.lib.fevcb_engine_setup_timings_v1(self.generation, C.byref(t), C.sizeof(t)))
        d = t.as_dict()
        names = ("cells", "units", "strata", "strata_scale", "strata_keys", "rows", "groups") + tuple(
            f"control_{k}" for k in range(9))
        d["builder_ms"] = {names[i]: round(list(t.builder_ms)[i], 2) for i in range(min(t.builders, 16))}
        return d

    def timings(self) -> dict:
        t = FevcbSolveTimingsV1()
        self.check(self.lib.fevcb_engine_timings_v1(self.generation, C.byref(t), C.sizeof(t)))
        return t.as_dict()

    def tuning(self) -> dict:
        """The autotuner's candidates and choice (precision option 2)."""
        t = FevcbTuningV1()
        self.check(self.lib.fevcb_engine_tuning_v1(self.generation, C.byref(t), C.sizeof(t)))
        n = t.candidates
        return {"chosen": t.chosen, "candidates": [
            {"precision": t.precision[c], "preconditioner": t.preconditioner[c], "ms": t.milliseconds[c]}
            for c in range(n)]}

    def prepare_timings(self) -> dict:
        """Host preparation wall time by phase, milliseconds."""
        t = FevcbPrepareTimingsV1()
        self.check(self.lib.fevcb_engine_prepare_timings_v1(self.generation, C.byref(t), C.sizeof(t)))
        return {k: getattr(t, k) for k, _ in FevcbPrepareTimingsV1._fields_ if k != "struct_size"}

    def resolve(self) -> None:
        self.check(self.lib.fevcb_engine_resolve_v1(self.generation))

    def kernel_benchmark(self, kernel: int, block_columns: int, launches: int) -> tuple[float, float]:
        ms, nbytes = f64(0), f64(0)
        self.check(self.lib.fevcb_engine_kernel_benchmark_v1(self.generation, kernel, block_columns, launches,
                                                             C.byref(ms), C.byref(nbytes)))
        return ms.value, nbytes.value

    def cmg_summary(self, eliminate_max_degree: int = 0) -> dict:
        """Host-built CMG hierarchy of this generation (no GPU needed)."""
        out = CmgSummaryV1()
        self.check(self.lib.fevcb_engine_cmg_summary_v1(self.generation, eliminate_max_degree, C.byref(out),
                                                        C.sizeof(out)))
        L = int(out.hierarchy_levels)
        return {"vertices": int(out.vertices), "edges": int(out.edges), "hierarchy_levels": L,
                "terminal_vertices": int(out.terminal_vertices), "terminal_reason": int(out.terminal_reason),
                "level_vertices": list(out.level_vertices[:L]), "level_edges": list(out.level_edges[:L]),
                "level_repeat": list(out.level_repeat[:max(L - 1, 0)])}

    def unit_detail(self, units: int, cells: int, probes: int) -> dict:
        names = ("projection_share", "residual_share", "finite_bias", "finite_variance", "residual_mass",
                 "deleted_mass")
        arrs = {n: np.zeros(units) for n in names}
        fitted, omega, draws = np.zeros(cells), np.zeros(cells), np.zeros(4 * probes)
        self.check(self.lib.fevcb_engine_unit_detail_v1(
            self.generation, units, *[_d(arrs[n]) for n in names], cells, _d(fitted), _d(omega), probes, _d(draws)))
        arrs["fitted_cell"] = fitted
        arrs["cell_correction_weight"] = omega
        arrs["target_draws"] = draws.reshape(probes, 4)
        return arrs


def device_atoms(lib: C.CDLL, seed: int, tag: int, first_probe: int, columns: int, entity, trials,
                 *, no_alloc: bool = False) -> np.ndarray:
    """Counter-V1 atoms computed on the device (``no_alloc`` selects the
    entry point that stages through the library's fixed device array)."""
    entity = np.ascontiguousarray(entity, dtype=np.uint64)
    trials = np.ascontiguousarray(trials, dtype=np.uint64)
    out = np.zeros(entity.size * columns, np.int64)
    fn = lib.fevcb_counter_atoms_noalloc_v1 if no_alloc else lib.fevcb_counter_atoms_v1
    st = fn(seed, tag, first_probe, columns, entity.ctypes.data_as(C.POINTER(u64)),
                                    trials.ctypes.data_as(C.POINTER(u64)), entity.size,
                                    out.ctypes.data_as(C.POINTER(i64)))
    if st != 0:
        raise EngineError(st, lib.vckss_rust_engine_last_error().decode())
    return out.reshape(entity.size, columns)
