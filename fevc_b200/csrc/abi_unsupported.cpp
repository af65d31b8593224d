// Entry points of the reference ABI outside the solve path this library
// replaces (rust/stata_backend/include/vckss_rust.h).  Schema probes report
// availability, the session last-error text is the engine's, and every
// other call returns UNSUPPORTED_FEATURE with its name in the error text.
#include "fevc_b200.h"

namespace fevcb {
int32_t unsupported_entry(const char* name);
}  // namespace fevcb

extern "C" {

int32_t vckss_rust_backend_request_capability_v1(const VckssBackendRequestCapabilityRequestV1 *, VckssBackendRequestCapabilityReceiptV1 *, uint32_t) { return fevcb::unsupported_entry("backend_request_capability_v1"); }
int32_t vckss_rust_backend_request_capability_v2(const VckssBackendRequestCapabilityRequestV2 *, VckssBackendRequestCapabilityReceiptV2 *, uint32_t) { return fevcb::unsupported_entry("backend_request_capability_v2"); }
uint32_t vckss_rust_centering_schema_v1(void) { return 1; }  // engine_centering_v1 is provided
uint32_t vckss_rust_component_inference_interface_version(void) { return 0; }  // component inference is not provided
int32_t vckss_rust_engine_admit_prepare_memory_v1(const VckssEnginePrepareRequestV4 *, const VckssMemoryPolicyV1 *, uint32_t) { return fevcb::unsupported_entry("engine_admit_prepare_memory_v1"); }
int32_t vckss_rust_engine_admit_prepare_probe_order_v1(const VckssEnginePrepareRequestV3 *, uint32_t) { return fevcb::unsupported_entry("engine_admit_prepare_probe_order_v1"); }
int32_t vckss_rust_engine_admit_prepare_v2(const VckssEnginePrepareRequestV2 *) { return fevcb::unsupported_entry("engine_admit_prepare_v2"); }
int32_t vckss_rust_engine_admit_prepare_v3(const VckssEnginePrepareRequestV3 *) { return fevcb::unsupported_entry("engine_admit_prepare_v3"); }
int32_t vckss_rust_engine_admit_prepare_v4(const VckssEnginePrepareRequestV4 *, uint32_t) { return fevcb::unsupported_entry("engine_admit_prepare_v4"); }
int32_t vckss_rust_engine_augment_component_inference_interrupt_v1(uint64_t, const VckssComponentInferenceAugmentationRequestInterruptV1 *) { return fevcb::unsupported_entry("engine_augment_component_inference_interrupt_v1"); }
int32_t vckss_rust_engine_augment_component_inference_interrupt_v2(uint64_t, const VckssComponentInferenceAugmentationRequestInterruptV1 *) { return fevcb::unsupported_entry("engine_augment_component_inference_interrupt_v2"); }
int32_t vckss_rust_engine_augment_component_inference_interrupt_v3(uint64_t, const VckssComponentInferenceAugmentationRequestInterruptV1 *) { return fevcb::unsupported_entry("engine_augment_component_inference_interrupt_v3"); }
int32_t vckss_rust_engine_augment_component_inference_interrupt_v4(uint64_t, const VckssComponentInferenceAugmentationRequestInterruptV1 *, uint32_t) { return fevcb::unsupported_entry("engine_augment_component_inference_interrupt_v4"); }
int32_t vckss_rust_engine_augment_component_inference_interrupt_v5(uint64_t, const VckssComponentInferenceAugmentationRequestInterruptV1 *, uint32_t) { return fevcb::unsupported_entry("engine_augment_component_inference_interrupt_v5"); }
int32_t vckss_rust_engine_augment_match_component_inference_interrupt_v1(uint64_t, const VckssComponentInferenceAugmentationRequestInterruptV1 *) { return fevcb::unsupported_entry("engine_augment_match_component_inference_interrupt_v1"); }
int32_t vckss_rust_engine_augment_match_component_inference_interrupt_v2(uint64_t, const VckssComponentInferenceAugmentationRequestInterruptV1 *) { return fevcb::unsupported_entry("engine_augment_match_component_inference_interrupt_v2"); }
int32_t vckss_rust_engine_augment_match_component_inference_interrupt_v3(uint64_t, const VckssComponentInferenceAugmentationRequestInterruptV1 *) { return fevcb::unsupported_entry("engine_augment_match_component_inference_interrupt_v3"); }
int32_t vckss_rust_engine_augment_match_component_inference_interrupt_v4(uint64_t, const VckssComponentInferenceAugmentationRequestInterruptV1 *, uint32_t) { return fevcb::unsupported_entry("engine_augment_match_component_inference_interrupt_v4"); }
int32_t vckss_rust_engine_augment_match_component_inference_interrupt_v5(uint64_t, const VckssComponentInferenceAugmentationRequestInterruptV1 *, uint32_t) { return fevcb::unsupported_entry("engine_augment_match_component_inference_interrupt_v5"); }
int32_t vckss_rust_engine_augment_stayers_interrupt_v1(uint64_t, const VckssStayerAugmentationRequestInterruptV1 *, const VckssStayerAugmentationColumnsV1 *) { return fevcb::unsupported_entry("engine_augment_stayers_interrupt_v1"); }
int32_t vckss_rust_engine_augment_stayers_v1(uint64_t, const VckssStayerAugmentationRequestV1 *, const VckssStayerAugmentationColumnsV1 *) { return fevcb::unsupported_entry("engine_augment_stayers_v1"); }
int32_t vckss_rust_engine_component_batch_receipt_v1(uint64_t, VckssComponentBatchReceiptV1 *, uint32_t) { return fevcb::unsupported_entry("engine_component_batch_receipt_v1"); }
int32_t vckss_rust_engine_component_inference_augmentation_receipt_v1(uint64_t, VckssComponentInferenceAugmentationReceiptV1 *, uint32_t) { return fevcb::unsupported_entry("engine_component_inference_augmentation_receipt_v1"); }
int32_t vckss_rust_engine_component_inference_result_v2(uint64_t, double *, uint64_t, double *, uint64_t, double *, uint64_t, double *, uint64_t, double *, uint64_t, double *, uint64_t, double *, uint64_t, double *, uint64_t, VckssComponentInferenceResultReceiptV2 *, uint32_t) { return fevcb::unsupported_entry("engine_component_inference_result_v2"); }
int32_t vckss_rust_engine_component_inference_result_v3(uint64_t, double *, uint64_t, double *, uint64_t, double *, uint64_t, double *, uint64_t, double *, uint64_t, double *, uint64_t, double *, uint64_t, double *, uint64_t, VckssComponentInferenceResultReceiptV3 *, uint32_t) { return fevcb::unsupported_entry("engine_component_inference_result_v3"); }
int32_t vckss_rust_engine_component_inference_result_v4(uint64_t, double *, uint64_t, double *, uint64_t, double *, uint64_t, double *, uint64_t, double *, uint64_t, double *, uint64_t, double *, uint64_t, double *, uint64_t, VckssComponentInferenceResultReceiptV4 *, uint32_t) { return fevcb::unsupported_entry("engine_component_inference_result_v4"); }
int32_t vckss_rust_engine_component_inference_result_v5(uint64_t, double *, uint64_t, double *, uint64_t, double *, uint64_t, double *, uint64_t, double *, uint64_t, double *, uint64_t, double *, uint64_t, double *, uint64_t, double *, uint64_t, VckssComponentInferenceResultReceiptV5 *, uint32_t) { return fevcb::unsupported_entry("engine_component_inference_result_v5"); }
int32_t vckss_rust_engine_component_inference_unit_receipt_v1(uint64_t, VckssComponentInferenceUnitReceiptV1 *, uint32_t) { return fevcb::unsupported_entry("engine_component_inference_unit_receipt_v1"); }
int32_t vckss_rust_engine_component_inference_unit_receipt_v2(uint64_t, VckssComponentInferenceUnitReceiptV2 *, uint32_t) { return fevcb::unsupported_entry("engine_component_inference_unit_receipt_v2"); }
int32_t vckss_rust_engine_default_component_inference_augmentation_request_interrupt_v1(VckssComponentInferenceAugmentationRequestInterruptV1 *, uint32_t) { return fevcb::unsupported_entry("engine_default_component_inference_augmentation_request_interrupt_v1"); }
int32_t vckss_rust_engine_default_solve_request_interrupt_v2(VckssEngineSolveRequestInterruptV2 *, uint32_t) { return fevcb::unsupported_entry("engine_default_solve_request_interrupt_v2"); }
int32_t vckss_rust_engine_default_solve_request_interrupt_v3(VckssEngineSolveRequestInterruptV3 *, uint32_t) { return fevcb::unsupported_entry("engine_default_solve_request_interrupt_v3"); }
int32_t vckss_rust_engine_default_solve_request_interrupt_v4(VckssEngineSolveRequestInterruptV4 *, uint32_t) { return fevcb::unsupported_entry("engine_default_solve_request_interrupt_v4"); }
int32_t vckss_rust_engine_default_solve_request_interrupt_v6(VckssEngineSolveRequestInterruptV6 *, uint32_t) { return fevcb::unsupported_entry("engine_default_solve_request_interrupt_v6"); }
int32_t vckss_rust_engine_default_solve_request_interrupt_v7(VckssEngineSolveRequestInterruptV7 *, uint32_t) { return fevcb::unsupported_entry("engine_default_solve_request_interrupt_v7"); }
int32_t vckss_rust_engine_default_solve_request_v6(VckssEngineSolveRequestV6 *, uint32_t) { return fevcb::unsupported_entry("engine_default_solve_request_v6"); }
int32_t vckss_rust_engine_default_stayer_augmentation_request_interrupt_v1(VckssStayerAugmentationRequestInterruptV1 *, uint32_t) { return fevcb::unsupported_entry("engine_default_stayer_augmentation_request_interrupt_v1"); }
int32_t vckss_rust_engine_exact_execution_receipt_v1(uint64_t, VckssExactExecutionReceiptV1 *, uint32_t) { return fevcb::unsupported_entry("engine_exact_execution_receipt_v1"); }
int32_t vckss_rust_engine_execution_plan_receipt_v1(uint64_t, VckssExecutionPlanReceiptV1 *, uint32_t) { return fevcb::unsupported_entry("engine_execution_plan_receipt_v1"); }
int32_t vckss_rust_engine_full_cmg_model_receipt_v1(uint64_t, VckssFullCmgModelReceiptV1 *, uint32_t) { return fevcb::unsupported_entry("engine_full_cmg_model_receipt_v1"); }
int32_t vckss_rust_engine_generic_execution_receipt_v1(uint64_t, VckssGenericExecutionReceiptV1 *, uint32_t) { return fevcb::unsupported_entry("engine_generic_execution_receipt_v1"); }
int32_t vckss_rust_engine_generic_execution_receipt_v2(uint64_t, VckssGenericExecutionReceiptV2 *, uint32_t) { return fevcb::unsupported_entry("engine_generic_execution_receipt_v2"); }
int32_t vckss_rust_engine_leaveout_residual_diagnostic_v1(uint64_t, VckssLeaveoutResidualDiagnosticV1 *, uint32_t) { return fevcb::unsupported_entry("engine_leaveout_residual_diagnostic_v1"); }
int32_t vckss_rust_engine_memory_forecast_v1(uint64_t, VckssMemoryForecastV1 *, uint32_t) { return fevcb::unsupported_entry("engine_memory_forecast_v1"); }
int32_t vckss_rust_engine_memory_policy_v1(uint64_t, VckssMemoryPolicyV1 *, uint32_t) { return fevcb::unsupported_entry("engine_memory_policy_v1"); }
int32_t vckss_rust_engine_numerical_cmg_work_v1(uint64_t, VckssFullCmgModelReceiptV1 *, uint32_t) { return fevcb::unsupported_entry("engine_numerical_cmg_work_v1"); }
int32_t vckss_rust_engine_numerical_preflight_v2(const VckssNumericalRequestV2 *) { return fevcb::unsupported_entry("engine_numerical_preflight_v2"); }
int32_t vckss_rust_engine_performance_receipt_v1(uint64_t, VckssEnginePerformanceReceiptV1 *, uint32_t) { return fevcb::unsupported_entry("engine_performance_receipt_v1"); }
int32_t vckss_rust_engine_prepare_interrupt_v3(const VckssEnginePrepareRequestInterruptV2 *, const VckssEngineColumnsV3 *, uint64_t *, uint32_t) { return fevcb::unsupported_entry("engine_prepare_interrupt_v3"); }
int32_t vckss_rust_engine_prepare_memory_interrupt_v1(const VckssEnginePrepareRequestInterruptV3 *, const VckssEngineColumnsV3 *, const VckssMemoryPolicyV1 *, uint64_t *, uint32_t) { return fevcb::unsupported_entry("engine_prepare_memory_interrupt_v1"); }
int32_t vckss_rust_engine_repeat_measurement_diagnostic_v1(uint64_t, VckssRepeatMeasurementDiagnosticV1 *, uint32_t) { return fevcb::unsupported_entry("engine_repeat_measurement_diagnostic_v1"); }
int32_t vckss_rust_engine_repeat_measurement_leading_v1(uint64_t, VckssRepeatMeasurementLeadingV1 *, uint32_t) { return fevcb::unsupported_entry("engine_repeat_measurement_leading_v1"); }
int32_t vckss_rust_engine_solve_exact_execution_interrupt_v1(uint64_t, const VckssExactExecutionRequestInterruptV1 *) { return fevcb::unsupported_entry("engine_solve_exact_execution_interrupt_v1"); }
int32_t vckss_rust_engine_solve_exact_execution_v1(uint64_t, const VckssExactExecutionRequestV1 *) { return fevcb::unsupported_entry("engine_solve_exact_execution_v1"); }
int32_t vckss_rust_engine_solve_exact_legacy_execution_interrupt_v1(uint64_t, const VckssEngineSolveRequestInterruptV2 *, uint32_t) { return fevcb::unsupported_entry("engine_solve_exact_legacy_execution_interrupt_v1"); }
int32_t vckss_rust_engine_solve_exact_resolved_execution_interrupt_v2(uint64_t, const VckssExactExecutionRequestInterruptV1 *) { return fevcb::unsupported_entry("engine_solve_exact_resolved_execution_interrupt_v2"); }
int32_t vckss_rust_engine_solve_exact_resolved_execution_v2(uint64_t, const VckssExactExecutionRequestV1 *) { return fevcb::unsupported_entry("engine_solve_exact_resolved_execution_v2"); }
int32_t vckss_rust_engine_solve_interrupt_v2(uint64_t, const VckssEngineSolveRequestInterruptV2 *) { return fevcb::unsupported_entry("engine_solve_interrupt_v2"); }
int32_t vckss_rust_engine_solve_interrupt_v3(uint64_t, const VckssEngineSolveRequestInterruptV3 *) { return fevcb::unsupported_entry("engine_solve_interrupt_v3"); }
int32_t vckss_rust_engine_solve_interrupt_v6(uint64_t, const VckssEngineSolveRequestInterruptV6 *) { return fevcb::unsupported_entry("engine_solve_interrupt_v6"); }
int32_t vckss_rust_engine_solve_interrupt_v7(uint64_t, const VckssEngineSolveRequestInterruptV7 *) { return fevcb::unsupported_entry("engine_solve_interrupt_v7"); }
int32_t vckss_rust_engine_solve_numerical_generic_legacy_v2(uint64_t, const VckssEngineSolveRequestInterruptV3 *) { return fevcb::unsupported_entry("engine_solve_numerical_generic_legacy_v2"); }
int32_t vckss_rust_engine_solve_numerical_interrupt_v2(uint64_t, const VckssNumericalRequestV2 *, VckssInterruptPollV1, void *, uint32_t) { return fevcb::unsupported_entry("engine_solve_numerical_interrupt_v2"); }
int32_t vckss_rust_engine_solve_numerical_legacy_v2(uint64_t, const VckssEngineSolveRequestInterruptV2 *) { return fevcb::unsupported_entry("engine_solve_numerical_legacy_v2"); }
int32_t vckss_rust_engine_solve_v2(uint64_t, const VckssEngineSolveRequestV2 *) { return fevcb::unsupported_entry("engine_solve_v2"); }
int32_t vckss_rust_engine_solve_v3(uint64_t, const VckssEngineSolveRequestV3 *) { return fevcb::unsupported_entry("engine_solve_v3"); }
int32_t vckss_rust_engine_solve_v6(uint64_t, const VckssEngineSolveRequestV6 *) { return fevcb::unsupported_entry("engine_solve_v6"); }
int32_t vckss_rust_engine_stayer_augmentation_receipt_v1(uint64_t, VckssStayerAugmentationReceiptV1 *, uint32_t) { return fevcb::unsupported_entry("engine_stayer_augmentation_receipt_v1"); }
int32_t vckss_rust_engine_stayer_hybrid_result_v1(uint64_t, VckssStayerHybridResultV1 *, uint32_t) { return fevcb::unsupported_entry("engine_stayer_hybrid_result_v1"); }
uint32_t vckss_rust_exact_execution_schema_v1(void) { return 0; }  // exact execution is not provided
uint32_t vckss_rust_exact_legacy_execution_schema_v1(void) { return 0; }  // exact execution is not provided
uint32_t vckss_rust_exact_resolved_execution_schema_v2(void) { return 0; }  // exact execution is not provided
uint32_t vckss_rust_numerical_schema_v2(void) { return 0; }  // the numerical attachment is not provided
int32_t vckss_rust_report_call_v1(const VckssProgressOptionsV1 *, VckssProgressOperationV1, void *) { return fevcb::unsupported_entry("report_call_v1"); }
int32_t vckss_rust_session_clear_abandoned_v1(void) { return fevcb::unsupported_entry("session_clear_abandoned_v1"); }
const char* vckss_rust_session_last_error(void) { return vckss_rust_engine_last_error(); }
int32_t vckss_rust_session_preparation_receipt_v1(uint64_t, VckssPreparationReceiptV1 *) { return fevcb::unsupported_entry("session_preparation_receipt_v1"); }
int32_t vckss_rust_session_prepare_v1(const VckssPrepareRequestV1 *, const VckssColumnsV1 *, uint64_t *) { return fevcb::unsupported_entry("session_prepare_v1"); }
int32_t vckss_rust_session_release_v1(uint64_t) { return fevcb::unsupported_entry("session_release_v1"); }
int32_t vckss_rust_session_snapshot_v1(VckssSessionSnapshotV1 *) { return fevcb::unsupported_entry("session_snapshot_v1"); }

}  // extern "C"
