// Host preparation: ingest validation, canonical re-densification, graph
// pruning to the leave-out connected set, compression to coefficient cells and
// the JLA semantic plan.  Everything here is integer / ordering work whose
// output must be bit-identical to the reference plugin's preparation, because
// the semantic ranks become Counter-V1 entity keys.
#pragma once

#include <cstdint>
#include <vector>

#include "common.h"

namespace fevcb {

enum class Deletion : uint32_t { Match = 1, Observation = 2 };

struct InputColumns {
  std::vector<uint64_t> worker, firm, deletion, frequency;
  std::vector<double> outcome, target;
  std::vector<std::vector<double>> controls;
  std::vector<double> probe_order;  // empty unless supplied
};

struct Canonical {
  std::vector<uint32_t> worker, firm, deletion;
  size_t workers = 0, firms = 0, deletion_units = 0;
  // distinct (worker, firm) coordinates in (worker, firm) order and the
  // coordinate of every row
  std::vector<uint32_t> coord, coord_worker, coord_firm;
  std::vector<double> outcome, target;
  std::vector<uint64_t> frequency;
  std::vector<std::vector<double>> controls;
  std::vector<double> probe_order;
  uint64_t physical_total = 0;
  double target_total = 0.0;
  size_t rows() const { return worker.size(); }
};

// Field-for-field the reference `GraphSelectionReceipt` (vckss-core/src/graph.rs:14-33).
struct GraphReceipt {
  uint64_t input_rows = 0, retained_rows = 0, input_physical_mass = 0, retained_physical_mass = 0;
  uint64_t initial_components = 0, maximum_components = 0, initial_component_rows = 0;
  uint64_t mover_input_rows = 0, initial_deletion_edges = 0, retained_deletion_edges = 0;
  uint64_t insufficient_workers_removed = 0, articulation_workers_removed = 0;
  uint64_t bridge_units_removed = 0, bridge_rows_removed = 0;
  uint64_t degree_iterations = 0, articulation_iterations = 0, bridge_iterations = 0;
  uint64_t fixed_point_iterations = 0;
};

struct GroupIndex {
  std::vector<uint64_t> ptr;
  std::vector<uint32_t> items;
};

struct Compressed {
  size_t workers = 0, firms = 0, cells = 0, deletion_units = 0, exact_target_strata = 0;
  uint64_t rows_physical = 0;
  std::vector<uint64_t> retained_rows;  // source row of each retained row
  std::vector<uint32_t> row_worker, row_firm, row_deletion, row_cell, row_target;
  std::vector<double> outcome, target;
  std::vector<uint64_t> frequency;
  std::vector<std::vector<double>> controls;
  std::vector<double> probe_order;
  std::vector<uint32_t> cell_worker, cell_firm;
  std::vector<double> cell_weight, cell_outcome_sum, cell_target_sum;
  GroupIndex worker_index, firm_index, deletion_index, target_index;
  GroupIndex cell_index;  // rows of every cell, in row order (the compression's sort)
  uint64_t physical_total = 0;
  double target_total = 0.0;
  size_t rows() const { return row_worker.size(); }
};

struct JlaPlan {
  bool generic = false;      // built by build_generic_plan
  bool observation = false;  // leave-observation-out units (classes of equal rank)
  std::vector<uint64_t> row_rank;
  // observation plan only: first Counter-V1 copy index of each row in its class
  std::vector<uint64_t> row_copy_offset;
  // generic plan only: rows of each deletion group in semantic-rank order
  // (observation plan: rows of each class in row order)
  std::vector<uint64_t> group_ptr;
  std::vector<uint32_t> group_rows;
  // deletion units
  std::vector<uint32_t> del_cell;
  std::vector<uint64_t> del_count, del_rank;
  std::vector<double> del_outcome_sum, del_target_mass;
  // target strata (cell, per-copy target mass)
  std::vector<uint32_t> tgt_cell;
  std::vector<double> tgt_per_copy, tgt_mass;
  std::vector<uint64_t> tgt_count, tgt_rank;
};

// Copies the caller's binary64 columns into typed columns (reference
// `copy_columns`, vckss-plugin/src/ffi_engine.rs:9568-9615, 10707-10800).
InputColumns copy_columns(uint64_t rows, const double* worker, const double* firm,
                          const double* deletion, const double* outcome, const double* frequency,
                          const double* target, const double* const* controls,
                          uint32_t controls_count, const double* probe_order);

// Reference `InputColumns::validate` (types.rs:175-260) followed by
// `CanonicalInput::from_validated_with_implicit_match_and_interrupt`
// (problem.rs:102-173).
Canonical canonicalize(InputColumns&& input, bool implicit_match);

// Reference `select_match_deletion_graph_standard_with_interrupt` (graph.rs:262-511).
std::vector<uint8_t> select_match_graph(const Canonical& in, GraphReceipt& receipt);
// Reference `select_implicit_match_no_prune_graph_with_interrupt` (graph.rs:513-588).
std::vector<uint8_t> select_implicit_match_graph(const Canonical& in, GraphReceipt& receipt);
// Reference `select_observation_deletion_graph_with_interrupt` (graph.rs:82-243).
std::vector<uint8_t> select_observation_graph(const Canonical& in, GraphReceipt& receipt);

// Reference `compress_with_implicit_match_and_interrupt` (problem.rs:206-606).
Compressed compress(const Canonical& in, const std::vector<uint8_t>& active, bool implicit_match);
// Reference `topology_checksum` of the compressed problem (problem.rs:1213-1248):
// FNV-1a over its sorted (worker, firm, deletion, frequency) records; computed
// on request (the detailed receipt reports it).
uint64_t compressed_topology_checksum(const Compressed& p);

// Reference `JlaPlan::build_no_controls_with_certified_match_and_interrupt`
// (jla.rs:59-108) generalised: controls do not enter the plan's orderings.
JlaPlan build_plan(const Compressed& p);

// The generic estimator's plan: semantic ranks that also order by the control
// values, the deletion units (match groups with their rows in rank order, or
// observation classes), and target strata (reference generic_jla.rs:3836-3900
// match ranks, 4052-4143 match plan, 4158-4334 observation classes,
// 3902-3995 target plan).
JlaPlan build_generic_plan(const Compressed& p, Deletion deletion = Deletion::Match);

}  // namespace fevcb
