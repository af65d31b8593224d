"""Detailed receipts V1-V7 against the reference plugin's on the same panels
and V5 requests (tests/golden/receipt_cases.json, made by make_golden.py
receipts): the request-side fields, counts, the topology checksum and the
solve's scalar results."""

import json
from pathlib import Path

import pytest

from fevc_b200 import abi

import make_golden

pytestmark = pytest.mark.gpu

HERE = Path(__file__).resolve().parent
CASES = json.loads((HERE / "golden" / "receipt_cases.json").read_text())["panels"]

EXACT = ["seed", "probes_requested", "leverage_probes_accepted", "target_probes_accepted", "solver_requested",
         "solver_selected", "solver_fallback", "solver_dimension", "leverage_batch_width", "target_batch_width",
         "rank_tolerance", "block_tolerance", "full_residual_tolerance", "full_fit_route", "full_fit_zero_rhs",
         "leverage_rhs_count", "target_rhs_count", "topology_checksum"]
CLOSE = ["full_fit_weighted_rss", "max_leverage"]
EXACT_V3 = ["rng_contract", "rhs_receipt_rows"]
EXACT_V4 = ["algorithm_requested", "algorithm_selected", "deletion_mode", "nuisance_mode", "parameters"]
EXACT_V6 = ["engine_requested", "engine_selected", "controls_count", "rhs_receipt_schema", "capability_schema",
            "capability_profile", "batch_mode", "stayers_mode", "target_weight_mode", "deletion_unit_source",
            "probeorder_supplied", "wallseconds_supplied", "frequency_use", "physical_limit", "request_signature"]


def solved(lib, name):
    case = CASES[name]
    spec = make_golden.RECEIPT_PANELS[name]
    panel = spec["build"]()
    e = abi.Engine(lib)
    e.prepare(panel, deletion_mode=case["deletion_mode"])
    q = make_golden.receipt_request(e, case["probes"], case["deletion_mode"], len(panel.controls))
    e.solve_v5(q, controls_count=len(panel.controls))
    return e, case["receipt"]


@pytest.mark.parametrize("name", list(CASES))
def test_detailed_receipt_matches_the_plugin(lib, name):
    e, ref = solved(lib, name)
    got = e.detailed_receipt(7).as_dict()
    e.release()
    bad = []
    gv2, rv2 = got["v6"]["v5"]["v4"]["v3"]["v2"], ref["v6"]["v5"]["v4"]["v3"]["v2"]
    for k in EXACT:
        if gv2[k] != rv2[k]:
            bad.append((k, gv2[k], rv2[k]))
    for k in CLOSE:
        if abs(gv2[k] - rv2[k]) > 1e-8 * max(abs(rv2[k]), 1.0):
            bad.append((k, gv2[k], rv2[k]))
    for k in EXACT_V3:
        if got["v6"]["v5"]["v4"]["v3"][k] != ref["v6"]["v5"]["v4"]["v3"][k]:
            bad.append((k, got["v6"]["v5"]["v4"]["v3"][k], ref["v6"]["v5"]["v4"]["v3"][k]))
    for k in EXACT_V4:
        if got["v6"]["v5"]["v4"][k] != ref["v6"]["v5"]["v4"][k]:
            bad.append((k, got["v6"]["v5"]["v4"][k], ref["v6"]["v5"]["v4"][k]))
    for k in EXACT_V6:
        if got["v6"][k] != ref["v6"][k]:
            bad.append((k, got["v6"][k], ref["v6"][k]))
    assert got["execution"]["request_signature"] == ref["execution"]["request_signature"]
    assert gv2["accounting_residual"] <= 1e-11 and gv2["max_reciprocal_residual"] <= 1e-12
    assert not bad, bad


def test_receipt_versions_are_prefixes(lib):
    e, _ = solved(lib, "controls")
    v7 = bytes(e.detailed_receipt(7))
    for k, size in ((2, 360), (3, 384), (4, 448), (5, 536), (6, 840)):
        assert bytes(e.detailed_receipt(k)) == v7[:size], k
    with pytest.raises(abi.EngineError) as err:  # V1 describes a no-control match solve
        e.detailed_receipt(1)
    assert err.value.code == 11
    e.release()
    e, _ = solved(lib, "match_small_2k")
    v1 = bytes(e.detailed_receipt(1))
    v2 = bytes(e.detailed_receipt(2))
    assert v1[4:272] == v2[4:272] and int.from_bytes(v1[:4], "little") == 272
    e.release()
