"""Numerical MCSE attachment on the device against the plugin's own
attachment (``tests/golden/numerical_cases.json``), on the compressed engine
and with leave-observation-out deletion (with and without controls, with
duplicated rows and literal frequencies): the replay counts, fold sizes and
status exactly; the conditional and leverage covariances, the usable matrix,
the MCSE and the share extremes within 1e-8 relative; the exact-zero
attachment when the automatic algorithm resolves to exact."""

import json
from pathlib import Path

import numpy as np
import pytest

from fevc_b200 import abi

import make_golden

pytestmark = pytest.mark.gpu

CASES = json.loads((Path(__file__).resolve().parent / "golden" / "numerical_cases.json").read_text())["cases"]
EXACT_FIELDS = ("status", "engine", "leverage_probes", "target_probes", "target_fold_a", "target_fold_b",
                "certified_replay_rhs", "executed_replay_rhs", "attempted_replay_rhs", "replay_generator_words",
                "allocation_bound_bytes", "failed_replay_probe", "replay_error_code", "point_rhs")
TOL = 1e-8


def rel(a, b):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def solved(lib):
    out = {}
    for name, spec in make_golden.NUMERICAL_PANELS.items():
        panel = spec["build"]()
        assert make_golden.panel_digest(panel) == CASES[name]["panel_sha256"]
        deletion = spec.get("deletion", 1)
        e = abi.Engine(lib)
        e.prepare(panel, deletion_mode=deletion)
        e.solve_numerical(make_golden.numerical_request(e, spec["probes"], spec["algorithm"], deletion,
                                                        len(panel.controls)))
        r = e.numerical_result()
        point = e.result()
        count, rhs = e.numerical_rhs(int(r["certified_replay_rhs"]) + 3)
        e.release()
        out[name] = (r, point, count, rhs)
    return out


@pytest.mark.parametrize("name", sorted(CASES))
def test_attachment_counts_match_the_plugin(solved, name):
    want = CASES[name]["record"]
    got, _, count, rhs = solved[name]
    for k in EXACT_FIELDS:
        assert got[k] == want[k], (k, got[k], want[k])
    assert count == len(want["rhs"])
    assert [x["probe"] for x in rhs] == [x[0] for x in want["rhs"]]
    assert all(x["phase"] == 1 and x["schema_version"] == 1 for x in rhs)
    if want["status"] != 1:
        assert max(x["complete_residual"] for x in rhs) < 1e-9
        assert got["maximum_point_complete_residual"] < 1e-9
        assert got["maximum_replay_complete_residual"] < 1e-9


@pytest.mark.parametrize("name", sorted(CASES))
def test_attachment_covariance_matches_the_plugin(solved, name):
    want = CASES[name]["record"]
    got, point, _, _ = solved[name]
    assert rel(point["corrected"], want["corrected"]) < TOL
    for key in ("conditional", "leverage", "raw", "usable", "mcse"):
        assert rel(got[key], want[key]) < TOL, (key, got[key], want[key])
    for key in ("minimum_constrained", "minimum_residual_margin", "maximum_sensitivity_ratio"):
        assert rel(got[key], want[key]) < TOL, (key, got[key], want[key])
    # the fold score means are zero up to roundoff of the fold scores
    spread = np.sqrt(max(np.max(np.abs(want["leverage"])), 1e-300)) * want["leverage_probes"]
    assert np.max(np.abs(np.array(got["score_means"]) - np.array(want["score_means"]))) <= 1e-9 * spread
    assert abs(got["psd_adjustment"] - want["psd_adjustment"]) <= TOL * max(np.max(np.abs(want["raw"])), 1e-300)


def test_attachment_leaves_the_point_estimate_unchanged(lib):
    """The attachment adds the replay after the point solve: the point result
    equals a plain V5 solve of the same request on another generation of the
    same panel, which has no attachment to report."""
    spec = make_golden.NUMERICAL_PANELS["small_2k"]
    panel = spec["build"]()
    e = abi.Engine(lib)
    e.prepare(panel)
    req = make_golden.numerical_request(e, spec["probes"], 2)
    e.solve_numerical(req)
    with_attachment = e.result()
    e.release()
    f = abi.Engine(lib)
    f.prepare(panel)
    q = f.default_request_v5(1)
    q.v4 = req.point
    q.threads = req.threads
    q.tolerance_supplied = req.tolerance_supplied
    f.solve_v5(q)
    plain = f.result()
    with pytest.raises(abi.EngineError) as err:
        f.numerical_result()
    assert err.value.code == 11
    f.release()
    for key in ("plugin", "correction", "corrected", "numerical_mcse"):
        assert with_attachment[key] == plain[key], key
