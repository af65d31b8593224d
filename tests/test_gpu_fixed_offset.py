"""Fixed-offset nuisance of the generic engine on the device: the joint
fit's control coefficients held fixed and the estimator run on the
worker-firm model of y - Q'beta (reference NuisanceMode::FixedOffset,
generic_jla.rs:2011-2046), against the plugin's own results for the same
panels, probes and seed (``tests/golden/fixed_offset_cases.json``, made by
running the plugin): point components, the numerical attachment and a
projection, through the C ABI on a B200.

Tolerances: components within 1e-8 relative to the largest (both engines
solve to 1e-12 on the same Counter-V1 probes); numerical covariances within
1e-6; projection coefficients 1e-8 and covariances 1e-6."""

import json
from pathlib import Path

import numpy as np
import pytest

from fevc_b200 import abi

import make_golden

pytestmark = pytest.mark.gpu

CASES = json.loads((Path(__file__).resolve().parent / "golden" / "fixed_offset_cases.json").read_text())["cases"]


def rel(a, b):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def engine(lib, case):
    panel = make_golden.projection_panel(case["panel"])
    assert make_golden.panel_digest(panel) == case["panel_sha256"]
    e = abi.Engine(lib)
    e.prepare(panel, deletion_mode=case["deletion"])
    if case["centering"]:
        e.centering(case["centering"])
    return e, panel


@pytest.mark.parametrize("name", sorted(CASES))
def test_point_solve_matches_the_plugin(lib, name):
    case = CASES[name]
    e, panel = engine(lib, case)
    try:
        q = make_golden.projection_request(e, case["probes"], case["deletion"], len(panel.controls))
        q.v4.v3.v2.nuisance_mode = 2
        e.solve_v5(q, controls_count=len(panel.controls))
        res = e.result()
        rc = e.rhs_receipts(int(e.timings()["rhs_columns"]) + 64)
    finally:
        e.release()
    for key in ("plugin", "correction", "corrected", "numerical_mcse"):
        assert rel(res[key], case[key]) < 1e-8, (key, res[key], case[key])
    # the joint fit (phase 1) and the fixed-offset working fit (phase 4)
    phases = [r["phase"] for r in rc]
    assert phases.count(1) == 1 and phases.count(4) == 1


@pytest.mark.parametrize("name", sorted(CASES))
def test_numerical_attachment_matches_the_plugin(lib, name):
    case = CASES[name]
    e, panel = engine(lib, case)
    try:
        req = make_golden.numerical_request(e, case["probes"], 2, case["deletion"], len(panel.controls))
        req.point.v3.v2.nuisance_mode = 2
        req.point.v3.request_signature = abi.capability_signature_v3(req.point, len(panel.controls))
        e.solve_numerical(req)
        r = e.numerical_result()
    finally:
        e.release()
    want = case["numerical"]
    assert r["status"] == want["status"] and r["engine"] == want["engine"]
    for k in ("raw", "usable", "mcse"):
        assert rel(r[k], want[k]) < 1e-6, (k, r[k], want[k])


@pytest.mark.parametrize("name", sorted(CASES))
def test_projection_matches_the_plugin(lib, name):
    case = CASES[name]
    e, panel = engine(lib, case)
    try:
        e.augment_projection(make_golden.projection_covariates(panel, e.retained_mask(panel.rows), 2, 20261204))
        q = make_golden.projection_request(e, case["probes"], case["deletion"], len(panel.controls))
        q.v4.v3.v2.nuisance_mode = 2
        e.solve_v5(q, controls_count=len(panel.controls))
        got = e.projection_result()
    finally:
        e.release()
    want = case["projection"]
    assert rel(got["coefficients"], want["coefficients"]) < 1e-8
    assert rel(got["covariance"], want["covariance"]) < 1e-6
    assert rel(got["naive_covariance"], want["naive_covariance"]) < 1e-6
    r = got["receipt"]
    assert [r["proxy_minimum"], r["proxy_maximum"]] == pytest.approx(want["proxy"], rel=1e-8)
