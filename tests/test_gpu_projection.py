"""Fixed-effect projection attachment on the device: coefficients, KSS and
naive covariances and the result receipt against the plugin's own results
for the same panels, covariates, probes and seed
(``tests/golden/projection_cases.json``, made by running the plugin), through
the C ABI on a B200, plus the solve-time refusals.

Tolerances: the coefficients come from the full fit (both engines solve it
to 1e-12 relative residual), so they agree to 1e-8 relative; the covariances
are sums of leave-out products built from the same Counter-V1 probes solved
to 1e-12, so they agree to 1e-6 relative to their largest entry (the
north-star component tolerance)."""

import json
from pathlib import Path

import numpy as np
import pytest

from fevc_b200 import abi

import make_golden

pytestmark = pytest.mark.gpu

FIXTURE = json.loads((Path(__file__).resolve().parent / "golden" / "projection_cases.json").read_text())
CASES = FIXTURE["cases"]


def rel(a, b):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def solved(lib, case):
    panel = make_golden.projection_panel(case["panel"])
    e = abi.Engine(lib)
    e.prepare(panel, deletion_mode=case["deletion"])
    cov = make_golden.projection_covariates(panel, e.retained_mask(panel.rows), case["covariates"], 20261204)
    if case["centering"]:
        e.centering(case["centering"])
    e.augment_projection(cov, case["effect"], case["weight"])
    e.solve_v5(make_golden.projection_request(e, case["probes"], case["deletion"], len(panel.controls)),
               controls_count=len(panel.controls))
    return e


@pytest.mark.parametrize("name", sorted(CASES))
def test_projection_matches_the_plugin(lib, name):
    case = CASES[name]
    e = solved(lib, case)
    try:
        got = e.projection_result()
        point = e.result()
        receipts = e.rhs_receipts(int(e.timings()["rhs_columns"]) + 64)
    finally:
        e.release()
    assert rel(point["corrected"], case["corrected"]) < 1e-8
    assert rel(got["coefficients"], case["coefficients"]) < 1e-8, (got["coefficients"], case["coefficients"])
    assert rel(got["covariance"], case["covariance"]) < 1e-6, (got["covariance"], case["covariance"])
    assert rel(got["naive_covariance"], case["naive_covariance"]) < 1e-6
    assert np.allclose(got["covariance"], np.transpose(got["covariance"]), rtol=0, atol=0)
    r, want = got["receipt"], case["receipt"]
    for k in ("columns", "effect", "weight", "gram_rcond", "gram_relres", "gram_original_relres",
              "full_residual_tolerance", "persistent_bytes", "result_bytes"):
        assert r[k] == want[k], (k, r[k], want[k])
    scale = max(abs(np.diag(np.asarray(case["covariance"]))))
    for k in ("covariance_smallest_eigenvalue", "covariance_largest_eigenvalue", "psd_cleanup"):
        assert abs(r[k] - want[k]) <= 1e-6 * scale, (k, r[k], want[k])
    for k in ("proxy_minimum", "proxy_maximum"):
        assert r[k] == pytest.approx(want[k], rel=1e-8), (k, r[k], want[k])
    assert r["maximum_iterations"] > 0 and r["maximum_complete_residual"] <= r["full_residual_tolerance"]
    # one phase-6 (projection) receipt per column, probe = the column's index
    proj = [x for x in receipts if x["phase"] == 6]
    assert [x["probe"] for x in proj] == list(range(case["receipt"]["columns"]))


def test_solve_time_refusals(lib):
    """A match panel without controls runs the compressed engine, which has
    no projection (11); the augmentation receipt is only read before the
    solve (81); a solve without an attachment has no projection result (11);
    the numerical attachment does not combine with a projection (11)."""
    errors = FIXTURE["errors"]

    def status(fn):
        try:
            fn()
            return 0
        except abi.EngineError as err:
            return err.code

    plain = make_golden.PANELS["small_2k"]["build"]()
    e = abi.Engine(lib)
    e.prepare(plain, use_v4=True)
    e.augment_projection(make_golden.projection_covariates(plain, e.retained_mask(plain.rows), 1, 7))
    assert status(lambda: e.solve_v5(make_golden.projection_request(e, 8, 1, 0), controls_count=0)) == \
        errors["compressed_engine_solve"] == 11
    e.release()
    case = CASES["controls_2k_worker"]
    e = solved(lib, case)
    assert status(lambda: e.projection_augmentation_receipt()) == errors["augmentation_receipt_after_solve"] == 81
    e.release()
    panel = make_golden.projection_panel("controls_2k")
    e = abi.Engine(lib)
    e.prepare(panel)
    e.solve_v5(make_golden.projection_request(e, 8, 1, len(panel.controls)), controls_count=len(panel.controls))
    assert status(lambda: e.projection_result()) == errors["result_without_projection"] == 11
    e.release()
    e = abi.Engine(lib)
    e.prepare(panel)
    e.augment_projection(make_golden.projection_covariates(panel, e.retained_mask(panel.rows), 2, 20261204))
    req = make_golden.numerical_request(e, 8, 2, 1, len(panel.controls))
    assert status(lambda: e.solve_numerical(req)) == 11
    e.release()


def test_resolve_repeats_the_projection(lib):
    """A repeated solve of the same generation gives the same projection bit
    for bit (same device program, same inputs)."""
    e = solved(lib, CASES["obs_2k_worker"])
    try:
        first = e.projection_result()
        e.resolve()
        again = e.projection_result()
    finally:
        e.release()
    assert first["coefficients"] == again["coefficients"]
    assert first["covariance"] == again["covariance"]
    assert first["naive_covariance"] == again["naive_covariance"]
