"""Fixed-effect projection attachment, host side (no device): the loadings'
Gram certificates in the augmentation receipt and the refusals of
``vckss_rust_engine_augment_projection_interrupt_v1``, against the plugin's
own receipts and statuses in ``tests/golden/projection_cases.json`` (made by
running the plugin, ``tests/golden/make_golden.py projection``)."""

import json
from pathlib import Path

import numpy as np
import pytest

from fevc_b200 import abi

import make_golden

FIXTURE = json.loads((Path(__file__).resolve().parent / "golden" / "projection_cases.json").read_text())
CASES = FIXTURE["cases"]


def augmented(lib, case):
    panel = make_golden.projection_panel(case["panel"])
    assert make_golden.panel_digest(panel) == case["panel_sha256"]
    e = abi.Engine(lib)
    e.prepare(panel, deletion_mode=case["deletion"])
    cov = make_golden.projection_covariates(panel, e.retained_mask(panel.rows), case["covariates"], 20261204)
    if case["centering"]:
        e.centering(case["centering"])
    e.augment_projection(cov, case["effect"], case["weight"])
    return e


@pytest.mark.parametrize("name", sorted(CASES))
def test_augmentation_receipt_matches_the_plugin(lib, name):
    """Rows, columns, effect, weight, copied and persistent bytes equal; the
    Gram's certified rcond and inverse residuals (cyclic Jacobi spectrum,
    Cholesky inverse, both in the reference's operation order) equal the
    plugin's bit for bit."""
    case = CASES[name]
    e = augmented(lib, case)
    try:
        r = e.projection_augmentation_receipt()
    finally:
        e.release()
    want = case["augmentation"]
    for k in ("rows", "columns", "effect", "weight", "caller_copy_bytes", "projection_persistent_bytes"):
        assert r[k] == want[k], (k, r[k], want[k])
    for k in ("gram_rcond", "gram_relres", "gram_original_relres"):
        assert r[k] == want[k], (k, r[k], want[k])
    assert r["struct_size"] == 96 and r["schema_version"] == 1
    assert r["total_prepared_resident_bytes"] >= r["projection_persistent_bytes"]
    assert r["augmentation_peak_forecast_bytes"] >= r["total_prepared_resident_bytes"]


@pytest.mark.parametrize("name", ["constant_covariate", "rank_tolerance_high", "rank_tolerance_low", "effect_unknown",
                                  "weight_unknown", "rows_short"])
def test_refused_augmentations_match_the_plugin(lib, name):
    """A constant covariate duplicates the automatic constant (singular
    Gram, 82); malformed requests are refused before the generation is
    touched (20) and a valid projection still attaches afterwards; a refusal
    inside the attachment (singular Gram, rows that differ from the retained
    sample) fails the generation (81 afterwards), as in the plugin."""
    panel = make_golden.projection_panel("controls_2k")
    e = abi.Engine(lib)
    e.prepare(panel)
    mask = e.retained_mask(panel.rows)
    cov = make_golden.projection_covariates(panel, mask, 2, 20261204)
    rows = int(mask.sum())
    args = {"constant_covariate": ([np.ones(rows)], 1, 1, 1e-10),
            "rank_tolerance_high": (cov, 1, 1, 0.5),
            "rank_tolerance_low": (cov, 1, 1, 1e-16),
            "effect_unknown": (cov, 3, 1, 1e-10),
            "weight_unknown": (cov, 1, 3, 1e-10),
            "rows_short": ([c[:-1] for c in cov], 1, 1, 1e-10)}[name]

    def status(fn):
        try:
            fn()
            return 0
        except abi.EngineError as err:
            return err.code

    try:
        assert status(lambda: e.augment_projection(*args)) == FIXTURE["errors"][name]
        assert status(lambda: e.augment_projection(cov)) == FIXTURE["errors"][name + "_then_valid"]
    finally:
        e.release()


def test_second_projection_is_refused(lib):
    case = CASES["controls_2k_worker"]
    e = augmented(lib, case)
    try:
        panel = make_golden.projection_panel(case["panel"])
        cov = make_golden.projection_covariates(panel, e.retained_mask(panel.rows), 2, 20261204)
        with pytest.raises(abi.EngineError) as err:
            e.augment_projection(cov)
        assert err.value.code == FIXTURE["errors"]["second_projection"] == 81
    finally:
        e.release()


def test_projection_entry_points_without_a_solve(lib):
    """Defaults (worker effect, frequency weight, tolerance 1e-10, the
    interrupt struct's size; a short output is an ABI mismatch, 10), the
    centering schema, and a result request on a generation that has not
    solved (81), with the plugin's statuses."""
    q = abi.ProjectionAugmentationRequestInterruptV1()
    assert lib.vckss_rust_engine_default_projection_augmentation_request_interrupt_v1(
        abi.C.byref(q), abi.C.sizeof(q)) == 0
    assert (q.options.abi_version, q.options.struct_size, q.options.effect, q.options.weight) == (1, 72, 1, 1)
    assert q.options.rank_tolerance == 1e-10 and q.options.rows == 0 and q.options.caller_copy_bytes == 0
    assert lib.vckss_rust_engine_default_projection_augmentation_request_interrupt_v1(abi.C.byref(q), 71) == 10  # short output: ABI mismatch
    assert lib.vckss_rust_projection_centering_schema_v1() == 1
    e = augmented(lib, CASES["obs_2k_worker"])
    try:
        with pytest.raises(abi.EngineError) as err:
            e.projection_result()
        assert err.value.code == 81
    finally:
        e.release()
