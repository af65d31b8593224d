"""Exact leverages on the device (algorithm EXACT, match deletion without
controls): the components of the plugin's own exact estimator on small
panels, the numpy restatement at the 20,000-worker / 1,000-firm size of the
exact-leverage benchmark panel (beyond the plugin's 2,000-parameter limit,
so the generation's ceiling is raised), and JLA estimates on that panel
approaching the exact components as the probe count grows."""

import json
from pathlib import Path

import numpy as np
import pytest

from fevc_b200 import abi
from fevc_b200.panel import named_panel

import make_golden

pytestmark = pytest.mark.gpu

EXACT = json.loads((Path(__file__).resolve().parent / "golden" / "exact_cases.json").read_text())["cases"]


def rel(a, b):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("name", sorted(EXACT))
@pytest.mark.parametrize("which", [0, 1])
def test_device_exact_matches_the_plugin_exact_estimator(lib, name, which):
    rec = EXACT[name]["records"][which]
    panel = make_golden.EXACT_PANELS[name]["build"]()
    e = abi.Engine(lib)
    e.prepare(panel)
    if rec["centering"]:
        e.centering(rec["centering"])
    q = e.exact_request_v5(2000)
    q.v4.v3.v2.v1.pcg_tolerance = 1e-12
    e.solve_v5(q)
    res = e.result()
    e.release()
    for key in ("plugin", "correction", "corrected"):
        assert rel(res[key], rec[key]) < 1e-8, (key, res[key], rec[key])
    assert np.all(np.array(res["numerical_mcse"]) == 0.0)


@pytest.fixture(scope="module")
def exact_20k(lib, oracle_mod):
    """The 20,000-worker panel: device exact components and the oracle's."""
    panel = named_panel("exact_20k")
    e = abi.Engine(lib)
    e.prepare(panel)
    e.centering(1)
    want = oracle_mod.exact(oracle_mod.problem_view(lib, e.generation), centering=1)
    e.exact_ceiling(20_000)
    q = e.exact_request_v5(2000)
    q.v4.v3.v2.v1.pcg_tolerance = 1e-12
    e.solve_v5(q)
    got = e.result()
    e.release()
    return panel, got, want


def test_device_exact_matches_the_oracle_at_the_benchmark_size(exact_20k):
    _, got, want = exact_20k
    for key in ("plugin", "correction", "corrected"):
        assert rel(got[key], want[key]) < 1e-8, (key, got[key], want[key])


@pytest.mark.parametrize("precision", [0, 1])
def test_jla_approaches_the_exact_components(lib, exact_20k, precision):
    """JLA (FP64, and FP32 storage with FP64 reductions and replacement) on
    the 20,000-worker panel: each component within five numerical standard
    errors of the exact one, the MCSE shrinking with the probes."""
    panel, got, _ = exact_20k
    exact = np.array(got["corrected"])
    errs = []
    for probes in (40, 640):
        e = abi.Engine(lib)
        e.prepare(panel)
        e.device_options(64, 1, precision)
        e.centering(1)
        req = e.default_request()
        req.probes = probes
        req.pcg_tolerance = 1e-10
        e.solve(req)
        res = e.result()
        e.release()
        err = np.abs(np.array(res["corrected"]) - exact)
        mcse = np.array(res["numerical_mcse"])
        # every component within five numerical standard errors of the exact value
        assert np.all(err <= 5.0 * mcse + 1e-12), (probes, err, mcse)
        errs.append((float(np.max(err[:3] / np.abs(exact[:3]))), float(np.max(mcse[:3] / np.abs(exact[:3])))))
    # sixteen times the probes: the Monte Carlo error shrinks about fourfold
    assert errs[1][1] < 0.35 * errs[0][1], errs


def test_fp32_storage_matches_fp64_on_the_exact_panel(lib, exact_20k):
    """The mixed-precision form's components equal the FP64 form's on the same
    probes to 1e-8 relative (both certified at the same residual in FP64),
    so its error against the exact leverages is the Monte Carlo error."""
    panel, _, _ = exact_20k
    out = []
    for precision in (0, 1):
        e = abi.Engine(lib)
        e.prepare(panel)
        e.device_options(64, 1, precision)
        e.centering(1)
        req = e.default_request()
        req.probes = 200
        req.pcg_tolerance = 1e-10
        e.solve(req)
        out.append(e.result())
        e.release()
    for key in ("plugin", "correction", "corrected"):
        assert rel(out[1][key], out[0][key]) < 1e-8, (key, out[1][key], out[0][key])
