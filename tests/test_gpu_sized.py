"""Parity with the reference plugin at reduced sizes of the benchmark panels.

tests/golden/sized_cases.json holds the plugin's four component groups
(plug-in, correction, corrected, numerical MCSE) for the benchmark's seeded
generator at 0.1 of the 1M-worker controls panel and 0.02 of the 10M-worker
leave-observation-out panel, with the same seed and probes and a supplied
tolerance of 1e-10 (tests/golden/make_golden.py sized).  The device engine
regenerates each panel, solves it in every production form and must match
each group within 1e-6 relative to the group's largest component, the
tolerance stated for the variance components.
"""

import json
from pathlib import Path

import numpy as np
import pytest

from fevc_b200 import abi, learned
from fevc_b200.panel import named_panel

import make_golden

pytestmark = pytest.mark.gpu

SIZED_RTOL = 1e-6
CASES = json.loads((Path(__file__).resolve().parent / "golden" / "sized_cases.json").read_text())["cases"]

# (preconditioner, precision): FP64 Jacobi, mixed-precision Jacobi, the
# uniform-weight polynomial stage in mixed precision, and the learned stage in
# mixed precision (the benchmark's combined form)
FORMS = [(1, 0), (1, 1), (4, 1), (3, 1)]


def rel(a, b):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("key", sorted(CASES))
def test_sized_components_match_the_plugin(lib, key, form):
    rec = CASES[key]
    precond, precision = form
    if precond == 3:
        params = learned.load_params()
        if params is None:
            pytest.skip("no trained network parameters are committed")
        learned.install(lib, params)
    panel = named_panel(rec["panel"], rec["scale"])
    assert make_golden.panel_digest(panel) == rec["panel_sha256"]
    e = abi.Engine(lib)
    e.prepare(panel, deletion_mode=rec["deletion_mode"])
    e.device_options(0, precond, precision)
    q = e.default_request_v5(rec["deletion_mode"])
    v1 = q.v4.v3.v2.v1
    v1.seed = rec["seed"]
    v1.probes = rec["probes"]
    v1.pcg_tolerance = rec["pcg_tolerance"]
    v1.maximum_iterations = 20000
    q.v4.v3.v2.algorithm = 2
    if rec["deletion_mode"] == 2:
        q.v4.v3.engine = 2
    q.tolerance_supplied = 1
    e.solve_v5(q, controls_count=rec["controls"])
    res = e.result()
    e.release()
    for group in ("plugin", "correction", "corrected", "numerical_mcse"):
        assert rel(res[group], rec[group]) < SIZED_RTOL, (group, res[group], rec[group])
