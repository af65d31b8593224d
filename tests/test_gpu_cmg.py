"""The CMG-preconditioned device solve (request route = CMG PCG): the same
components as the reference plugin, and fewer iterations than Jacobi on a
poorly connected panel."""

import numpy as np
import pytest

from fevc_b200 import abi

import make_golden

pytestmark = pytest.mark.gpu

COMPONENT_RTOL = 1e-8


def rel(a, b):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def solve(lib, panel, *, probes, route, centering=0, tol=1e-12, block=0, seed=8675309):
    e = abi.Engine(lib)
    e.prepare(panel)
    if centering:
        e.centering(centering)
    e.device_options(block, 0)
    req = e.default_request()
    req.seed = seed
    req.probes = probes
    req.pcg_tolerance = tol
    req.maximum_iterations = 20000
    req.solver_route = route
    e.solve(req)
    return e


@pytest.mark.parametrize("name,block", [("small_2k", 0), ("exact_20k", 0), ("weighted_1500", 0), ("regions_4k", 0),
                                        ("small_2k", 2)])
def test_cmg_route_matches_reference(lib, golden, name, block):
    """Block 2 is the plain form: one target probe (two right-hand sides) per solve."""
    rec = golden["jla"]["panels"][name][1]
    panel = make_golden.PANELS[name]["build"]()
    e = solve(lib, panel, probes=rec["probes"], route=3, centering=rec["centering"], seed=rec["seed"], block=block)
    res = e.result()
    e.release()
    for key in ("plugin", "correction", "corrected", "numerical_mcse"):
        assert rel(res[key], rec[key]) < COMPONENT_RTOL, (key, res[key], rec[key])


@pytest.mark.parametrize("block", [8, 64])
def test_cmg_and_jacobi_agree(lib, block):
    from fevc_b200.panel import generate_panel

    panel = generate_panel(60000, 6000, 6, regions=2, cross_p=0.002, seed=63)
    out = {}
    for route in (2, 3):
        e = solve(lib, panel, probes=16, route=route, tol=1e-10, block=block)
        out[route] = (e.result(), e.timings())
        e.release()
    for key in ("plugin", "correction", "corrected"):
        assert rel(out[3][0][key], out[2][0][key]) < 1e-7, key
    # the two-region bottleneck: the hierarchy's coarse solve carries the
    # slow mode that Jacobi has to iterate out (about half the iterations)
    assert out[3][1]["column_iterations"] < 0.7 * out[2][1]["column_iterations"], (
        out[3][1]["column_iterations"], out[2][1]["column_iterations"])
    assert out[3][1]["levels"] >= 2
