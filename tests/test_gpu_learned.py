"""The learned preconditioner on the device: forward and backward kernels
against the numpy oracle, training lowers the loss, flexible PCG with the
trained network reproduces the reference's components, and the network
saves iterations over the same flexible PCG without the learned stage."""

import numpy as np
import pytest

from fevc_b200 import abi, learned
from fevc_b200.panel import generate_panel
from oracle import gnn_oracle

import make_golden

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def trained(lib):
    """A network trained on a few small seeded panels (seconds)."""
    params, losses = learned.train_default(lib, panels=6, steps=300, lr=3e-3, columns=16, workers=8000, firms=700)
    return params, losses


@pytest.mark.parametrize("perturb", [0.0, 0.05])
def test_device_gradient_matches_oracle(lib, perturb):
    with learned.Trainer(lib, seed=3) as t:
        t.add_panel(generate_panel(3000, 300, 5, move_p=0.2, seed=5), columns=8, seed=11)
        if perturb:
            rng = np.random.default_rng(4)
            t.params = t.params + perturb * rng.standard_normal(t.count).astype(np.float32)
        params = t.params
        loss, grad = t.gradient(0)
        d = t.dump(0)
    ref_loss, ref_grad = gnn_oracle.loss_and_grad(d, params)
    assert abs(loss - ref_loss) <= 1e-4 * abs(ref_loss), (loss, ref_loss)
    err = np.linalg.norm(grad - ref_grad) / np.linalg.norm(ref_grad)
    assert err < 2e-3, err
    # every layer receives gradient
    offs, oh, _ = gnn_oracle.layout()
    for o, i in offs:
        assert np.linalg.norm(grad[o:o + 2 * i * 64]) > 0


def test_training_lowers_the_loss(trained):
    _, losses = trained
    first, last = np.mean(losses[:6]), np.mean(losses[-6:])
    assert last < 0.95 * first, (first, last)


def solve(lib, panel, *, probes, precond, centering=0, tol=1e-12, seed=8675309, block=0):
    e = abi.Engine(lib)
    e.prepare(panel)
    if centering:
        e.centering(centering)
    e.device_options(block, precond)
    req = e.default_request()
    req.seed = seed
    req.probes = probes
    req.pcg_tolerance = tol
    req.maximum_iterations = 20000
    e.solve(req)
    return e


@pytest.mark.parametrize("name", ["small_2k", "exact_20k", "regions_4k"])
def test_learned_flexible_pcg_matches_reference(lib, golden, trained, name):
    learned.install(lib, trained[0])
    rec = golden["jla"]["panels"][name][1]
    panel = make_golden.PANELS[name]["build"]()
    e = solve(lib, panel, probes=rec["probes"], precond=3, centering=rec["centering"], seed=rec["seed"])
    res = e.result()
    e.release()
    for key in ("plugin", "correction", "corrected", "numerical_mcse"):
        assert rel(res[key], rec[key]) < 1e-8, (key, res[key], rec[key])


def test_learned_stage_saves_iterations(lib, trained):
    """Same panel (two regions joined by few moves, the hard case): flexible
    PCG with the trained network against the same flexible PCG with the
    untrained network (unit coefficients, the truncated Neumann series) and
    against Jacobi PCG, the method without the learned stage."""
    panel = generate_panel(60000, 4000, 5, regions=2, cross_p=0.002, seed=78)
    it = {}
    for label, params, precond in (("trained", trained[0], 3), ("untrained", learned.initial_params(lib, 1), 3),
                                   ("jacobi", None, 1)):
        if params is not None:
            learned.install(lib, params)
        e = solve(lib, panel, probes=32, precond=precond, tol=1e-8)
        t = e.timings()
        res = e.result()
        e.release()
        it[label] = (t["column_iterations"] / t["rhs_columns"], t["fallbacks"], res["corrected"])
    assert it["trained"][1] == 0
    assert rel(it["trained"][2], it["jacobi"][2]) < 1e-6
    assert it["trained"][0] < it["untrained"][0], it
    assert it["trained"][0] < 0.5 * it["jacobi"][0], it
