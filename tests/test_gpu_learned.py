"""The learned preconditioner on the device: forward and backward kernels
against the numpy oracle, training lowers the loss, PCG with the trained
network's per-vertex weights reproduces the reference's components, and
what the trained network gains over the same stage without it (uniform
weights) and over Jacobi PCG, in iterations and in device time per
right-hand side."""

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


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", ["small_2k", "exact_20k", "regions_4k"])
def test_learned_stage_matches_reference(lib, golden, trained, name, precision):
    learned.install(lib, trained[0])
    rec = golden["jla"]["panels"][name][1]
    panel = make_golden.PANELS[name]["build"]()
    e = abi.Engine(lib)
    e.prepare(panel)
    if rec["centering"]:
        e.centering(rec["centering"])
    e.device_options(0, 3, precision)
    req = e.default_request()
    req.seed = rec["seed"]
    req.probes = rec["probes"]
    req.pcg_tolerance = 1e-12
    req.maximum_iterations = 20000
    e.solve(req)
    res = e.result()
    e.release()
    for key in ("plugin", "correction", "corrected", "numerical_mcse"):
        assert rel(res[key], rec[key]) < 1e-8, (key, res[key], rec[key])


def timed_form(lib, panel, *, probes, precond, precision, params=None):
    """Iterations per right-hand side and device milliseconds per
    right-hand side of one resolve (CUDA events on the library's stream)."""
    import ctypes as C

    import torch

    if params is not None:
        learned.install(lib, params)
    stream = torch.cuda.Stream()
    lib.fevcb_set_stream(C.c_void_p(stream.cuda_stream))
    try:
        e = abi.Engine(lib)
        e.prepare(panel)
        e.device_options(64, precond, precision)
        req = e.default_request()
        req.probes = probes
        req.pcg_tolerance = 1e-8
        req.maximum_iterations = 20000
        e.solve(req)
        e.resolve()  # warm
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        e.resolve()
        stop.record(stream)
        stop.synchronize()
        t = e.timings()
        res = e.result()
        e.release()
    finally:
        lib.fevcb_set_stream(C.c_void_p(None))
    rhs = t["rhs_columns"]
    return {"iters": t["column_iterations"] / rhs, "ms_per_rhs": start.elapsed_time(stop) / rhs,
            "fallbacks": t["fallbacks"], "corrected": res["corrected"]}


def test_learned_stage_gain(lib, trained):
    """One panel, four forms: the trained network's weights and the untrained
    network's (uniform first-order Neumann weights, the stage without the
    network) in the mixed-precision single-kernel PCG, mixed-precision Jacobi,
    and the FP64 Jacobi kernel.  The learned mixed form must take under 0.7 of
    the iterations of Jacobi and fewer device milliseconds per right-hand side
    than Jacobi at the same precision, at the same components, and no more
    than 1.05 of the iterations of the uniform weights.  Against FP64 Jacobi
    it is not required to win: the second gather of the degree-1 stage costs
    about what the halved iteration count saves on this latency-bound kernel
    (measured 0.043 against 0.038 ms per right-hand side here), which is why
    the autotuned precision times the forms and keeps the fastest."""
    panel = generate_panel(400_000, 40_000, 5, pareto_shape=1.2, seed=78)
    forms = {
        "learned_mixed": dict(precond=3, precision=1, params=trained[0]),
        "uniform_mixed": dict(precond=3, precision=1, params=learned.initial_params(lib, 1)),
        "jacobi_mixed": dict(precond=1, precision=1),
        "jacobi_fp64": dict(precond=1, precision=0),
    }
    out = {k: timed_form(lib, panel, probes=64, **v) for k, v in forms.items()}
    print({k: (round(v["iters"], 2), round(v["ms_per_rhs"], 4)) for k, v in out.items()})
    assert out["learned_mixed"]["fallbacks"] == 0
    for k in out:
        assert rel(out[k]["corrected"], out["jacobi_fp64"]["corrected"]) < 1e-6, k
    assert out["learned_mixed"]["iters"] < 0.7 * out["jacobi_mixed"]["iters"], out
    assert out["learned_mixed"]["ms_per_rhs"] < out["jacobi_mixed"]["ms_per_rhs"], out
    # on these expander-like firm Laplacians vertex-dependent weights buy no
    # iterations beyond the degree-1 structure (measured: 14.04 trained vs
    # 14.01 uniform at 400k workers); the trained weights must not lose more
    # than 5 % to the uniform ones
    assert out["learned_mixed"]["iters"] <= 1.05 * out["uniform_mixed"]["iters"], out
