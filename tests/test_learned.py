"""The learned preconditioner's CPU side: the numpy oracle's reverse-mode
gradient against finite differences, the parameter layout, and the C ABI
entry points (no GPU)."""

import ctypes as C

import numpy as np
import pytest

from fevc_b200 import abi, learned
from oracle import gnn_oracle


def small_problem(seed=0, n=30, P=6):
    rng = np.random.default_rng(seed)
    rows = [set() for _ in range(n)]
    for v in range(n):
        for u in rng.choice(n, 3, replace=False):
            if u != v:
                rows[v].add(int(u))
                rows[u].add(v)
    w = {}
    for v in range(n):
        for u in rows[v]:
            k = (min(u, v), max(u, v))
            w.setdefault(k, float(rng.uniform(0.2, 2.0)))
    ptr, col, val = [0], [], []
    for v in range(n):
        for u in sorted(rows[v]):
            col.append(u)
            val.append(w[(min(u, v), max(u, v))])
        ptr.append(len(col))
    ptr, col, val = np.array(ptr), np.array(col), np.array(val)
    diag = np.array([val[ptr[v]:ptr[v + 1]].sum() for v in range(n)])
    d = {"n": n, "pairs": P, "ptr": ptr, "col": col, "val": val, "diag": diag,
         "X": rng.normal(size=(n, 8)), "E": rng.normal(size=(n, P))}
    _, L, _ = gnn_oracle.adjacency(d)
    # pairs consistent with the loss: y_0 = r / d with r = L e
    d["Y"] = ((L @ d["E"]) / diag[:, None])[None]
    d["ELE"] = np.einsum("vj,vj->j", d["E"], L @ d["E"])
    return d


def test_oracle_gradient_matches_finite_differences():
    d = small_problem()
    _, _, total = gnn_oracle.layout()
    rng = np.random.default_rng(3)
    params = rng.normal(scale=0.15, size=total)
    loss, grad = gnn_oracle.loss_and_grad(d, params, round_weights=False)
    assert np.isfinite(loss) and grad.shape == (total,)
    h = 1e-6
    for idx in rng.choice(total, 16, replace=False):
        up, dn = params.copy(), params.copy()
        up[idx] += h
        dn[idx] -= h
        fd = (gnn_oracle.loss_and_grad(d, up, round_weights=False)[0]
              - gnn_oracle.loss_and_grad(d, dn, round_weights=False)[0]) / (2 * h)
        assert abs(fd - grad[idx]) <= 1e-6 + 1e-5 * abs(fd), (idx, fd, grad[idx])


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -2.5, 3.0e-3], dtype=np.float32)
    r = gnn_oracle.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # halfway to 1.0078125 rounds to even
    assert r[2] == 1.0078125
    assert r[3] == -2.5


def test_parameter_layout_and_initial_params(lib):
    n = learned.param_count(lib)
    assert n == gnn_oracle.layout()[2] == 25986
    p0, p1 = learned.initial_params(lib, 1), learned.initial_params(lib, 1)
    assert np.array_equal(p0, p1) and np.all(np.isfinite(p0))
    # untrained network: s = softplus(b_s) = 1 and a = s^2 + a_min + softplus(b_a)
    # = 1.05 at every vertex (the uniform first-order Neumann stage)
    s = np.logaddexp(0.0, p0[-1])
    a = s * s + gnn_oracle.A_MIN + np.logaddexp(0.0, p0[-2])
    assert abs(s - 1.0) < 1e-6 and abs(a - 1.05) < 1e-6


def test_install_validates_parameters(lib):
    with pytest.raises(abi.EngineError) as err:
        learned.install(lib, np.zeros(10, dtype=np.float32))
    assert err.value.code == 20
    bad = learned.initial_params(lib)
    bad[5] = np.nan
    with pytest.raises(abi.EngineError):
        learned.install(lib, bad)


def test_trainer_refuses_without_gpu(lib, has_gpu):
    if has_gpu:
        pytest.skip("a GPU is visible")
    h = C.c_uint64(0)
    assert lib.fevcb_learned_trainer_create_v1(1, C.byref(h)) == 11
