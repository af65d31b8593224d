"""Numerical MCSE attachment, host side (no device): the request gates of
``vckss_rust_engine_numerical_preflight_v1`` against the plugin's statuses
for the same requests, and the covariance algebra (raw, PSD projection,
MCSE with contrast (1, 1, 2)) against the plugin's own results, both from
``tests/golden/numerical_cases.json`` (made by running the plugin)."""

import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

from fevc_b200 import abi

import make_golden

CASES = json.loads((Path(__file__).resolve().parent / "golden" / "numerical_cases.json").read_text())


def finalize(lib, conditional, leverage) -> dict:
    out = abi.NumericalResultV1()
    c = np.ascontiguousarray(conditional, dtype=np.float64).reshape(9)
    l = np.ascontiguousarray(leverage, dtype=np.float64).reshape(9)
    st = lib.fevcb_numerical_finalize_v1(c.ctypes.data_as(C.c_void_p), l.ctypes.data_as(C.c_void_p),
                                         C.byref(out), C.sizeof(out))
    assert st == 0
    return {k: (list(getattr(out, k)) if k in ("raw", "usable", "mcse") else getattr(out, k))
            for k in ("status", "raw", "usable", "mcse", "psd_adjustment")}


@pytest.mark.parametrize("name", sorted(CASES["preflight"]))
def test_preflight_status_matches_the_plugin(lib, name):
    e = abi.Engine(lib)
    req = make_golden.numerical_request(e, 24, 2)
    muts = make_golden.NUMERICAL_PREFLIGHT[name]
    for path, value in muts:
        make_golden._set_path(req, path, value)
    if any(p.startswith("point.") for p, _ in muts) and not any(
            p in ("point.v3.request_signature", "controls_count") for p, _ in muts):
        req.point.v3.request_signature = abi.capability_signature_v3(req.point, req.controls_count)
    assert lib.vckss_rust_engine_numerical_preflight_v1(C.byref(req)) == CASES["preflight"][name]


@pytest.mark.parametrize("name", sorted(CASES["cases"]))
def test_covariance_algebra_matches_the_plugin(lib, name):
    rec = CASES["cases"][name]["record"]
    got = finalize(lib, rec["conditional"], rec["leverage"])
    assert got["status"] == (2 if rec["status"] == 1 else rec["status"])
    scale = max(np.max(np.abs(rec["raw"])), 1e-300)
    for key in ("raw", "usable"):
        assert np.max(np.abs(np.array(got[key]) - np.array(rec[key]))) <= 1e-14 * scale, key
    want = np.array(rec["mcse"])
    assert np.max(np.abs(np.array(got["mcse"]) - want)) <= 1e-13 * max(np.max(want), 1e-300)
    assert abs(got["psd_adjustment"] - rec["psd_adjustment"]) <= 1e-14 * scale


def test_covariance_algebra_edge_cases(lib):
    zero = np.zeros((3, 3))
    got = finalize(lib, zero, zero)
    assert got["status"] == 2 and got["mcse"] == [0.0] * 4 and got["usable"] == [0.0] * 9
    cond = np.diag([4e-8, 1e-8, 2e-8])
    # a leverage part that makes the sum indefinite well beyond roundoff: unstable, no usable matrix
    got = finalize(lib, cond, np.diag([0.0, -3e-8, 0.0]))
    assert got["status"] == 4 and np.all(np.isnan(got["usable"])) and np.all(np.isnan(got["mcse"]))
    # nonfinite input
    got = finalize(lib, cond, np.full((3, 3), np.nan))
    assert got["status"] == 6 and np.all(np.isnan(got["mcse"]))
    # a PSD sum: the symmetrised raw matrix is usable as it stands
    lev = np.array([[1e-8, 2e-9, 0.0], [2e-9, 3e-9, 1e-9], [0.0, 1e-9, 5e-9]])
    got = finalize(lib, cond, lev)
    raw = cond + lev
    assert got["status"] == 2
    assert np.allclose(np.array(got["usable"]).reshape(3, 3), raw, rtol=1e-15, atol=0)
    c = np.array([1.0, 1.0, 2.0])
    assert np.isclose(got["mcse"][3], np.sqrt(c @ raw @ c), rtol=1e-14)
    assert np.allclose(got["mcse"][:3], np.sqrt(np.diag(raw)), rtol=1e-15)


def test_numerical_result_without_attachment_is_refused(lib):
    e = abi.Engine(lib)
    out = abi.NumericalResultV1()
    # unknown generation
    assert lib.vckss_rust_engine_numerical_result_v1(987654321, C.byref(out), C.sizeof(out)) != 0
    assert lib.vckss_rust_numerical_schema_v1() == 1
