"""ctypes bridge to the C oracle (test infrastructure only).

``run(lib, generation, ...)`` reads the prepared problem of an active
generation through ``fevcb_engine_problem_view_v1`` and runs the CPU
restatement of the reference estimator on it.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import build as _build

u32p, u64p, dp = C.POINTER(C.c_uint32), C.POINTER(C.c_uint64), C.POINTER(C.c_double)


class OracleProblem(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("rows", "workers", "firms", "cells", "units", "strata", "physical_total")] + [
        ("target_total", C.c_double), ("row_worker", u32p), ("row_firm", u32p), ("row_cell", u32p),
        ("row_outcome", dp), ("row_target", dp), ("row_frequency", u64p), ("cell_worker", u32p),
        ("cell_firm", u32p), ("cell_weight", dp), ("cell_outcome_sum", dp), ("cell_target_sum", dp),
        ("unit_cell", u32p), ("unit_count", u64p), ("unit_rank", u64p), ("unit_outcome_sum", dp),
        ("stratum_cell", u32p), ("stratum_per_copy", dp), ("stratum_count", u64p), ("stratum_rank", u64p),
        ("controls", C.c_uint64), ("control_values", dp), ("group_ptr", u64p), ("group_rows", u32p),
        ("row_rank", u64p), ("row_copy_offset", u64p), ("deletion_mode", C.c_uint64)]


class ProblemView(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("reserved", C.c_uint32)] + OracleProblem._fields_


class OracleOptions(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("probes", C.c_uint32), ("centering", C.c_uint32), ("tolerance", C.c_double),
                ("rank_tolerance", C.c_double), ("block_tolerance", C.c_double), ("dense_limit", C.c_uint32),
                ("probe_begin", C.c_uint32), ("probe_end", C.c_uint32), ("phase", C.c_int32),
                ("reserved", C.c_uint32), ("shard_io", dp)]


class OracleResult(C.Structure):
    _fields_ = [("plugin", C.c_double * 4), ("correction", C.c_double * 4), ("corrected", C.c_double * 4),
                ("mcse", C.c_double * 4)] + [(n, dp) for n in (
                    "fitted_cell", "projection_share", "residual_share", "finite_bias", "finite_variance",
                    "residual_mass", "deleted_mass", "cell_correction_weight", "target_draws")] + [
                ("solves", C.c_uint64), ("cg_iterations", C.c_uint64), ("error_code", C.c_int),
                ("error", C.c_char * 256)]


_LIB = None


def library() -> C.CDLL:
    global _LIB
    if _LIB is None:
        _LIB = C.CDLL(str(_build.build()))
        _LIB.oracle_jla.restype = C.c_int
        _LIB.oracle_jla.argtypes = [C.POINTER(OracleProblem), C.POINTER(OracleOptions), C.POINTER(OracleResult)]
        _LIB.oracle_jla_generic.restype = C.c_int
        _LIB.oracle_jla_generic.argtypes = _LIB.oracle_jla.argtypes
        _LIB.oracle_rademacher_sum.restype = C.c_int64
        _LIB.oracle_rademacher_sum.argtypes = [C.c_uint64] * 5 + [C.POINTER(C.c_int)]
        _LIB.oracle_philox_block.restype = None
        _LIB.oracle_philox_block.argtypes = [C.c_uint64] * 5 + [C.POINTER(C.c_uint64)]
    return _LIB


def philox_block(seed, tag, probe_block, entity, word):
    out = (C.c_uint64 * 4)()
    library().oracle_philox_block(seed, tag, probe_block, entity, word, out)
    return list(out)


def rademacher_sum(seed, tag, probe, entity, trials):
    ok = C.c_int(0)
    v = library().oracle_rademacher_sum(seed, tag, probe, entity, trials, C.byref(ok))
    if not ok.value:
        raise ValueError("trial count must lie in [1, 2^53]")
    return v


def problem_view(lib, generation) -> OracleProblem:
    lib.fevcb_engine_problem_view_v1.restype = C.c_int32
    lib.fevcb_engine_problem_view_v1.argtypes = [C.c_uint64, C.c_void_p, C.c_uint32]
    v = ProblemView()
    st = lib.fevcb_engine_problem_view_v1(generation, C.byref(v), C.sizeof(v))
    if st != 0:
        raise RuntimeError(f"problem view failed: {st}")
    p = OracleProblem()
    for name, _ in OracleProblem._fields_:
        setattr(p, name, getattr(v, name))
    return p


def run(problem: OracleProblem, *, seed=8675309, probes=200, centering=0, tolerance=1e-13, rank_tolerance=1e-10,
        block_tolerance=1e-10, dense_limit=3000) -> dict:
    lib = library()
    G, Cn, P = problem.units, problem.cells, probes
    arrays = {n: np.zeros(G) for n in ("projection_share", "residual_share", "finite_bias", "finite_variance",
                                       "residual_mass", "deleted_mass")}
    arrays["fitted_cell"] = np.zeros(Cn)
    arrays["cell_correction_weight"] = np.zeros(Cn)
    arrays["target_draws"] = np.zeros(4 * P)
    res = OracleResult()
    for n, a in arrays.items():
        setattr(res, n, a.ctypes.data_as(dp))
    opt = OracleOptions(seed, probes, centering, tolerance, rank_tolerance, block_tolerance, dense_limit, 0, 0, 0, 0,
                        None)
    fn = lib.oracle_jla_generic if (problem.controls or problem.deletion_mode == 2) else lib.oracle_jla
    code = fn(C.byref(problem), C.byref(opt), C.byref(res))
    if code != 0:
        raise RuntimeError(f"oracle failed [{code}]: {res.error.decode()}")
    out = {k: np.array(getattr(res, k)[:]) for k in ("plugin", "correction", "corrected", "mcse")}
    arrays["target_draws"] = arrays["target_draws"].reshape(P, 4)
    out.update(arrays)
    out["solves"] = res.solves
    out["cg_iterations"] = res.cg_iterations
    return out


def shard(problem: OracleProblem, *, phase: int, probe_begin: int, probe_end: int, io: np.ndarray, seed=8675309,
          probes=200, centering=0, tolerance=1e-13, rank_tolerance=1e-10, block_tolerance=1e-10,
          dense_limit=3000) -> dict:
    """One phase of a probe shard of the compressed estimator: phase 1 writes
    the range's leverage moment sums into `io` (units x 5); phase 2 reads the
    summed moments from `io` and returns the range's target draws and the
    plug-in components."""
    lib = library()
    G, Cn, P = problem.units, problem.cells, probes
    arrays = {n: np.zeros(G) for n in ("projection_share", "residual_share", "finite_bias", "finite_variance",
                                       "residual_mass", "deleted_mass")}
    arrays["fitted_cell"] = np.zeros(Cn)
    arrays["cell_correction_weight"] = np.zeros(Cn)
    arrays["target_draws"] = np.zeros(4 * P)
    res = OracleResult()
    for n, a in arrays.items():
        setattr(res, n, a.ctypes.data_as(dp))
    io = np.ascontiguousarray(io, dtype=np.float64)
    opt = OracleOptions(seed, probes, centering, tolerance, rank_tolerance, block_tolerance, dense_limit,
                        probe_begin, probe_end, phase, 0, io.ctypes.data_as(dp))
    code = lib.oracle_jla(C.byref(problem), C.byref(opt), C.byref(res))
    if code != 0:
        raise RuntimeError(f"oracle failed [{code}]: {res.error.decode()}")
    draws = arrays["target_draws"].reshape(P, 4)[probe_begin:probe_end].copy()
    return {"io": io, "draws": draws, "plugin": np.array(res.plugin[:])}


def exact(problem: OracleProblem, *, centering: int = 0, block_tolerance: float = 1e-10) -> dict:
    """Exact leverages for match deletion without controls (dense numpy).

    Restates the reference's dense estimator (rust/crates/vckss-core/src/
    exact_estimator.rs:560-1000 full fit and match loop, 1448-1600
    match_block_action, 1698-1786 TargetMoments::bilinear) for blocks whose
    rows share one design row x_c = (e_w, e_f): with S = X'WX grounded at the
    last firm, z_c = S^-1 x_c and h_c = x_c' z_c, a deletion unit g of n_g
    frequency mass in cell c contributes (sum of centred outcomes)(sum of
    residuals) / (1 - n_g h_c) times the target bilinear forms of z_c.
    """
    W, F, Cn, G = int(problem.workers), int(problem.firms), int(problem.cells), int(problem.units)
    arr = lambda p, n: np.ctypeslib.as_array(p, shape=(n,)).copy()  # noqa: E731
    cw = arr(problem.cell_worker, Cn).astype(np.int64)
    cf = arr(problem.cell_firm, Cn).astype(np.int64)
    wgt = arr(problem.cell_weight, Cn)
    ysum = arr(problem.cell_outcome_sum, Cn)
    tsum = arr(problem.cell_target_sum, Cn)
    ucell = arr(problem.unit_cell, G).astype(np.int64)
    ucount = arr(problem.unit_count, G).astype(np.float64)
    uys = arr(problem.unit_outcome_sum, G)
    T = float(problem.target_total)
    dim = W + F - 1  # the last firm is grounded (the quotient's zero-sum firm block)
    S = np.zeros((W + F, W + F))
    np.add.at(S, (cw, cw), wgt)
    np.add.at(S, (W + cf, W + cf), wgt)
    np.add.at(S, (cw, W + cf), wgt)
    np.add.at(S, (W + cf, cw), wgt)
    Sinv = np.linalg.inv(S[:dim, :dim])
    # S^+ in the grounded coordinates, padded with the grounded firm's zero
    # row and column (x_c of a cell in the last firm has no coordinate there)
    full = np.zeros((W + F, W + F))
    full[:dim, :dim] = Sinv
    # the fit: beta = S^+ X'Wy, effects centred by the target weights below
    rhs = np.bincount(cw, ysum, W + F) + np.bincount(W + cf, ysum, W + F)
    beta = full @ rhs
    alpha_fit, psi_fit = beta[:W], beta[W:]
    fitted = alpha_fit[cw] + psi_fit[cf]
    ws = np.bincount(cw, tsum, W) / T
    fs = np.bincount(cf, tsum, F) / T
    m = tsum / T
    am, pm = ws @ alpha_fit, fs @ psi_fit
    plugin_w = ws @ (alpha_fit - am) ** 2
    plugin_f = fs @ (psi_fit - pm) ** 2
    plugin_c = m @ ((alpha_fit[cw] - am) * (psi_fit[cf] - pm))
    plugin = np.array([plugin_w, plugin_f, plugin_c, plugin_w + plugin_f + 2 * plugin_c])
    # exact leverages and target forms of z_c, in column chunks
    B = np.zeros((Cn, 3))
    h = np.zeros(Cn)
    for lo in range(0, Cn, 2048):
        idx = np.arange(lo, min(Cn, lo + 2048))
        Z = full[:, cw[idx]] + full[:, W + cf[idx]]  # (W+F) x chunk: columns z_c
        Za, Zp = Z[:W], Z[W:]
        h[idx] = Za[cw[idx], np.arange(idx.size)] + Zp[cf[idx], np.arange(idx.size)]
        a1, p1 = ws @ Za, fs @ Zp
        B[idx, 0] = ws @ Za ** 2 - a1 ** 2
        B[idx, 1] = fs @ Zp ** 2 - p1 ** 2
        B[idx, 2] = m @ (Za[cw] * Zp[cf]) - a1 * p1
    ybar = 0.0
    if centering == 1:
        rows, phys = int(problem.rows), float(problem.physical_total)
        y = arr(problem.row_outcome, rows)
        freq = arr(problem.row_frequency, rows).astype(np.float64)
        ybar = y[0] + np.sum((y - y[0]) * (freq / phys))
    maker = 1.0 - ucount * h[ucell]
    if np.any(maker <= block_tolerance):
        raise RuntimeError("a match residual block is singular")
    omega = np.bincount(ucell, (uys - ybar * ucount) * (uys - ucount * fitted[ucell]) / maker, Cn)
    corr = omega @ B
    correction = np.array([corr[0], corr[1], corr[2], corr[0] + corr[1] + 2 * corr[2]])
    return {"plugin": plugin, "correction": correction, "corrected": plugin - correction,
            "mcse": np.zeros(4), "leverage": ucount * h[ucell]}
