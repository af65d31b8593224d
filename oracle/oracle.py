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
