"""Regenerate the golden fixtures in this directory from the reference plugin.

The reference's shipped Linux plugin (``fevc/fevc_rust_linux_x64.plugin`` in
the reference checkout) is loaded with dlopen and driven only through its C ABI
(the same ctypes bindings the tests use for this library).  Every fixture
records the inputs (or the seeded generator call that reproduces them, with a
checksum of the generated columns) and the plugin's outputs:

* ``prep_cases.json``   retained masks, preparation receipts and status codes
                         for panels and adversarial inputs;
* ``jla_cases.json``     components (plug-in, correction, corrected, MCSE) of
                         solved panels at a tight diagonal-PCG tolerance.

Run from the repository root:  ``python tests/golden/make_golden.py``.
"""

from __future__ import annotations

import ctypes as C
import hashlib
import json
import os
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from fevc_b200 import abi  # noqa: E402
from fevc_b200.panel import Panel, generate_panel  # noqa: E402

PLUGIN = Path("/root/reference/fevc/fevc_rust_linux_x64.plugin")
HERE = Path(__file__).resolve().parent


def panel_digest(p: Panel) -> str:
    h = hashlib.sha256()
    for a in (p.worker, p.firm, p.deletion, p.outcome, p.frequency, p.target_weight, *p.controls):
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return h.hexdigest()


def kat12() -> Panel:
    """The 12-row design of the reference's shared-atom known-answer test
    (rust/crates/vckss-core/tests/rust_mata_shared_atoms.rs:39-47), in its
    permuted row order."""
    worker = [1, 1, 1, 1, 2, 2, 2, 2, 9, 9, 10, 10]
    firm = [1, 1, 2, 2, 1, 1, 2, 2, 9, 10, 9, 10]
    deletion = [11, 12, 21, 22, 31, 32, 41, 42, 91, 92, 93, 94]
    outcome = [1, 3, 0, 2, -1, 1, 2, -2, 10, 11, 12, 13]
    frequency = [1, 2, 1, 2, 1, 3, 2, 1, 1, 1, 1, 1]
    target = [1, 2, 2, 2, 3, 9, 8, 4, 1, 1, 1, 1]
    order = [7, 2, 8, 5, 0, 9, 3, 11, 10, 1, 6, 4]
    g = lambda a: np.array([a[r] for r in order], dtype=np.float64)  # noqa: E731
    return Panel(g(worker), g(firm), g(deletion), g(outcome), g(frequency), g(target))


def weighted_panel(seed: int) -> Panel:
    """A generated panel with literal frequency weights, uneven target weights
    and several rows per deletion unit (exercises the per-copy mass strata)."""
    p = generate_panel(1500, 120, 5, move_p=0.25, seed=seed)
    rng = np.random.default_rng(seed + 1)
    p.frequency = rng.integers(1, 4, p.rows).astype(np.float64)
    p.target_weight = np.round(rng.uniform(0.5, 3.0, p.rows) * 4) / 4 * p.frequency
    return p


PANELS = {
    "kat12": dict(build=lambda: kat12(), probes=5),
    "small_2k": dict(build=lambda: generate_panel(2000, 150, 5, move_p=0.2, seed=11), probes=24),
    "exact_20k": dict(build=lambda: generate_panel(20000, 1000, 5, seed=20261203), probes=40),
    "weighted_1500": dict(build=lambda: weighted_panel(5), probes=16),
    "pareto13_4k": dict(build=lambda: generate_panel(4000, 200, 6, move_p=0.08, pareto_shape=1.3, seed=3), probes=20),
    "regions_4k": dict(build=lambda: generate_panel(4000, 200, 6, regions=2, cross_p=0.01, seed=4), probes=20),
}


CONTROL_PANELS = {
    "controls_2k": dict(build=lambda: generate_panel(2000, 150, 5, move_p=0.2, year_controls=True, seed=11), probes=16),
    "controls_weighted_1500": dict(build=lambda: weighted_controls_panel(6), probes=12),
    "controls_6p_4k": dict(build=lambda: generate_panel(4000, 200, 6, move_p=0.15, year_controls=True, seed=9),
                           probes=12),
}


def weighted_controls_panel(seed: int) -> Panel:
    """Year controls with literal frequencies, uneven target weights and
    repeated rows per match (multi-row deletion groups)."""
    p = generate_panel(1500, 120, 5, move_p=0.25, year_controls=True, seed=seed)
    rng = np.random.default_rng(seed + 1)
    p.frequency = rng.integers(1, 4, p.rows).astype(np.float64)
    p.target_weight = np.round(rng.uniform(0.5, 3.0, p.rows) * 4) / 4 * p.frequency
    return p


def duplicated_rows_panel(seed: int, controls: bool) -> Panel:
    """Literal frequencies plus repeated rows: about a sixth of the rows appear
    again with the same worker, firm, outcome, controls and per-copy target
    mass (some with another frequency), so leave-observation-out classes hold
    several rows whose copies are numbered through the class."""
    p = generate_panel(1500, 120, 5, move_p=0.25, year_controls=controls, seed=seed)
    rng = np.random.default_rng(seed + 2)
    p.frequency = rng.integers(1, 4, p.rows).astype(np.float64)
    per_copy = np.round(rng.uniform(0.5, 3.0, p.rows) * 4) / 4
    p.target_weight = per_copy * p.frequency
    pick = np.sort(rng.choice(p.rows, p.rows // 6, replace=False))
    freq = p.frequency[pick].copy()
    refreq = rng.random(pick.size) < 0.4
    freq[refreq] = rng.integers(1, 5, int(refreq.sum()))
    cat = lambda a, b: np.concatenate([a, b])
    return Panel(cat(p.worker, p.worker[pick]), cat(p.firm, p.firm[pick]), cat(p.deletion, p.deletion[pick]),
                 cat(p.outcome, p.outcome[pick]), cat(p.frequency, freq), cat(p.target_weight, per_copy[pick] * freq),
                 [cat(c, c[pick]) for c in p.controls])


OBSERVATION_PANELS = {
    "obs_2k": dict(build=lambda: generate_panel(2000, 150, 5, move_p=0.2, seed=11), probes=16),
    "obs_controls_2k": dict(build=lambda: generate_panel(2000, 150, 5, move_p=0.2, year_controls=True, seed=11),
                            probes=16),
    "obs_duplicates_1500": dict(build=lambda: duplicated_rows_panel(8, False), probes=12),
    "obs_controls_duplicates_1500": dict(build=lambda: duplicated_rows_panel(9, True), probes=12),
}


def solve_record_v5(lib, panel: Panel, probes: int, centering: int, deletion_mode: int = 1) -> dict:
    """The plugin's generic engine (controls or leave-observation-out) through
    V5, diagonal PCG at 1e-13."""
    e = abi.Engine(lib)
    e.prepare(panel, deletion_mode=deletion_mode)
    if centering:
        e.centering(centering)
    q = e.default_request_v5(deletion_mode)
    v1 = q.v4.v3.v2.v1
    v1.probes = probes
    v1.solver_route = 2
    v1.pcg_tolerance = 1e-13
    v1.maximum_iterations = 20000
    v1.leverage_batch_width = 4
    v1.target_batch_width = 4
    q.v4.v3.v2.algorithm = 2
    q.v4.v3.engine = 2
    q.v4.v3.batch_mode = 1
    q.v4.leverage_batch_mode = 1
    q.v4.target_batch_mode = 1
    q.threads = 4
    q.tolerance_supplied = 1
    e.solve_v5(q, controls_count=len(panel.controls))
    res = e.result()
    e.release()
    return {"seed": int(v1.seed), "probes": probes, "centering": centering, "pcg_tolerance": 1e-13,
            **{k: list(v) for k, v in res.items()}}


CMG_PANELS = {
    **{k: PANELS[k] for k in ("kat12", "small_2k", "exact_20k", "weighted_1500", "pareto13_4k", "regions_4k")},
    "cmg_60k": dict(build=lambda: generate_panel(60000, 6000, 5, seed=61), probes=4),
    "cmg_pareto_40k": dict(build=lambda: generate_panel(40000, 4000, 6, move_p=0.08, pareto_shape=1.3, seed=62),
                           probes=4),
    "cmg_regions_60k": dict(build=lambda: generate_panel(60000, 6000, 6, regions=2, cross_p=0.002, seed=63),
                            probes=4),
}


def cmg_record(lib, panel: Panel) -> dict:
    """The plugin's hybrid graph and CMG hierarchy as its full-CMG receipt
    reports them, after a 4-probe CMG_FULL_V2 solve."""
    e = abi.Engine(lib)
    e.prepare(panel)
    q = e.default_request_v5()
    v1 = q.v4.v3.v2.v1
    v1.probes = 4
    v1.pcg_tolerance = 1e-8
    v1.solver_route = 3
    q.v4.v3.v2.algorithm = 2
    q.threads = 4
    q.tolerance_supplied = 1
    q.full_cmg_v2 = 1
    e.solve_v5(q)
    r = abi.FullCmgReceiptV1()
    e.check(lib.vckss_rust_engine_full_cmg_receipt_v1(e.generation, C.byref(r), C.sizeof(r)))
    e.release()
    return {k: int(getattr(r, k)) for k in ("vertices", "edges", "hierarchy_levels", "terminal_vertices")}


def error_cases():
    base = kat12()

    def mod(**kw):
        p = Panel(*(np.array(getattr(base, f), copy=True) for f in
                    ("worker", "firm", "deletion", "outcome", "frequency", "target_weight")))
        for k, fn in kw.items():
            setattr(p, k, fn(getattr(p, k)))
        return p

    def setv(i, v):
        def f(a):
            a[i] = v
            return a
        return f

    return {
        "nonfinite_outcome": mod(outcome=setv(3, np.nan)),
        "zero_frequency": mod(frequency=setv(2, 0.0)),
        "fractional_frequency": mod(frequency=setv(2, 1.5)),
        "negative_target": mod(target_weight=setv(1, -1.0)),
        "zero_worker_id": mod(worker=setv(0, 0.0)),
        "fractional_firm_id": mod(firm=setv(0, 1.5)),
        "deletion_crosses_cells": mod(deletion=setv(0, 12.0)),
        "all_zero_target": mod(target_weight=lambda a: a * 0.0),
        # two identical disconnected blocks: largest-component tie
        "tied_components": Panel(np.array([1, 1, 2, 2, 3, 3, 4, 4], float), np.array([1, 2, 1, 2, 3, 4, 3, 4], float),
                                 np.arange(1, 9, dtype=float), np.arange(8, dtype=float), np.ones(8), np.ones(8)),
        # a single firm: nothing identified
        "single_firm": Panel(np.array([1, 1, 2, 2], float), np.array([1, 1, 1, 1], float),
                             np.arange(1, 5, dtype=float), np.arange(4, dtype=float), np.ones(4), np.ones(4)),
    }


def prepare_record(lib, panel: Panel, deletion_mode: int = 1) -> dict:
    e = abi.Engine(lib)
    try:
        e.prepare(panel, deletion_mode=deletion_mode)
    except abi.EngineError as err:
        return {"status": err.code}
    rc = e.receipt()
    mask = e.retained_mask(panel.rows)
    e.release()
    keep = {k: v for k, v in rc.items() if k not in (
        "generation", "struct_size", "reserved", "memory_limit_bytes", "caller_copy_bytes",
        "preparation_peak_forecast_bytes", "prepared_resident_bytes")}
    return {"status": 0, "receipt": keep, "mask_sha256": hashlib.sha256(mask.tobytes()).hexdigest(),
            "retained": int(mask.sum())}


def solve_record(lib, panel: Panel, probes: int, centering: int) -> dict:
    e = abi.Engine(lib)
    e.prepare(panel)
    if centering:
        e.centering(centering)
    q = e.default_request()
    q.probes = probes
    q.leverage_batch_width = 4
    q.target_batch_width = 4
    q.solver_route = 2  # diagonal PCG
    q.allow_automatic_cmg_setup_fallback = 0
    q.pcg_tolerance = 1e-13
    q.maximum_iterations = 20000
    q.residual_replacement_interval = 50
    e.solve(q)
    res = e.result()
    e.release()
    return {"seed": int(q.seed), "probes": probes, "centering": centering, "pcg_tolerance": 1e-13,
            **{k: list(v) for k, v in res.items()}}


# Detailed receipts V7 of V5 solves: the request-side and count fields the B200
# engine reports the same way (tests/test_gpu_receipts.py lists them).
RECEIPT_PANELS = {
    "match_small_2k": dict(build=lambda: PANELS["small_2k"]["build"](), probes=8, deletion_mode=1),
    "controls": dict(build=lambda: CONTROL_PANELS[next(iter(CONTROL_PANELS))]["build"](), probes=8,
                     deletion_mode=1),
    "observation": dict(build=lambda: OBSERVATION_PANELS[next(iter(OBSERVATION_PANELS))]["build"](), probes=8,
                        deletion_mode=2),
}


def receipt_request(e, probes: int, deletion_mode: int, controls: int):
    q = e.default_request_v5(deletion_mode)
    v1 = q.v4.v3.v2.v1
    v1.probes = probes
    v1.solver_route = 2
    v1.pcg_tolerance = 1e-13
    v1.maximum_iterations = 20000
    v1.leverage_batch_width = 4
    v1.target_batch_width = 4
    q.v4.v3.v2.algorithm = 2
    q.v4.v3.engine = 2 if (controls or deletion_mode == 2) else 0
    q.v4.v3.batch_mode = 1
    q.v4.leverage_batch_mode = 1
    q.v4.target_batch_mode = 1
    q.threads = 4
    q.tolerance_supplied = 1
    return q


def receipt_record(lib, panel: Panel, probes: int, deletion_mode: int) -> dict:
    e = abi.Engine(lib)
    e.prepare(panel, deletion_mode=deletion_mode)
    q = receipt_request(e, probes, deletion_mode, len(panel.controls))
    e.solve_v5(q, controls_count=len(panel.controls))
    r = e.detailed_receipt(7)
    e.release()
    return {"probes": probes, "deletion_mode": deletion_mode, "receipt": r.as_dict()}


def write_receipt_cases(lib, meta: dict) -> None:
    cases = {}
    for name, spec in RECEIPT_PANELS.items():
        panel = spec["build"]()
        cases[name] = {"panel_sha256": panel_digest(panel),
                       **receipt_record(lib, panel, spec["probes"], spec["deletion_mode"])}
        print(name, cases[name]["receipt"]["v6"]["v5"]["v4"]["v3"]["v2"]["topology_checksum"])
    (HERE / "receipt_cases.json").write_text(json.dumps({"meta": meta, "panels": cases}, indent=1))


def write_cmg_cases(lib, meta: dict) -> None:
    lib.vckss_rust_engine_full_cmg_receipt_v1.restype = C.c_int32
    lib.vckss_rust_engine_full_cmg_receipt_v1.argtypes = [C.c_uint64, C.c_void_p, C.c_uint32]
    cmg = {}
    for name, spec in CMG_PANELS.items():
        panel = spec["build"]()
        cmg[name] = {"panel_sha256": panel_digest(panel), **cmg_record(lib, panel)}
        print(name, cmg[name])
    (HERE / "cmg_cases.json").write_text(json.dumps({"meta": meta, "panels": cmg}, indent=1))


# Components of the plugin at reduced sizes of the configured benchmark
# panels (fevc_b200/panel.py named panels): the same seeded generator, the
# same probes and seed, supplied tolerance 1e-10.  The plugin's production
# route (CMG_FULL_V2) is tried first; when its refinement ladder refuses the
# panel the record falls back to the plugin's diagonal PCG route and says so.
SIZED_PANELS = {
    "plain_1m@0.1": dict(name="plain_1m", scale=0.1, probes=24),
    "learned_10m@0.02": dict(name="learned_10m", scale=0.02, probes=48),
}


def sized_record(lib, name: str, scale: float, probes: int) -> dict:
    from fevc_b200.panel import named_panel

    panel = named_panel(name, scale)
    deletion = 2 if panel.info.get("deletion") == "observation" else 1
    last = None
    for route in ("cmg_full_v2", "diagonal"):
        e = abi.Engine(lib)
        e.prepare(panel, deletion_mode=deletion)
        q = e.default_request_v5(deletion)
        v1 = q.v4.v3.v2.v1
        v1.probes = probes
        v1.pcg_tolerance = 1e-10
        v1.maximum_iterations = 20000
        q.v4.v3.v2.algorithm = 2
        if deletion == 2:
            q.v4.v3.engine = 2
        q.tolerance_supplied = 1
        q.threads = os.cpu_count() or 1
        if route == "cmg_full_v2":
            q.full_cmg_v2 = 1
        else:
            v1.solver_route = 2
        try:
            e.solve_v5(q, controls_count=len(panel.controls))
        except abi.EngineError as err:
            last = f"{route}: {err}"
            e.release()
            continue
        res = e.result()
        e.release()
        return {"panel": name, "scale": scale, "rows": panel.rows, "panel_sha256": panel_digest(panel),
                "deletion_mode": deletion, "controls": len(panel.controls), "seed": int(v1.seed), "probes": probes,
                "pcg_tolerance": 1e-10, "route": route, "refused_route": last,
                **{k: list(v) for k, v in res.items()}}
    raise RuntimeError(f"the plugin refused {name}@{scale}: {last}")


def write_sized_cases(lib, meta: dict) -> None:
    cases = {}
    for key, spec in SIZED_PANELS.items():
        cases[key] = sized_record(lib, **spec)
        print(key, cases[key]["route"], cases[key]["corrected"])
    (HERE / "sized_cases.json").write_text(json.dumps({"meta": meta, "cases": cases}, indent=1))


# The plugin's exact estimator (algorithm EXACT through its solve_v2; the
# V4+ solves need the EXACT capability profile) on panels small enough for
# its single-threaded dense path (identified dimension <= 2000).
EXACT_PANELS = {
    "kat12": dict(build=lambda: kat12()),
    "exact_400": dict(build=lambda: generate_panel(400, 60, 5, move_p=0.3, seed=3)),
    "exact_weighted_500": dict(build=lambda: _weighted_small(500, 50, 13)),
}


def _weighted_small(workers: int, firms: int, seed: int) -> Panel:
    """Literal frequencies and uneven target weights on a small panel."""
    p = generate_panel(workers, firms, 5, move_p=0.3, seed=seed)
    rng = np.random.default_rng(seed + 1)
    p.frequency = rng.integers(1, 4, p.rows).astype(np.float64)
    p.target_weight = np.round(rng.uniform(0.5, 3.0, p.rows) * 4) / 4 * p.frequency
    return p


def exact_record(lib, panel: Panel, centering: int) -> dict:
    lib.vckss_rust_engine_solve_v2.restype = C.c_int32
    lib.vckss_rust_engine_solve_v2.argtypes = [C.c_uint64, C.c_void_p]
    e = abi.Engine(lib)
    e.prepare(panel)
    if centering:
        e.centering(centering)
    q = abi.SolveRequestV2()
    e.check(lib.vckss_rust_engine_default_solve_request_v2(C.byref(q), C.sizeof(q)))
    q.algorithm = 1
    q.exact_estimator_limit = 2000
    e.check(lib.vckss_rust_engine_solve_v2(e.generation, C.byref(q)))
    res = e.result()
    e.release()
    return {"centering": centering, "pcg_tolerance": q.v1.pcg_tolerance, **{k: list(v) for k, v in res.items()}}


def write_exact_cases(lib, meta: dict) -> None:
    cases = {}
    for name, spec in EXACT_PANELS.items():
        panel = spec["build"]()
        cases[name] = {"panel_sha256": panel_digest(panel), "records": [exact_record(lib, panel, c) for c in (0, 1)]}
        print(name, cases[name]["records"][0]["corrected"])
    (HERE / "exact_cases.json").write_text(json.dumps({"meta": meta, "cases": cases}, indent=1))


# The plugin's numerical MCSE attachment (vckss_rust_engine_solve_numerical_v1
# around a V4 point request, then numerical_result_v1 and numerical_rhs_v1):
# JLA on the compressed engine at a tight diagonal-PCG tolerance, an odd probe
# count (unequal target folds), literal frequencies, and the automatic
# algorithm on a panel within the exact limit (the exact-zero attachment).
NUMERICAL_PANELS = {
    "small_2k": dict(build=lambda: generate_panel(2000, 150, 5, move_p=0.2, seed=11), probes=24, algorithm=2),
    "odd_probes_2k": dict(build=lambda: generate_panel(2000, 150, 5, move_p=0.2, seed=12), probes=15, algorithm=2),
    "weighted_1500": dict(build=lambda: weighted_panel(5), probes=16, algorithm=2),
    "pareto13_4k": dict(build=lambda: generate_panel(4000, 200, 6, move_p=0.08, pareto_shape=1.3, seed=3),
                        probes=20, algorithm=2),
    "kat12_jla": dict(build=lambda: kat12(), probes=5, algorithm=2),
    "kat12_auto": dict(build=lambda: kat12(), probes=5, algorithm=0),
    "obs_2k": dict(build=lambda: generate_panel(2000, 150, 5, move_p=0.2, seed=11), probes=16, algorithm=2,
                   deletion=2),
    "obs_odd_2k": dict(build=lambda: generate_panel(2000, 150, 5, move_p=0.2, seed=13), probes=13, algorithm=2,
                       deletion=2),
    "obs_controls_2k": dict(build=lambda: generate_panel(2000, 150, 5, move_p=0.2, year_controls=True, seed=11),
                            probes=16, algorithm=2, deletion=2),
    "obs_duplicates_1500": dict(build=lambda: duplicated_rows_panel(8, False), probes=12, algorithm=2, deletion=2),
    "obs_controls_duplicates_1500": dict(build=lambda: duplicated_rows_panel(9, True), probes=12, algorithm=2,
                                         deletion=2),
    "controls_2k": dict(build=lambda: generate_panel(2000, 150, 5, move_p=0.2, year_controls=True, seed=11),
                        probes=16, algorithm=2),
    "controls_odd_2k": dict(build=lambda: generate_panel(2000, 150, 5, move_p=0.2, year_controls=True, seed=14),
                            probes=11, algorithm=2),
    "controls_weighted_1500": dict(build=lambda: weighted_controls_panel(6), probes=12, algorithm=2),
}

NUMERICAL_FIELDS = ("status", "engine", "leverage_probes", "target_probes", "target_fold_a", "target_fold_b",
                    "certified_replay_rhs", "executed_replay_rhs", "attempted_replay_rhs", "replay_generator_words",
                    "allocation_bound_bytes", "failed_replay_probe", "replay_error_code", "psd_adjustment",
                    "minimum_constrained", "minimum_residual_margin", "maximum_sensitivity_ratio", "score_means",
                    "conditional", "leverage", "raw", "usable", "mcse", "point_rhs")


def numerical_request(e, probes: int, algorithm: int, deletion: int = 1, controls: int = 0):
    """The numerical-attachment request the fixtures and tests use: a default
    V5 point with the probes, JLA or the automatic algorithm, diagonal PCG at
    1e-12 for JLA (the automatic algorithm keeps the automatic route), the
    panel's deletion mode and control count."""
    q = e.default_request_v5(deletion)
    v1 = q.v4.v3.v2.v1
    v1.probes = probes
    v1.pcg_tolerance = 1e-12
    v1.maximum_iterations = 20000
    q.v4.v3.v2.algorithm = algorithm
    if algorithm == 2:
        v1.solver_route = 2
    q.threads = 4
    q.tolerance_supplied = 1
    return e.numerical_request(q, controls)


def numerical_record(lib, panel: Panel, probes: int, algorithm: int, deletion: int = 1) -> dict:
    e = abi.Engine(lib)
    e.prepare(panel, deletion_mode=deletion)
    e.solve_numerical(numerical_request(e, probes, algorithm, deletion, len(panel.controls)))
    r = e.numerical_result()
    point = e.result()
    count, rhs = e.numerical_rhs(int(r["certified_replay_rhs"]))
    e.release()
    rec = {k: r[k] for k in NUMERICAL_FIELDS}
    rec = {k: (str(v) if isinstance(v, float) and not np.isfinite(v) else v) for k, v in rec.items()}
    rec["corrected"] = list(point["corrected"])
    rec["rhs"] = [[x["probe"], x["phase"], x["complete_residual"]] for x in rhs]
    return {"probes": probes, "algorithm": algorithm, "deletion": deletion, "pcg_tolerance": 1e-12, **rec}


# Request mutations for the preflight fixture (field path, value).
NUMERICAL_PREFLIGHT = {
    "base": [],
    "schema_2": [("schema_version", 2)],
    "reserved": [("reserved", 1)],
    "reserved_2": [("reserved_2", 3)],
    "tolerance_supplied_2": [("tolerance_supplied", 2)],
    "threads_0": [("threads", 0)],
    "probes_1": [("point.v3.v2.v1.probes", 1)],
    "projection": [("projection_requested", 1)],
    "component": [("component_requested", 1)],
    "exact_algorithm": [("point.v3.v2.algorithm", 1)],
    "exact_route": [("point.v3.v2.v1.solver_route", 1)],
    "no_rng": [("point.v3.v2.v1.rng_contract", 0)],
    "bad_signature": [("point.v3.request_signature", 12345)],
    "engine_compressed": [("point.v3.engine", 1)],
    "engine_unknown": [("point.v3.engine", 7)],
    "controls_mismatch": [("controls_count", 2)],
    "point_reserved": [("point.reserved_4", 1)],
    "abi_version": [("abi_version", 2)],
}


def _set_path(obj, path: str, value) -> None:
    *head, last = path.split(".")
    for h in head:
        obj = getattr(obj, h)
    setattr(obj, last, value)


def numerical_preflight_record(lib) -> dict:
    out = {}
    for name, muts in NUMERICAL_PREFLIGHT.items():
        e = abi.Engine(lib)
        req = numerical_request(e, 24, 2)
        resign = not any(p == "point.v3.request_signature" for p, _ in muts)
        for path, value in muts:
            _set_path(req, path, value)
        if resign and any(p.startswith("point.") or p == "controls_count" for p, _ in muts):
            if not any(p == "controls_count" for p, _ in muts):
                req.point.v3.request_signature = abi.capability_signature_v3(req.point, req.controls_count)
        out[name] = int(lib.vckss_rust_engine_numerical_preflight_v1(C.byref(req)))
    return out


def write_numerical_cases(lib, meta: dict) -> None:
    cases = {}
    for name, spec in NUMERICAL_PANELS.items():
        panel = spec["build"]()
        cases[name] = {"panel_sha256": panel_digest(panel),
                       "record": numerical_record(lib, panel, spec["probes"], spec["algorithm"],
                                                  spec.get("deletion", 1))}
        print(name, cases[name]["record"]["status"], cases[name]["record"]["mcse"])
    pre = numerical_preflight_record(lib)
    print(pre)
    (HERE / "numerical_cases.json").write_text(json.dumps({"meta": meta, "cases": cases, "preflight": pre},
                                                          indent=1))


# The plugin's fixed-effect projection attachment
# (vckss_rust_engine_augment_projection_interrupt_v1 on a prepared generation,
# a generic-engine V5 solve, then projection_result_v1): covariates are seeded
# functions of the retained rows (a normal draw per input row, the row's
# period index, a product of the two), restricted to the retained rows in
# input order.  Each case names the panel, deletion mode, effect (1 worker,
# 2 firm), weight (1 frequency, 2 target), covariates and centering.
PROJECTION_CASES = {
    "controls_2k_worker": dict(panel="controls_2k", deletion=1, effect=1, weight=1, covariates=2, centering=0,
                               probes=16),
    "controls_2k_firm_mean": dict(panel="controls_2k", deletion=1, effect=2, weight=1, covariates=3, centering=1,
                                  probes=16),
    "controls_weighted_1500_target": dict(panel="controls_weighted_1500", deletion=1, effect=1, weight=2,
                                          covariates=1, centering=0, probes=12),
    "obs_2k_worker": dict(panel="obs_2k", deletion=2, effect=1, weight=1, covariates=2, centering=0, probes=16),
    "obs_controls_2k_firm": dict(panel="obs_controls_2k", deletion=2, effect=2, weight=2, covariates=2,
                                 centering=1, probes=16),
    "obs_controls_duplicates_worker": dict(panel="obs_controls_duplicates_1500", deletion=2, effect=1, weight=1,
                                           covariates=3, centering=0, probes=12),
}

PROJECTION_RESULT_FIELDS = ("columns", "effect", "weight", "gram_rcond", "gram_relres", "gram_original_relres",
                            "covariance_smallest_eigenvalue", "covariance_largest_eigenvalue", "psd_cleanup",
                            "proxy_minimum", "proxy_maximum", "maximum_iterations", "full_residual_tolerance",
                            "persistent_bytes", "result_bytes")
PROJECTION_AUGMENTATION_FIELDS = ("rows", "columns", "effect", "weight", "caller_copy_bytes",
                                  "projection_persistent_bytes", "gram_rcond", "gram_relres", "gram_original_relres")


def projection_panel(name: str) -> Panel:
    specs = {**CONTROL_PANELS, **OBSERVATION_PANELS}
    return specs[name]["build"]()


def projection_covariates(panel: Panel, mask: np.ndarray, count: int, seed: int) -> list:
    """Seeded covariates for the retained rows (input order)."""
    rng = np.random.default_rng(seed)
    z = rng.standard_normal(panel.rows)
    period = (np.arange(panel.rows) % 5).astype(np.float64)
    full = [z, period, z * period + 0.5 * z * z][:count]
    keep = mask.astype(bool)
    return [np.ascontiguousarray(c[keep]) for c in full]


def projection_request(e, probes: int, deletion: int, controls: int):
    """V5 generic-engine request: diagonal PCG at 1e-12, the given probes."""
    q = e.default_request_v5(deletion)
    v1 = q.v4.v3.v2.v1
    v1.probes = probes
    v1.solver_route = 2
    v1.pcg_tolerance = 1e-12
    v1.maximum_iterations = 20000
    q.v4.v3.v2.algorithm = 2
    q.threads = 4
    q.tolerance_supplied = 1
    return q


def projection_record(lib, spec: dict) -> dict:
    panel = projection_panel(spec["panel"])
    e = abi.Engine(lib)
    e.prepare(panel, deletion_mode=spec["deletion"])
    mask = e.retained_mask(panel.rows)
    cov = projection_covariates(panel, mask, spec["covariates"], 20261204)
    if spec["centering"]:
        e.centering(spec["centering"])
    e.augment_projection(cov, spec["effect"], spec["weight"])
    aug = e.projection_augmentation_receipt()
    e.solve_v5(projection_request(e, spec["probes"], spec["deletion"], len(panel.controls)),
               controls_count=len(panel.controls))
    res = e.projection_result()
    point = e.result()
    e.release()
    return {"panel_sha256": panel_digest(panel), "pcg_tolerance": 1e-12, **spec,
            "augmentation": {k: aug[k] for k in PROJECTION_AUGMENTATION_FIELDS},
            "coefficients": res["coefficients"], "covariance": res["covariance"],
            "naive_covariance": res["naive_covariance"],
            "receipt": {k: res["receipt"][k] for k in PROJECTION_RESULT_FIELDS},
            "corrected": list(point["corrected"])}


def projection_error_record(lib) -> dict:
    """Status codes of refused projection calls, each on a fresh generation,
    and the status of a valid augmentation after a refused one."""
    out = {}
    panel = projection_panel("controls_2k")

    def fresh():
        e = abi.Engine(lib)
        e.prepare(panel)
        mask = e.retained_mask(panel.rows)
        return e, projection_covariates(panel, mask, 2, 20261204), int(mask.sum())

    def status(fn) -> int:
        try:
            fn()
            return 0
        except abi.EngineError as err:
            return err.code

    e, cov, rows = fresh()
    e.release()
    cases = {"constant_covariate": ([np.ones(rows)], 1, 1, 1e-10),
             "rank_tolerance_high": (cov, 1, 1, 0.5),
             "rank_tolerance_low": (cov, 1, 1, 1e-16),
             "effect_unknown": (cov, 3, 1, 1e-10),
             "weight_unknown": (cov, 1, 3, 1e-10),
             "rows_short": ([c[:-1] for c in cov], 1, 1, 1e-10)}
    for name, args in cases.items():
        e, cov, rows = fresh()
        out[name] = status(lambda: e.augment_projection(*args))
        out[name + "_then_valid"] = status(lambda: e.augment_projection(cov))
        e.release()
    e, cov, rows = fresh()
    e.augment_projection(cov)
    out["second_projection"] = status(lambda: e.augment_projection(cov))
    e.release()
    e, cov, rows = fresh()
    e.augment_projection(cov)
    e.solve_v5(projection_request(e, 8, 1, len(panel.controls)), controls_count=len(panel.controls))
    out["augmentation_receipt_after_solve"] = status(lambda: e.projection_augmentation_receipt())
    e.release()
    e, cov, rows = fresh()
    e.solve_v5(projection_request(e, 8, 1, len(panel.controls)), controls_count=len(panel.controls))
    out["result_without_projection"] = status(lambda: e.projection_result())
    e.release()
    # a match panel without controls runs the compressed engine: refused
    plain = PANELS["small_2k"]["build"]()
    e = abi.Engine(lib)
    e.prepare(plain, use_v4=True)
    e.augment_projection(projection_covariates(plain, e.retained_mask(plain.rows), 1, 7))
    out["compressed_engine_solve"] = status(
        lambda: e.solve_v5(projection_request(e, 8, 1, 0), controls_count=0))
    e.release()
    return out


def write_projection_cases(lib, meta: dict) -> None:
    cases = {}
    for name, spec in PROJECTION_CASES.items():
        cases[name] = projection_record(lib, spec)
        print(name, cases[name]["coefficients"], cases[name]["receipt"]["psd_cleanup"])
    errors = projection_error_record(lib)
    print(errors)
    (HERE / "projection_cases.json").write_text(json.dumps({"meta": meta, "cases": cases, "errors": errors},
                                                           indent=1))


# The plugin's generic engine under the fixed-offset nuisance (nuisance_mode
# 2: the joint fit's control coefficients held fixed, the estimator on the
# worker-firm model of y - Q'beta): point solves through V5 at 1e-12 on the
# diagonal route, the numerical attachment, and a projection.
FIXED_OFFSET_CASES = {
    "controls_2k": dict(panel="controls_2k", deletion=1, centering=0, probes=16),
    "controls_2k_mean": dict(panel="controls_2k", deletion=1, centering=1, probes=16),
    "controls_weighted_1500": dict(panel="controls_weighted_1500", deletion=1, centering=0, probes=12),
    "controls_6p_4k": dict(panel="controls_6p_4k", deletion=1, centering=0, probes=12),
    "obs_controls_2k": dict(panel="obs_controls_2k", deletion=2, centering=0, probes=16),
    "obs_controls_2k_mean": dict(panel="obs_controls_2k", deletion=2, centering=1, probes=16),
    "obs_controls_duplicates_1500": dict(panel="obs_controls_duplicates_1500", deletion=2, centering=0, probes=12),
}


def fixed_offset_record(lib, spec: dict) -> dict:
    panel = projection_panel(spec["panel"])
    q_count = len(panel.controls)
    out = {"panel_sha256": panel_digest(panel), "pcg_tolerance": 1e-12, **spec}
    e = abi.Engine(lib)
    e.prepare(panel, deletion_mode=spec["deletion"])
    if spec["centering"]:
        e.centering(spec["centering"])
    q = projection_request(e, spec["probes"], spec["deletion"], q_count)
    q.v4.v3.v2.nuisance_mode = 2
    e.solve_v5(q, controls_count=q_count)
    out.update({k: list(v) for k, v in e.result().items()})
    e.release()
    # the numerical attachment under the same nuisance
    e = abi.Engine(lib)
    e.prepare(panel, deletion_mode=spec["deletion"])
    if spec["centering"]:
        e.centering(spec["centering"])
    req = numerical_request(e, spec["probes"], 2, spec["deletion"], q_count)
    req.point.v3.v2.nuisance_mode = 2
    req.point.v3.request_signature = abi.capability_signature_v3(req.point, q_count)
    e.solve_numerical(req)
    r = e.numerical_result()
    e.release()
    out["numerical"] = {k: r[k] for k in ("status", "engine", "mcse", "raw", "usable", "psd_adjustment",
                                          "minimum_constrained", "minimum_residual_margin",
                                          "maximum_sensitivity_ratio")}
    # a projection on the worker effect (two covariates)
    e = abi.Engine(lib)
    e.prepare(panel, deletion_mode=spec["deletion"])
    if spec["centering"]:
        e.centering(spec["centering"])
    e.augment_projection(projection_covariates(panel, e.retained_mask(panel.rows), 2, 20261204))
    q = projection_request(e, spec["probes"], spec["deletion"], q_count)
    q.v4.v3.v2.nuisance_mode = 2
    e.solve_v5(q, controls_count=q_count)
    res = e.projection_result()
    e.release()
    out["projection"] = {"coefficients": res["coefficients"], "covariance": res["covariance"],
                         "naive_covariance": res["naive_covariance"],
                         "proxy": [res["receipt"]["proxy_minimum"], res["receipt"]["proxy_maximum"]]}
    return out


def write_fixed_offset_cases(lib, meta: dict) -> None:
    cases = {}
    for name, spec in FIXED_OFFSET_CASES.items():
        cases[name] = fixed_offset_record(lib, spec)
        print(name, cases[name]["corrected"], cases[name]["numerical"]["status"])
    (HERE / "fixed_offset_cases.json").write_text(json.dumps({"meta": meta, "cases": cases}, indent=1))


def main() -> None:
    """All fixtures; with the argument ``cmg`` only cmg_cases.json, with
    ``receipts`` only receipt_cases.json, with ``sized`` only sized_cases.json, with
    ``exact`` only exact_cases.json, with ``numerical`` only numerical_cases.json, with
    ``projection`` only projection_cases.json, with ``fixed_offset`` only
    fixed_offset_cases.json."""
    if not PLUGIN.exists():
        raise SystemExit(f"reference plugin not found at {PLUGIN}")
    lib = abi.load(PLUGIN, bind_extensions=False)
    if sys.argv[1:] == ["cmg"]:
        write_cmg_cases(lib, {"generator": "tests/golden/make_golden.py cmg", "reference_plugin_version":
                              lib.vckss_rust_backend_version().decode()})
        return
    if sys.argv[1:] == ["exact"]:
        write_exact_cases(lib, {"generator": "tests/golden/make_golden.py exact", "reference_plugin_version":
                                lib.vckss_rust_backend_version().decode()})
        return
    if sys.argv[1:] == ["numerical"]:
        write_numerical_cases(lib, {"generator": "tests/golden/make_golden.py numerical",
                                    "reference_plugin_version": lib.vckss_rust_backend_version().decode()})
        return
    if sys.argv[1:] == ["fixed_offset"]:
        write_fixed_offset_cases(lib, {"generator": "tests/golden/make_golden.py fixed_offset",
                                       "reference_plugin_version": lib.vckss_rust_backend_version().decode()})
        return
    if sys.argv[1:] == ["projection"]:
        write_projection_cases(lib, {"generator": "tests/golden/make_golden.py projection",
                                     "reference_plugin_version": lib.vckss_rust_backend_version().decode()})
        return
    if sys.argv[1:] == ["sized"]:
        write_sized_cases(lib, {"generator": "tests/golden/make_golden.py sized", "reference_plugin_version":
                                lib.vckss_rust_backend_version().decode()})
        return
    if sys.argv[1:] == ["receipts"]:
        write_receipt_cases(lib, {"generator": "tests/golden/make_golden.py receipts",
                                  "reference_plugin_version": lib.vckss_rust_backend_version().decode()})
        return
    prep, jla = {}, {}
    for name, spec in PANELS.items():
        panel = spec["build"]()
        rec = prepare_record(lib, panel)
        rec["rows"] = panel.rows
        rec["panel_sha256"] = panel_digest(panel)
        prep[name] = rec
        jla[name] = [solve_record(lib, panel, spec["probes"], 0), solve_record(lib, panel, spec["probes"], 1)]
        print(name, rec["retained"], jla[name][0]["corrected"])
    controls = {}
    for name, spec in CONTROL_PANELS.items():
        panel = spec["build"]()
        rec = prepare_record(lib, panel)
        rec["rows"] = panel.rows
        rec["panel_sha256"] = panel_digest(panel)
        prep[name] = rec
        controls[name] = [solve_record_v5(lib, panel, spec["probes"], 0), solve_record_v5(lib, panel, spec["probes"], 1)]
        print(name, rec["retained"], controls[name][0]["corrected"])
    observation = {}
    for name, spec in OBSERVATION_PANELS.items():
        panel = spec["build"]()
        rec = prepare_record(lib, panel, 2)
        rec["rows"] = panel.rows
        rec["panel_sha256"] = panel_digest(panel)
        rec["deletion_mode"] = 2
        prep[name] = rec
        observation[name] = [solve_record_v5(lib, panel, spec["probes"], 0, 2),
                             solve_record_v5(lib, panel, spec["probes"], 1, 2)]
        print(name, rec["retained"], observation[name][0]["corrected"])
    write_cmg_cases(lib, meta)
    errs = {}
    for name, panel in error_cases().items():
        rec = prepare_record(lib, panel)
        rec["columns"] = {f: [float(x) if np.isfinite(x) else str(x) for x in getattr(panel, f)]
                          for f in ("worker", "firm", "deletion", "outcome", "frequency", "target_weight")}
        errs[name] = rec
        print(name, rec["status"])
    meta = {"generator": "tests/golden/make_golden.py", "reference_plugin_version":
            lib.vckss_rust_backend_version().decode()}
    (HERE / "prep_cases.json").write_text(json.dumps({"meta": meta, "panels": prep, "errors": errs}, indent=1))
    (HERE / "jla_cases.json").write_text(json.dumps({"meta": meta, "panels": jla, "controls": controls,
                                                        "observation": observation}, indent=1))



if __name__ == "__main__":
    main()
