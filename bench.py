"""Benchmark: JLA probe solves/s and time-to-decomposition on a seeded panel.

Workload (default): the 10M-worker leave-observation-out panel
(10,000,000 workers, 1,000,000 firms, 5 periods, Pareto(1.2) firm sizes,
4 year controls, observation deletion; seeded generator fevc_b200/panel.py),
1000 probes (3001 right-hand sides), tolerance 1e-8.  A step is one complete
leave-out decomposition of the prepared panel: the full fit, P leverage probes
and 2P target solves, the leverage adjustment, the target contraction and the
four components.

* ``value``  device-resident throughput of the headline form: the prepared
  problem is in HBM and a step re-runs the solve (``fevcb_engine_resolve_v1``);
  CUDA events on the library's stream bracket exactly K steps after W warm-up
  steps.  The headline form is the learned degree-1 preconditioner stage
  (network weights from fevc_b200/learned_params.f32) inside the single-kernel
  blocked PCG with FP32 storage and FP64 reductions and residual replacement
  (blocks of 64 columns); without committed parameters, the same stage with
  uniform weights.
* ``e2e``    the same metric through the plugin C ABI a caller uses: each step
  is ``solve_v5`` + ``result_v1`` on a freshly prepared generation, so the
  host->device upload of the prepared problem and the device->host result read
  are inside the timed region (host preparation is outside it and reported as
  ``prepare_s``; prepare + solve is the time-to-decomposition).
* ``roofline``  the dominant kernel (the single-kernel blocked PCG of the
  headline form) timed standalone with CUDA events, L2 flushed before each
  launch; algorithmic bytes per launch from the library's formula.
* ``forms``  the other solver forms on the same panel, one device-resident
  step each: FP64 Jacobi blocked PCG, mixed-precision Jacobi, the degree-1
  stage with uniform weights (the method without the network) and the plain
  GPU CMG-PCG (FP64, one target probe per solve) on a bounded probe sample.
* ``parity``  the reference plugin and this engine on the same panel, seed and
  probes at a size the plugin finishes: the largest relative difference of
  each component group.
* ``cpu_baseline``  the reference's own CPU implementation (its shipped
  plugin, staged in oracle/_ref by oracle/build.py) on a bounded sample of the
  same workload, all host cores.

``--impl reference`` times the reference plugin alone (rank 0) on the same
workload, metric and config and prints its own JSON line.
"""

from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import platform
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = "learned_10m"
PROBES = 1000
METRIC = "JLA probe solves/s & time-to-decomposition, learned+batched vs plain GPU PCG"
UNIT = "probe solves/s"
PARITY_RTOL = 1e-6
# the 10M-worker panel is compared at this scale, where the plugin finishes a 32-probe solve
PARITY_C5_SCALE = 0.2
FALLBACK_HBM_GBS = 6650.0

# solver forms: (preconditioner, precision, block columns, description)
FORMS = {
    "autotuned": (3, 2, 64, "autotuned per generation: the fastest of FP64 Jacobi, FP32 Jacobi and the FP32 "
                            "learned degree-1 stage, timed on the first leverage block (fevcb_engine_tuning_v1)"),
    "learned_mixed": (3, 1, 64, "learned per-vertex degree-1 stage in the single-kernel PCG, FP32 storage with "
                                "FP64 reductions and residual replacement, blocks of 64"),
    "polynomial_mixed": (4, 1, 64, "degree-1 stage with uniform weights (the method without the network), "
                                   "FP32 storage with FP64 reductions and residual replacement, blocks of 64"),
    "jacobi_mixed": (1, 1, 64, "Jacobi, FP32 storage with FP64 reductions and residual replacement, blocks of 64"),
    "jacobi_fp64": (1, 0, 64, "Jacobi blocked PCG in FP64 (three grid barriers per iteration), blocks of 64"),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--probes", type=int, default=PROBES)
    ap.add_argument("--tolerance", type=float, default=1e-8)
    ap.add_argument("--form", default="auto", choices=["auto"] + list(FORMS))
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-probes", type=int, default=0, help="probe sample of the CPU legs (0: per workload)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true")
    ap.add_argument("--no-parity", action="store_true")
    ap.add_argument("--parity-probes", type=int, default=24)
    ap.add_argument("--sharded", action="store_true", help="use the probe-sharded path at any N (launch with torchrun)")
    ap.add_argument("--strong", action="store_true",
                    help="strong scaling: --probes is the whole decomposition's probe count, split over the ranks "
                         "(default: weak scaling, --probes per rank)")
    ap.add_argument("--plain-probes", type=int, default=8)
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._thread = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                parts = [p.strip() for p in out.stdout.strip().split(",")]
                if len(parts) == 7:
                    self.samples.append(parts)
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._thread.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def build_panel(workload, scale):
    from fevc_b200.panel import named_panel

    return named_panel(workload, scale)


def deletion_mode(panel) -> int:
    """1 leave-match-out, 2 leave-observation-out (the learned_10m panel)."""
    return 2 if panel.info.get("deletion") == "observation" else 1


def workload_config(args, panel):
    """The config dict of the JSON line; the same in both arms."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    total = args.probes if args.strong else args.probes * world
    return {"workload": f"{args.workload} panel ({panel.info['workers']} workers, {panel.info['firms']} firms, "
                        f"{panel.info['periods']} periods), {total} probes, {len(panel.controls)} year controls, "
                        f"{'observation' if deletion_mode(panel) == 2 else 'match'} deletion",
            "probes": total, "rhs_per_step": 1 + 3 * total, "tolerance": args.tolerance,
            "controls": len(panel.controls),
            "parallelism": (f"probe-sharded x{world}: {total / world:g} probes per GPU, {total} in the decomposition; "
                            "NCCL all-reduce of the leverage accumulators and gather of the draws")
            if world > 1 or args.sharded else "single GPU",
            "l2": "inputs larger than L2 (the prepared problem and the 64-column blocks exceed 126 MB)"}


def v5_request(engine, probes, tolerance, *, reference=False, deletion=1, route=None):
    """A V5 solve request: JLA, the panel's deletion mode, supplied tolerance.
    With controls the generic engine runs; the reference additionally selects
    its production CMG_FULL_V2 route (or `route`) on all host cores."""
    q = engine.default_request_v5(deletion)
    if deletion == 2:
        q.v4.v3.engine = 2  # leave-observation-out runs the generic engine
    v1 = q.v4.v3.v2.v1
    v1.probes = probes
    v1.pcg_tolerance = tolerance
    v1.maximum_iterations = 20000
    q.v4.v3.v2.algorithm = 2
    q.tolerance_supplied = 1
    if reference:
        q.threads = os.cpu_count() or 1
        if route == "diagonal":
            v1.solver_route = 2
        else:
            q.full_cmg_v2 = 1
    return q


def reference_plugin_path():
    p = ROOT / "oracle" / "_ref" / "fevc_rust_linux_x64.plugin"
    return p if p.exists() else None


def cpu_model() -> str:
    try:
        for line in subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout.splitlines():
            if line.startswith("Model name:"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return platform.processor() or "unknown"


def reference_solve(lib, panel, probes, tolerance, *, route=None):
    """One reference solve through its V5 C ABI on a fresh generation (the
    plugin solves a prepared generation once): its production route
    (CMG_FULL_V2) first, its diagonal PCG route when the production
    refinement refuses the panel.  Returns (route used, prepare seconds,
    solve_v5 + result_v1 seconds, result, refusal text)."""
    from fevc_b200 import abi

    refused = None
    for r in ([route] if route else ["cmg_full_v2", "diagonal"]):
        e = abi.Engine(lib)
        t0 = time.perf_counter()
        e.prepare(panel, deletion_mode=deletion_mode(panel))
        prep = time.perf_counter() - t0
        q = v5_request(e, probes, tolerance, reference=True, deletion=deletion_mode(panel), route=r)
        t0 = time.perf_counter()
        try:
            e.solve_v5(q, controls_count=len(panel.controls))
            res = e.result()
        except abi.EngineError as err:
            refused = f"{r}: {err}"
            e.release()
            continue
        solve = time.perf_counter() - t0
        e.release()
        return r, prep, solve, res, refused
    raise RuntimeError(f"the reference plugin refused the panel: {refused}")


# The CPU legs (cpu_baseline and --impl reference) on the 10M-worker
# leave-observation-out workload: the reference plugin prepares 50M rows on
# one thread (about 4 minutes) and its production route refuses the full
# panel's fit, so they time the same generator and request at 0.02 of the
# panel (200,000 workers, 20,000 firms, 1M rows), where its production route
# completes.  The per-RHS cost grows with the panel, so this overstates the
# reference's full-size rate.
CPU_SCALE = {"learned_10m": 0.02}


def cpu_panel(args, panel):
    scale = CPU_SCALE.get(args.workload)
    if scale is None or args.scale != 1.0:
        return panel, None
    return build_panel(args.workload, scale), scale


def cpu_probes(args) -> int:
    if args.cpu_probes:
        return args.cpu_probes
    # leave-observation-out inverts 1 - P_ii per row: a sample must be large
    # enough for every estimate to stay positive
    return 24 if args.workload != "learned_10m" else 32


def time_reference(panel, probes, tolerance, steps, warmup):
    """`warmup + steps` reference solves of a `probes`-probe sample, each on a
    freshly prepared generation (preparation not timed); the median of the
    timed solve_v5 + result_v1 walls."""
    from fevc_b200 import abi

    lib = abi.load(reference_plugin_path(), bind_extensions=False)
    threads = os.cpu_count() or 1
    route, prep, first, res, refused = reference_solve(lib, panel, probes, tolerance)
    times, preps = [], [prep]
    for i in range(warmup + steps):
        _, prep, solve, res, _ = reference_solve(lib, panel, probes, tolerance, route=route)
        preps.append(prep)
        if i >= warmup:
            times.append(solve)
    solve_s = float(np.median(times)) if times else first
    return {"rhs_per_s": (1 + 3 * probes) / solve_s, "solve_s": solve_s, "prepare_s": float(np.median(preps)),
            "threads": threads, "route": route, "refused": refused, "components": res, "timed": len(times)}


def reference_sample_text(r, probes, scale, panel):
    where = (f"the same generator and request at {scale:g} of the panel ({panel.info['workers']} workers, "
             f"{panel.info['firms']} firms, {panel.rows} rows; the full panel's single-threaded preparation "
             "takes about 4 minutes and its production route refuses the full panel's fit)") if scale else \
        "the same panel"
    return (f"reference plugin ({r['route']} route{'; ' + r['refused'] if r['refused'] else ''}) on {where}: "
            f"{probes} probes ({1 + 3 * probes} RHS) per solve at tol {{tol}}, each solve on a fresh generation "
            f"(preparation {r['prepare_s']:.1f} s, not in the rate); median of {r['timed']} solve_v5 + result_v1 "
            f"walls of {r['solve_s']:.2f} s")


def cpu_baseline(args, panel):
    """Warm median of 3 reference solves of a bounded probe sample (one
    discarded first solve), rank 0, all host cores."""
    if reference_plugin_path() is None:
        return None
    probes = min(args.probes, cpu_probes(args))
    cpanel, scale = cpu_panel(args, panel)
    r = time_reference(cpanel, probes, args.tolerance, steps=3, warmup=0)
    return {"value": round(r["rhs_per_s"], 4), "unit": UNIT, "cores": r["threads"], "kind": "reference",
            "cpu_model": cpu_model(),
            "sample": reference_sample_text(r, probes, scale, cpanel).replace("{tol}", f"{args.tolerance:g}")}


def time_form(lib, panel, probes, tolerance, block, precond, precision, stream, barrier, *, timed=True):
    """One device-resident step of a solver form: ms, RHS/s, iterations per RHS
    and the corrected components."""
    import torch

    from fevc_b200 import abi

    e = abi.Engine(lib)
    e.prepare(panel, deletion_mode=deletion_mode(panel))
    e.device_options(block, precond, precision)
    q = v5_request(e, probes, tolerance, deletion=deletion_mode(panel))
    t0 = time.perf_counter()
    e.solve_v5(q, controls_count=len(panel.controls))
    torch.cuda.synchronize()
    first = time.perf_counter() - t0
    ms = None
    if timed:
        barrier()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        e.resolve()
        stop.record(stream)
        barrier()
        ms = start.elapsed_time(stop)
    t = e.timings()
    res = e.result()
    e.release()
    rhs = 1 + 3 * probes
    ms = ms if ms is not None else first * 1000.0
    return {"ms_per_step": round(ms, 3), "value": round(rhs / (ms / 1000.0), 3), "unit": UNIT, "probes": probes,
            "iterations_per_rhs": round(t["column_iterations"] / max(t["rhs_columns"], 1), 3),
            "fallbacks": t["fallbacks"], "corrected": [round(x, 10) for x in res["corrected"]]}


def plain_form_rate(lib, panel, probes, tolerance):
    """The plain GPU CMG-PCG form (FP64, aggregation multigrid, one target
    probe per solve) on a bounded probe sample: RHS solved per second of
    solve wall.  A sample too small for the leave-out inverses to stay
    positive is refused after the fit and the leverage solves; the rate then
    counts those 1 + P solves."""
    import torch

    from fevc_b200 import abi

    e = abi.Engine(lib)
    e.prepare(panel, deletion_mode=deletion_mode(panel))
    e.device_options(2, 2, 0)
    q = v5_request(e, probes, tolerance, deletion=deletion_mode(panel))
    t0 = time.perf_counter()
    refused = None
    try:
        e.solve_v5(q, controls_count=len(panel.controls))
        rhs = 1 + 3 * probes
    except abi.EngineError as err:
        refused = str(err)
        rhs = 1 + probes
    torch.cuda.synchronize()
    s = time.perf_counter() - t0
    e.release()
    return {"value": round(rhs / s, 4), "unit": UNIT, "probes": probes, "rhs_solved": rhs,
            "seconds": round(s, 3), "refused_after_leverage": refused,
            "form": "FP64 CMG-PCG (device aggregation multigrid V-cycle), one target probe (two right-hand sides) "
                    f"per solve, bounded sample of {probes} probes (wall of solve_v5 including the hierarchy build)"}


def numerical_attachment(lib, panel, probes, tolerance):
    """The numerical MCSE attachment (``vckss_rust_engine_solve_numerical_v1``)
    on the same panel and request: wall of the point solve plus the leverage
    replay on a fresh generation (preparation outside), the replay's share,
    the attachment's status and MCSE beside the point estimate's."""
    import torch

    from fevc_b200 import abi, learned

    e = abi.Engine(lib)
    e.prepare(panel, deletion_mode=deletion_mode(panel))
    # the headline's form: autotuned precision, the learned stage (uniform weights without parameters)
    e.device_options(64, 3 if learned.load_params() is not None else 4, 2)
    q = v5_request(e, probes, tolerance, deletion=deletion_mode(panel))
    req = e.numerical_request(q, len(panel.controls))
    t0 = time.perf_counter()
    e.solve_numerical(req)
    torch.cuda.synchronize()
    s = time.perf_counter() - t0
    r = e.numerical_result()
    point = e.result()
    t = e.timings()
    e.release()
    return {"seconds": round(s, 3), "status": r["status"], "engine": r["engine"],
            "replay_rhs": r["certified_replay_rhs"], "mcse": [round(x, 12) for x in r["mcse"]],
            "point_mcse": [round(x, 12) for x in point["numerical_mcse"]],
            "maximum_replay_complete_residual": r["maximum_replay_complete_residual"],
            "phase_ms": {k: round(t[k], 1) for k in ("fit_ms", "leverage_ms", "target_ms", "total_ms")},
            "form": "numerical MCSE attachment (mcse(all)): point solve + replay of the leverage probes, through "
                    "the C ABI, wall of solve_numerical_v1 on a fresh generation"}


def projection_attachment(lib, panel, probes, tolerance):
    """The fixed-effect projection attachment on the same panel and request:
    the worker effect projected on three seeded covariates (a normal draw,
    the row's period index, their product) plus the constant, frequency
    weights, on a fresh generation.  Reports the host augmentation (loadings
    and Gram certificates), the solve's wall and the projection's share of it
    (its four model solves and the streamed covariance pass)."""
    import numpy as np
    import torch

    from fevc_b200 import abi, learned

    e = abi.Engine(lib)
    e.prepare(panel, deletion_mode=deletion_mode(panel))
    e.device_options(64, 3 if learned.load_params() is not None else 4, 2)
    keep = e.retained_mask(panel.rows).astype(bool)
    rng = np.random.default_rng(20261204)
    z = rng.standard_normal(panel.rows)
    period = (np.arange(panel.rows) % 5).astype(np.float64)
    cov = [np.ascontiguousarray(c[keep]) for c in (z, period, z * period)]
    t0 = time.perf_counter()
    e.augment_projection(cov)
    augment_s = time.perf_counter() - t0
    q = v5_request(e, probes, tolerance, deletion=deletion_mode(panel))
    t0 = time.perf_counter()
    e.solve_v5(q, controls_count=len(panel.controls))
    torch.cuda.synchronize()
    s = time.perf_counter() - t0
    t = e.timings()
    res = e.projection_result()
    e.release()
    r = res["receipt"]
    return {"augment_s": round(augment_s, 3), "solve_s": round(s, 3),
            "projection_ms": round(t["total_ms"] - t["fit_ms"] - t["leverage_ms"] - t["target_ms"], 1),
            "columns": r["columns"], "coefficients": [round(x, 9) for x in res["coefficients"]],
            "covariance_diagonal": [res["covariance"][i][i] for i in range(r["columns"])],
            "psd_cleanup": r["psd_cleanup"], "maximum_iterations": r["maximum_iterations"],
            "maximum_complete_residual": r["maximum_complete_residual"],
            "form": "projection attachment: worker effect on 3 covariates + constant, frequency weights; host "
                    "augmentation, then solve_v5 on a fresh generation (projection solves and covariance pass "
                    "after the target phase)"}


def time_forms(lib, panel, args, stream, barrier, headline):
    from fevc_b200 import abi, learned

    def guarded(fn):
        try:
            return fn()
        except abi.EngineError as err:
            return {"error": str(err)}

    forms = {}
    have_params = learned.load_params() is not None
    for name, (precond, precision, block, text) in FORMS.items():
        if name == headline or (precond == 3 and not have_params):
            continue
        forms[name] = {**guarded(lambda: time_form(lib, panel, args.probes, args.tolerance, block, precond, precision,
                                                   stream, barrier)), "form": text}
    forms["plain_gpu_cmg_pcg"] = guarded(lambda: plain_form_rate(lib, panel, min(args.probes, args.plain_probes),
                                                                 args.tolerance))
    forms["numerical_attachment"] = guarded(lambda: numerical_attachment(lib, panel, args.probes, args.tolerance))
    forms["projection_attachment"] = guarded(lambda: projection_attachment(lib, panel, args.probes, args.tolerance))
    return forms


def parity(lib, headline, tolerance, workload, scale, probes):
    """The reference plugin and this engine (headline form) on the same panel,
    seed and probes: the largest relative difference of each component group,
    relative to the group's largest component."""
    from fevc_b200 import abi

    panel = build_panel(workload, scale)
    ref_lib = abi.load(reference_plugin_path(), bind_extensions=False)
    try:
        route, _, solve_s, ref, refused = reference_solve(ref_lib, panel, probes, tolerance, route="cmg_full_v2")
    except RuntimeError as err:
        return {"workload": f"{workload} panel at scale {scale:g}", "probes": probes, "reference_refused": str(err)}
    precond, precision, block, _ = FORMS[headline]
    g = abi.Engine(lib)
    g.prepare(panel, deletion_mode=deletion_mode(panel))
    g.device_options(block, precond, precision)
    g.solve_v5(v5_request(g, probes, tolerance, deletion=deletion_mode(panel)), controls_count=len(panel.controls))
    ours = g.result()
    g.release()
    diffs = {}
    for group in ("plugin", "correction", "corrected", "numerical_mcse"):
        a, b = np.asarray(ours[group], dtype=float), np.asarray(ref[group], dtype=float)
        diffs[group] = float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
    return {"workload": f"{workload} panel at scale {scale:g} ({panel.info['workers']} workers, "
                        f"{panel.info['firms']} firms)", "probes": probes, "tolerance": tolerance,
            "reference_route": route, "reference_solve_s": round(solve_s, 2),
            "form": headline, "max_rel_diff": diffs, "rtol": PARITY_RTOL,
            "ok": all(v <= PARITY_RTOL for v in diffs.values()),
            "corrected": {"ours": [float(x) for x in ours["corrected"]], "reference": [float(x) for x in ref["corrected"]]}}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    panel = build_panel(args.workload, args.scale)
    if reference_plugin_path() is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference plugin not staged (run oracle/build.py)"}))
        return
    probes = min(args.probes, cpu_probes(args))
    cpanel, scale = cpu_panel(args, panel)
    r = time_reference(cpanel, probes, args.tolerance, args.steps, args.warmup)
    sample = reference_sample_text(r, probes, scale, cpanel).replace("{tol}", f"{args.tolerance:g}")
    line = {"metric": METRIC, "value": round(r["rhs_per_s"], 4), "unit": UNIT, "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1000 * r["solve_s"], 2), "higher_is_better": True, "scaling": "strong" if args.strong else "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, fevc_b200/panel.py)",
            "config": workload_config(args, panel),
            "prepare_s": round(r["prepare_s"], 3),
            "cpu_baseline": {"value": round(r["rhs_per_s"], 4), "unit": UNIT, "cores": r["threads"],
                             "kind": "reference", "cpu_model": cpu_model(), "sample": sample},
            "e2e": {"value": round(r["rhs_per_s"], 4), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1 or args.sharded:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    from fevc_b200 import abi, learned

    lib = abi.load()
    stream = torch.cuda.Stream()  # the library launches on this stream; the events below record on it
    torch.cuda.set_stream(stream)
    lib.fevcb_set_stream(C.c_void_p(stream.cuda_stream))
    panel = build_panel(args.workload, args.scale)
    controls = len(panel.controls)

    params = learned.load_params()
    headline = args.form
    if headline == "auto":
        headline = "autotuned"
    if params is not None:
        learned.install(lib, params)
    elif FORMS[headline][0] == 3 and headline != "autotuned":
        raise SystemExit("the learned form needs fevc_b200/learned_params.f32 (python -m fevc_b200.learned)")
    precond, precision, block, form_text = FORMS[headline]
    if headline == "autotuned" and params is None:
        precond = 4  # the degree-1 stage with uniform weights

    e = abi.Engine(lib)
    t0 = time.perf_counter()
    e.prepare(panel, deletion_mode=deletion_mode(panel))
    prepare_s = time.perf_counter() - t0
    prepare_phases = {k: round(v / 1e3, 3) if k.endswith("_ms") else v for k, v in e.prepare_timings().items()}
    e.device_options(block, precond, precision)
    # N ranks: every rank contributes `probes` probes to one decomposition of
    # probes x N (weak scaling); the leverage accumulators are all-reduced and
    # the target draws gathered over NCCL (fevc_b200/sharded.py)
    # (--strong: `probes` in all, split over the ranks)
    total_probes = args.probes if args.strong else args.probes * world
    req = v5_request(e, total_probes, args.tolerance, deletion=deletion_mode(panel))
    rhs = 1 + 3 * total_probes / world  # right-hand sides per rank per step (every rank solves the fit)
    use_shards = world > 1 or args.sharded
    if use_shards:
        from fevc_b200 import sharded

        collectives = sharded.torch_collectives(torch.device("cuda", local))

        def step(engine):
            backend = sharded.DeviceBackend(engine, req, controls, device=torch.device("cuda", local))
            return sharded.solve_sharded(backend, total_probes, rank, world, *collectives)
    else:
        def step(engine):
            engine.resolve()

    t0 = time.perf_counter()
    if use_shards:
        result = step(e)
    else:
        e.solve_v5(req, controls_count=controls)
        result = e.result()
    torch.cuda.synchronize()
    first_solve_s = time.perf_counter() - t0

    for _ in range(args.warmup):
        step(e)
    barrier()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        start.record(stream)
        torch.cuda.nvtx.range_push("timed")  # ncu --nvtx-include "timed/" selects these launches
        for _ in range(args.steps):
            step(e)
        torch.cuda.nvtx.range_pop()
        stop.record(stream)
        barrier()
    ms = start.elapsed_time(stop)
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_per_step = ms / args.steps
    timings = e.timings()
    value = world * rhs * args.steps / (ms / 1000.0)

    # roofline: the headline form's single-kernel PCG, standalone launches
    # with L2 flushed (mode 10: the polynomial stage, 9: Jacobi; both FP32
    # storage); the FP64 Jacobi kernel beside it for comparison
    eff_pre, eff_prec = precond, precision
    if precision == 2:
        t = e.tuning()
        c = t["candidates"][t["chosen"]] if t["chosen"] >= 0 else {"precision": 0, "preconditioner": 1}
        eff_pre, eff_prec = c["preconditioner"], c["precision"]
    roof_mode = 10 if (eff_prec == 1 and eff_pre in (3, 4)) else (9 if eff_prec == 1 else 1)
    torch.cuda.nvtx.range_push("roofline")  # the roofline kernel's standalone launches
    roof_ms, roof_bytes = e.kernel_benchmark(roof_mode, block, 10)
    torch.cuda.nvtx.range_pop()
    fp64_ms, fp64_bytes = e.kernel_benchmark(1, block, 10)
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        pass
    peak = float(peaks["hbm_gbs"]) if "hbm_gbs" in peaks else FALLBACK_HBM_GBS
    peak_source = "measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks else "fallback (6.65 TB/s)"
    roof_kernel = {10: f"k_pcg_flex<{block}, float, true>", 9: f"k_pcg_flex<{block}, float, false>",
                   1: f"k_pcg_persistent<{block}, double, 1, 1>"}[roof_mode]
    traffic = None
    traffic_note = None
    try:
        recs = json.loads((ROOT / "profiles" / "roofline_traffic.json").read_text()).get(roof_kernel) or []
        for rec in recs if isinstance(recs, list) else [recs]:
            if rec.get("workload") == args.workload and args.scale == rec.get("scale", 1.0):
                traffic = float(rec["bytes_per_launch"])
                traffic_note = rec.get("source")
    except Exception:
        pass
    achieved = roof_bytes / (roof_ms / 1000.0) / 1e9
    h2d = int(timings["h2d_bytes"])
    tuning = e.tuning() if precision == 2 else None
    e.release()

    # e2e through the C ABI: solve + result on a fresh generation per step
    e2e_times = []
    for i in range(max(args.e2e_steps, 1) + 1):
        g = abi.Engine(lib)
        g.prepare(panel, deletion_mode=deletion_mode(panel))
        g.device_options(block, precond, precision)
        barrier()
        t0 = time.perf_counter()
        if use_shards:
            step(g)
        else:
            g.solve_v5(req, controls_count=controls)
        g.result()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        g.release()
        if i > 0:
            e2e_times.append(t1 - t0)
    e2e_s = float(np.median(e2e_times))
    if dist is not None:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = world * rhs / e2e_s

    forms = {}
    if not args.no_forms and world == 1:
        forms = time_forms(lib, panel, args, stream, barrier, headline)

    parity_blocks = []
    if rank == 0 and world == 1 and not args.no_parity and reference_plugin_path() is not None:
        parity_blocks.append(parity(lib, headline, args.tolerance, "plain_1m", 1.0, args.parity_probes))
        if args.workload == "learned_10m" and args.scale == 1.0:
            parity_blocks.append(parity(lib, headline, args.tolerance, "learned_10m", PARITY_C5_SCALE, 32))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args, panel)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_per_step, 3), "higher_is_better": True,
            "scaling": "strong" if args.strong else "weak", "vs_baseline": None, "dtype": "f32 storage / f64 reductions" if eff_prec == 1 else "f64",
            "data": "synthetic (seeded generator, fevc_b200/panel.py)",
            "config": workload_config(args, panel),
            "form": {"name": headline, "description": form_text, "preconditioner": precond, "precision": precision,
                     "block_columns": block, "tuning": tuning},
            "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": 144, "seconds_per_step": round(e2e_s, 4)},
            "time_to_decomposition_s": round(prepare_s + e2e_s, 3), "prepare_s": round(prepare_s, 3),
            "prepare_phases_s": {k.replace("_ms", ""): v for k, v in prepare_phases.items()},
            "first_solve_s": round(first_solve_s, 3),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic, "traffic_source": traffic_note,
                         "kernel": roof_kernel + " (20 iterations per launch, L2 flushed before each)",
                         "bytes_per_launch": roof_bytes, "ms_per_launch": round(roof_ms, 5),
                         "peak_source": peak_source,
                         "fp64_jacobi_kernel": {"ms_per_launch": round(fp64_ms, 5),
                                                "achieved": round(fp64_bytes / (fp64_ms / 1000.0) / 1e9, 1)}},
            "gpu_launches": int(timings["kernel_launches"]) * args.steps,
            "solver": {k: timings[k] for k in ("block_iterations", "column_iterations", "rhs_columns",
                                               "vertices", "edges", "kept_workers", "levels", "fallbacks")},
            "phase_ms": {k: round(timings[k], 3) for k in ("fit_ms", "leverage_ms", "target_ms", "total_ms")},
            "components": {k: [round(float(x), 10) for x in v] for k, v in result.items()},
            "clocks": clocks.summary(),
        }
        if forms:
            line["forms"] = forms
            plain = forms.get("plain_gpu_cmg_pcg", {}).get("value")
            line["speedup_vs_plain_gpu_cmg_pcg"] = round(value / plain, 2) if plain else None
            f64 = forms.get("jacobi_fp64", {}).get("value")
            line["speedup_vs_fp64_jacobi"] = round(value / f64, 3) if f64 else None
        if parity_blocks:
            line["parity"] = parity_blocks
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
