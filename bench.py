"""Benchmark: JLA probe solves/s (and time-to-decomposition) on a seeded panel.

A step is one complete leave-out decomposition of the prepared panel: the full
fit, P leverage probes and 2P target solves (1 + 3P right-hand sides), the
leverage adjustment, the target contraction and the four components.

* ``value``  device-resident throughput: the prepared problem is in HBM and a
  step re-runs the solve (``fevcb_engine_resolve_v1``); CUDA events on the
  library's stream bracket exactly K steps after W warm-up steps.
* ``e2e``    the same metric through the plugin C ABI a caller uses: each step
  is ``solve_v5`` + ``result_v1`` on a freshly prepared generation, so the
  host->device upload of the prepared problem and the device->host result read
  are inside the timed region (host preparation is outside it and reported
  separately as ``prepare_s``; prepare + solve is the time-to-decomposition).
* ``roofline``  the dominant kernel (blocked SpMM on the hybrid Laplacian)
  timed standalone with CUDA events, L2 flushed before each launch.
* ``cpu_baseline``  the reference's own CPU implementation (its shipped plugin,
  staged in oracle/_ref by oracle/build.py; else the C oracle) on a bounded
  sample of the same panel, all host cores.

* ``forms``  the other solver forms on the same panel, one device-resident
  step each: the plain GPU CMG-PCG form (FP64, one target probe per solve, a
  bounded probe sample), the blocked CMG-PCG, the learned flexible PCG (with
  the committed network parameters) and the mixed-precision solve;
  ``speedup_vs_plain_gpu_cmg_pcg`` is ``value`` over the plain form's rate.

``--impl reference`` times the reference plugin alone (rank 0) on the same
panel and metric and prints its own JSON line.
"""

from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = "plain_1m"
METRIC = "JLA probe solves/s & time-to-decomposition, learned+batched vs plain GPU PCG"
UNIT = "probe solves/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--probes", type=int, default=200)
    ap.add_argument("--tolerance", type=float, default=1e-8)
    ap.add_argument("--block", type=int, default=0)
    ap.add_argument("--precond", type=int, default=0)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-probes", type=int, default=24)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true")
    ap.add_argument("--sharded", action="store_true", help="use the probe-sharded path at any N (launch with torchrun)")
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


def build_panel(args):
    from fevc_b200.panel import named_panel

    panel = named_panel(args.workload, args.scale)
    return panel, len(panel.controls)


def deletion_mode(panel) -> int:
    """1 leave-match-out, 2 leave-observation-out (the learned_10m panel)."""
    return 2 if panel.info.get("deletion") == "observation" else 1


def v5_request(engine, probes, tolerance, *, reference=False, deletion=1):
    """A V5 solve request: JLA, the panel's deletion mode, supplied tolerance.
    With controls the generic engine runs; the reference additionally selects
    its production CMG_FULL_V2 route on all host cores."""
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
        q.full_cmg_v2 = 1
    return q


def reference_plugin_path():
    p = ROOT / "oracle" / "_ref" / "fevc_rust_linux_x64.plugin"
    return p if p.exists() else None


def time_reference(panel, probes, tolerance, steps, warmup):
    """The reference plugin's V5 full-CMG solve (CMG_FULL_V2) on all host cores."""
    from fevc_b200 import abi

    lib = abi.load(reference_plugin_path(), bind_extensions=False)
    threads = os.cpu_count() or 1
    times, prep_times, res = [], [], None
    for i in range(warmup + steps):
        e = abi.Engine(lib)
        t0 = time.perf_counter()
        e.prepare(panel, deletion_mode=deletion_mode(panel))
        t1 = time.perf_counter()
        q = v5_request(e, probes, tolerance, reference=True, deletion=deletion_mode(panel))
        e.solve_v5(q, controls_count=len(panel.controls))
        res = e.result()
        t2 = time.perf_counter()
        e.release()
        if i >= warmup:
            times.append(t2 - t1)
            prep_times.append(t1 - t0)
    rhs = 1 + 3 * probes
    return {"rhs_per_s": rhs / float(np.median(times)), "solve_s": float(np.median(times)),
            "prepare_s": float(np.median(prep_times)), "threads": threads, "components": res}


def cpu_baseline(panel, probes, tolerance):
    if reference_plugin_path() is not None:
        r = time_reference(panel, probes, tolerance, steps=1, warmup=0)
        return {"value": round(r["rhs_per_s"], 3), "unit": UNIT, "cores": r["threads"], "kind": "reference",
                "sample": f"reference plugin CMG_FULL_V2 solve of the same panel with {probes} probes "
                          f"({1 + 3 * probes} RHS) at tol {tolerance:g}; solve phase {r['solve_s']:.2f} s, "
                          f"prepare {r['prepare_s']:.2f} s"}
    return None


def time_form(lib, panel, controls, probes, tolerance, block, precond, precision, stream, barrier):
    """One device-resident step of a solver form: (ms, RHS/s, column iterations per RHS)."""
    import torch

    from fevc_b200 import abi

    e = abi.Engine(lib)
    e.prepare(panel, deletion_mode=deletion_mode(panel))
    e.device_options(block, precond, precision)
    e.solve_v5(v5_request(e, probes, tolerance, deletion=deletion_mode(panel)), controls_count=controls)
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
    return {"ms_per_step": round(ms, 3), "value": round(rhs / (ms / 1000.0), 3), "unit": UNIT, "probes": probes,
            "iterations_per_rhs": round(t["column_iterations"] / max(t["rhs_columns"], 1), 3),
            "fallbacks": t["fallbacks"], "corrected": [round(x, 10) for x in res["corrected"]]}


def time_forms(lib, panel, controls, args, stream, barrier):
    from fevc_b200 import abi, learned

    def guarded(fn):
        # a form that the estimator refuses on this panel (e.g. a leave-out
        # inverse that a small probe sample leaves nonpositive) is reported,
        # not fatal to the line
        try:
            return fn()
        except abi.EngineError as err:
            return {"error": str(err)}

    forms = {}
    plain_probes = min(args.probes, args.plain_probes)
    if deletion_mode(panel) == 2:
        # leave-observation-out inverts 1 - P_ii per row: a few probes leave
        # some estimates nonpositive, so the plain form's sample is larger
        plain_probes = min(args.probes, max(args.plain_probes, 200))
    forms["plain_gpu_cmg_pcg"] = {
        **guarded(lambda: time_form(lib, panel, controls, plain_probes, args.tolerance, 2, 2, 0, stream, barrier)),
        "form": "FP64 CMG-PCG, one target probe (two right-hand sides) per solve, "
                f"bounded sample of {plain_probes} probes"}
    params = learned.load_params()
    if params is not None:
        learned.install(lib, params)
        forms["learned_flexible_pcg"] = {
            **guarded(lambda: time_form(lib, panel, controls, args.probes, args.tolerance, 64, 3, 0, stream, barrier)),
            "form": "graph-network polynomial preconditioner in flexible PCG, blocks of 64 (learned_params.f32)"}
    forms["mixed_precision"] = {
        **guarded(lambda: time_form(lib, panel, controls, args.probes, args.tolerance, 64, 1, 1, stream, barrier)),
        "form": "single-precision inner PCG with double refinement, blocks of 64"}
    forms["cmg_blocked"] = {
        **guarded(lambda: time_form(lib, panel, controls, args.probes, args.tolerance, 64, 2, 0, stream, barrier)),
        "form": "FP64 CMG-PCG, blocks of 64"}
    return forms


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    panel, controls = build_panel(args)
    if reference_plugin_path() is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference plugin not staged (run oracle/build.py)"}))
        return
    probes = min(args.probes, args.cpu_probes)
    r = time_reference(panel, probes, args.tolerance, args.steps, args.warmup)
    line = {"metric": METRIC, "value": round(r["rhs_per_s"], 4), "unit": UNIT, "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1000 * r["solve_s"], 2), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, fevc_b200/panel.py)",
            "config": {"workload": f"{args.workload} panel, {probes}-probe sample", "probes": probes,
                       "tolerance": args.tolerance, "controls": controls},
            "prepare_s": round(r["prepare_s"], 3),
            "cpu_baseline": {"value": round(r["rhs_per_s"], 4), "unit": UNIT, "cores": r["threads"],
                             "kind": "reference", "sample": f"{probes} probes ({1 + 3 * probes} RHS) per step"},
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

    from fevc_b200 import abi

    lib = abi.load()
    stream = torch.cuda.Stream()  # the library launches on this stream; the events below record on it
    torch.cuda.set_stream(stream)
    lib.fevcb_set_stream(C.c_void_p(stream.cuda_stream))
    panel, controls = build_panel(args)

    e = abi.Engine(lib)
    t0 = time.perf_counter()
    e.prepare(panel, deletion_mode=deletion_mode(panel))
    prepare_s = time.perf_counter() - t0
    e.device_options(args.block, args.precond)
    # N ranks: every rank contributes `probes` probes to one decomposition of
    # probes x N (weak scaling); the leverage accumulators are all-reduced and
    # the target draws gathered over NCCL (fevc_b200/sharded.py)
    total_probes = args.probes * world
    req = v5_request(e, total_probes, args.tolerance, deletion=deletion_mode(panel))
    rhs = 1 + 3 * args.probes  # right-hand sides this rank solves per step
    collectives = None
    use_shards = world > 1 or args.sharded
    if use_shards:
        from fevc_b200 import sharded

        collectives = sharded.torch_collectives(torch.device("cuda", local))

        def step(engine):
            backend = sharded.DeviceBackend(engine, req, controls)
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

    # roofline: the persistent blocked PCG kernel, standalone launches with L2 flushed
    block = args.block or 64
    torch.cuda.nvtx.range_push("roofline")  # the roofline kernel's standalone launches
    spmm_ms, spmm_bytes = e.kernel_benchmark(1, block, 10)
    torch.cuda.nvtx.range_pop()
    # the same iterations in both persistent forms, for comparison
    three_ms, _ = e.kernel_benchmark(5, block, 10)
    two_ms, _ = e.kernel_benchmark(6, block, 10)
    two_barrier = block == 32  # the form the solver picks at this width (double, one warp per segment)
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    # DRAM traffic per launch of this kernel from the committed ncu capture
    # (profiles/roofline_traffic.json), when it covers this kernel and workload
    roof_kernel = f"k_pcg_persistent_cg<{block}, double>" if block == 32 else f"k_pcg_persistent<{block}, double>"
    traffic = None
    try:
        rec = json.loads((ROOT / "profiles" / "roofline_traffic.json").read_text()).get(roof_kernel)
        if rec and rec.get("workload") == args.workload and args.scale == 1.0:
            traffic = float(rec["bytes_per_launch"])
    except Exception:
        pass
    achieved = spmm_bytes / (spmm_ms / 1000.0) / 1e9
    h2d = int(timings["h2d_bytes"])
    e.release()

    # e2e through the C ABI: solve + result on a fresh generation per step
    e2e_times = []
    for i in range(max(args.e2e_steps, 1) + 1):
        g = abi.Engine(lib)
        g.prepare(panel, deletion_mode=deletion_mode(panel))
        g.device_options(args.block, args.precond)
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

    # the other solver forms on the same panel (device-resident, one timed step
    # each): the plain GPU CMG-PCG form on a bounded probe sample, the learned
    # flexible PCG and the mixed-precision solve
    forms = {}
    if not args.no_forms and world == 1:
        forms = time_forms(lib, panel, controls, args, stream, barrier)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(panel, min(args.probes, args.cpu_probes), args.tolerance)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_per_step, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator, fevc_b200/panel.py)",
            "config": {"workload": f"{args.workload} panel ({panel.info['workers']} workers, "
                                   f"{panel.info['firms']} firms, {panel.info['periods']} periods), "
                                   f"{total_probes} probes, {controls} year controls, "
                                   f"{'observation' if deletion_mode(panel) == 2 else 'match'} deletion",
                       "probes": total_probes, "rhs_per_step": rhs * world, "tolerance": args.tolerance,
                       "block_columns": block, "preconditioner": "jacobi" if args.precond == 1 else "auto",
                       "controls": controls,
                       "parallelism": (f"probe-sharded x{world}: {args.probes} probes per GPU, "
                                       f"{total_probes} in the decomposition; NCCL all-reduce of the "
                                       "leverage accumulators and gather of the draws") if use_shards
                       else "single GPU",
                       "l2": "working set per step larger than L2 (126 MB)",
                       "retained": {"workers": int(timings["vertices"]) and None}},
            "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": 144, "seconds_per_step": round(e2e_s, 4)},
            "time_to_decomposition_s": round(prepare_s + e2e_s, 3), "prepare_s": round(prepare_s, 3),
            "first_solve_s": round(first_solve_s, 3),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "kernel": (f"k_pcg_persistent_cg<{block}, double> (two grid barriers per iteration"
                                    if two_barrier else
                                    f"k_pcg_persistent<{block}, double> (three grid barriers per iteration")
                                   + ", 20 iterations per launch, L2 flushed before each)",
                         "bytes_per_launch": spmm_bytes,
                         "ms_per_launch": round(spmm_ms, 5), "peak_source": "measured (MEASURED_PEAKS.json)",
                         "three_barrier_ms_per_launch": round(three_ms, 5),
                         "two_barrier_ms_per_launch": round(two_ms, 5)},
            "gpu_launches": int(timings["kernel_launches"]) * args.steps,
            "solver": {k: timings[k] for k in ("block_iterations", "column_iterations", "rhs_columns",
                                               "vertices", "edges", "kept_workers", "levels")},
            "phase_ms": {k: round(timings[k], 3) for k in ("fit_ms", "leverage_ms", "target_ms", "total_ms")},
            "components": {k: [round(float(x), 10) for x in v] for k, v in result.items()},
            "clocks": clocks.summary(),
        }
        del line["config"]["retained"]
        if forms:
            line["forms"] = forms
            plain = forms["plain_gpu_cmg_pcg"].get("value")
            line["speedup_vs_plain_gpu_cmg_pcg"] = round(value / plain, 2) if plain else None
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
