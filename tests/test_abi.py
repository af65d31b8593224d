"""The C-ABI library loads without a GPU, exports every entry point the header
declares, keeps the plugin's struct layouts and request defaults, and reports
typed errors for misuse (reference vckss-plugin tests/engine_ffi.rs pattern)."""

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from fevc_b200 import abi

ROOT = Path(__file__).resolve().parents[1]
PLUGIN = ROOT / "oracle" / "_ref" / "fevc_rust_linux_x64.plugin"


def declared_functions():
    text = (ROOT / "include" / "fevc_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b((?:vckss_rust|fevcb)_\w+)\s*\(", text)))


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 45
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(abi.SIGNATURES), set(names) ^ set(abi.SIGNATURES)


def test_identity(lib):
    assert lib.vckss_rust_abi_version() == 1
    assert b"fevc-b200" in lib.vckss_rust_backend_version()
    assert b"VCKSS-COUNTER-V1" in lib.vckss_rust_capabilities_json()


class PrepareRequestInterruptV1(abi.Struct):
    _fields_ = [("options", abi.PrepareRequestV2), ("interrupt_poll", abi.InterruptPoll),
                ("interrupt_context", C.c_void_p), ("checkpoint_interval", C.c_uint32), ("reserved", C.c_uint32)]


class SolveRequestInterruptV5(abi.Struct):
    _fields_ = [("options", abi.SolveRequestV5), ("interrupt_poll", abi.InterruptPoll),
                ("interrupt_context", C.c_void_p), ("checkpoint_interval", C.c_uint32), ("reserved", C.c_uint32)]


@pytest.mark.skipif(not PLUGIN.exists(), reason="reference plugin not staged")
@pytest.mark.parametrize("name,cls", [
    ("solve_request_v1", abi.SolveRequestV1), ("solve_request_v2", abi.SolveRequestV2),
    ("solve_request_v3", abi.SolveRequestV3), ("solve_request_v4", abi.SolveRequestV4),
    ("solve_request_v5", abi.SolveRequestV5), ("solve_request_interrupt_v1", abi.SolveRequestInterruptV1),
    ("solve_request_v8", abi.SolveRequestV8), ("solve_request_interrupt_v8", abi.SolveRequestInterruptV8),
    ("solve_request_interrupt_v5", SolveRequestInterruptV5), ("prepare_request_v3", abi.PrepareRequestV3),
    ("prepare_request_interrupt_v1", PrepareRequestInterruptV1),
    ("prepare_request_interrupt_v2", abi.PrepareRequestInterruptV2),
    ("prepare_request_interrupt_v3", abi.PrepareRequestInterruptV3)])
def test_default_requests_match_reference(lib, name, cls):
    ref = abi.load(PLUGIN, bind_extensions=False)
    a, b = cls(), cls()
    assert getattr(lib, f"vckss_rust_engine_default_{name}")(C.byref(a), C.sizeof(a)) == 0
    assert getattr(ref, f"vckss_rust_engine_default_{name}")(C.byref(b), C.sizeof(b)) == 0
    assert bytes(a) == bytes(b), (a.as_dict(), b.as_dict())


def test_output_capacity_checked(lib):
    """A short output capacity is an ABI mismatch (10), a null output an
    invalid input (20), as the plugin reports them."""
    req = abi.SolveRequestV1()
    ref = abi.load(PLUGIN, bind_extensions=False)
    for L in (lib, ref):
        assert L.vckss_rust_engine_default_solve_request_v1(C.byref(req), 8) == 10
        assert L.vckss_rust_engine_default_solve_request_v1(None, C.sizeof(req)) == 20
    assert b"capacity" in lib.vckss_rust_engine_last_error() or b"pointer" in lib.vckss_rust_engine_last_error()


def test_lifecycle_errors(lib):
    from make_golden import kat12

    e = abi.Engine(lib)
    lib.vckss_rust_engine_clear_abandoned_v1()
    gen = e.prepare(kat12(), cleanup=False)
    # a second prepare without cleanup is refused while a generation is active
    e2 = abi.Engine(lib)
    with pytest.raises(abi.EngineError) as err:
        e2.prepare(kat12(), cleanup=False)
    assert err.value.code == 81
    # stale generation
    r = abi.ResultV1()
    assert lib.vckss_rust_engine_result_v1(gen + 7, C.byref(r), C.sizeof(r)) == 80
    # result before solve
    assert lib.vckss_rust_engine_result_v1(gen, C.byref(r), C.sizeof(r)) == 80
    snap = abi.SnapshotV1()
    assert lib.vckss_rust_engine_snapshot_v1(C.byref(snap), C.sizeof(snap)) == 0
    assert snap.state == 1 and snap.generation == gen
    e.release()
    assert lib.vckss_rust_engine_release_v1(gen) == 0  # releasing a released generation is idempotent
    assert lib.vckss_rust_engine_snapshot_v1(C.byref(snap), C.sizeof(snap)) == 0
    assert snap.state == 0 and snap.last_released_generation == gen


def test_solve_request_validation(lib):
    from make_golden import kat12

    e = abi.Engine(lib)
    e.prepare(kat12())
    req = e.default_request()
    req.probes = 1
    with pytest.raises(abi.EngineError) as err:
        e.solve(req)
    assert err.value.code == 20
    e.release()


def test_solve_without_gpu_fails_loudly(lib):
    if lib.fevcb_device_count() > 0:
        pytest.skip("a GPU is visible")
    from make_golden import kat12

    e = abi.Engine(lib)
    e.prepare(kat12())
    req = e.default_request()
    req.probes = 5
    with pytest.raises(abi.EngineError) as err:
        e.solve(req)
    assert err.value.code == 11 and "GPU" in err.value.message
    e.release()


def test_interrupt_poll_breaks_preparation(lib):
    """A callback that asks to stop on its second poll ends preparation with
    USER_BREAK and no generation, as the reference plugin does."""
    from fevc_b200.panel import generate_panel

    p = generate_panel(3000, 150, 5, seed=1)  # 15,000 rows: several polls at interval 4096
    calls = []

    @abi.InterruptPoll
    def poll(ctx):
        calls.append(1)
        return 1 if len(calls) >= 2 else 0

    cols = [np.ascontiguousarray(x) for x in (p.worker, p.firm, p.deletion, p.outcome, p.frequency, p.target_weight)]
    c1 = abi.ColumnsV1(C.sizeof(abi.ColumnsV3), 0, p.rows, *[x.ctypes.data_as(abi.dptr) for x in cols])
    c3 = abi.ColumnsV3(abi.ColumnsV2(c1, None, 0, 0), None, 0, 0)
    v2 = abi.PrepareRequestV2(1, C.sizeof(abi.PrepareRequestInterruptV3), p.rows, 1, 0, 1 << 30, p.rows * 6 * 8)
    req = abi.PrepareRequestInterruptV3(abi.PrepareRequestV4(abi.PrepareRequestV3(v2, 1, 0, 0), 0, 0), poll, None,
                                        4096, 0)
    libs = [lib] + ([abi.load(PLUGIN, bind_extensions=False)] if PLUGIN.exists() else [])
    for target in libs:
        calls.clear()
        out = C.c_uint64(99)
        assert target.vckss_rust_engine_prepare_interrupt_v4(C.byref(req), C.byref(c3), C.byref(out), 8) == 1
        assert out.value == 0 and len(calls) == 2
        target.vckss_rust_engine_clear_abandoned_v1()


def test_short_struct_size_is_an_abi_mismatch(lib):
    from make_golden import kat12

    e = abi.Engine(lib)
    e.prepare(kat12())
    req = e.default_request()
    req.struct_size = 100
    with pytest.raises(abi.EngineError) as err:
        e.solve(req)
    assert err.value.code == 10 and "below required size 176" in err.value.message
    e.release()


def capability_requests():
    """A grid of V3 capability requests: the default solve request's fields
    and single-field variations across valid and invalid values."""
    base = dict(abi_version=1, request_schema=3, algorithm=2, deletion_mode=1, nuisance_mode=1, solver_route=0,
                rng_contract=1, controls_count=0, frequency_use=0, engine=0, batch_mode=0, stayers_mode=1,
                target_weight_mode=0, deletion_unit_source=1, probeorder_supplied=0, wallseconds_supplied=0,
                physical_limit=1 << 40, leverage_batch_mode=0, target_batch_mode=0,
                allow_automatic_cmg_setup_fallback=0, wallseconds=0.0)
    variations = dict(request_schema=[1, 2, 4], algorithm=[0, 1, 3], deletion_mode=[0, 2, 3], nuisance_mode=[0, 2, 3],
                      solver_route=[1, 2, 3, 4], rng_contract=[0, 2], controls_count=[4, 32, 33],
                      frequency_use=[1, 2], engine=[1, 2, 3], batch_mode=[1, 2, 3], stayers_mode=[0, 2, 3],
                      target_weight_mode=[1, 2], deletion_unit_source=[0, 2, 3, 4], probeorder_supplied=[1, 2],
                      wallseconds_supplied=[1, 2], physical_limit=[0, (1 << 53) + 1],
                      leverage_batch_mode=[1, 2], target_batch_mode=[1], allow_automatic_cmg_setup_fallback=[1, 2],
                      wallseconds=[5.0, -1.0])
    yield base
    for k, vals in variations.items():
        for v in vals:
            yield {**base, k: v}
    # combinations that reach the algorithm-specific branches
    for alg in (0, 1, 2):
        for route in (0, 1, 2, 3):
            for engine in (0, 1, 2):
                for deletion, source in ((1, 1), (2, 3)):
                    for rng in (0, 1):
                        for stayers in (1, 2):
                            yield {**base, "algorithm": alg, "solver_route": route, "engine": engine,
                                   "deletion_mode": deletion, "deletion_unit_source": source, "rng_contract": rng,
                                   "stayers_mode": stayers, "controls_count": 4 if engine == 1 else 0}


def make_capability_request(d):
    r = abi.CapabilityRequestV3()
    v1, v2 = r.v2.v1, r.v2
    v1.struct_size = C.sizeof(r)
    for k in ("abi_version", "request_schema", "algorithm", "deletion_mode", "nuisance_mode", "solver_route",
              "rng_contract", "controls_count", "frequency_use"):
        setattr(v1, k, d[k])
    for k in ("engine", "batch_mode", "stayers_mode", "target_weight_mode", "deletion_unit_source",
              "probeorder_supplied", "wallseconds_supplied", "physical_limit"):
        setattr(v2, k, d[k])
    for k in ("leverage_batch_mode", "target_batch_mode", "allow_automatic_cmg_setup_fallback", "wallseconds"):
        setattr(r, k, d[k])
    return r


@pytest.mark.skipif(not PLUGIN.exists(), reason="reference plugin not staged")
def test_request_capability_receipts_match_reference(lib):
    """Reason, profile, signature and every receipt byte equal the plugin's."""
    ref = abi.load(PLUGIN, bind_extensions=False)
    ref.vckss_rust_backend_request_capability_v3.restype = C.c_int32
    n = 0
    for d in capability_requests():
        req = make_capability_request(d)
        a, b = (C.c_uint8 * 160)(), (C.c_uint8 * 160)()
        sa = lib.vckss_rust_backend_request_capability_v3(C.byref(req), a, 160)
        sb = ref.vckss_rust_backend_request_capability_v3(C.byref(req), b, 160)
        assert sa == sb, d
        assert bytes(a) == bytes(b), d
        n += 1
    assert n > 100


@pytest.mark.skipif(not PLUGIN.exists(), reason="reference plugin not staged")
def test_v4_solve_refuses_an_unreconciled_request(lib):
    """A V4 solve whose signature does not match its capability receipt is
    refused (11) before any work, by both libraries; so is a profile of zero."""
    from make_golden import kat12

    for L in (lib, abi.load(PLUGIN, bind_extensions=False)):
        for mutate in ("signature", "profile"):
            e = abi.Engine(L)
            e.prepare(kat12())
            q = abi.SolveRequestV4()
            assert L.vckss_rust_engine_default_solve_request_v4(C.byref(q), C.sizeof(q)) == 0
            q.v3.v2.v1.probes = 4
            q.v3.v2.algorithm = 2
            q.v3.request_signature = abi.capability_signature_v3(q, 0)
            if mutate == "signature":
                q.v3.request_signature ^= 1
            else:
                q.v3.capability_profile = 0
            st = L.vckss_rust_engine_solve_v4(e.generation, C.byref(q))
            msg = L.vckss_rust_engine_last_error().decode()
            e.release()
            assert st == 11 and ("reconcile" in msg or "capability profile" in msg), (L, mutate, st, msg)


def test_entry_points_outside_the_solve_path(lib):
    """Every other reference entry point exists: schema probes report what is
    available (centering, the numerical attachment V1 and Mean-centred
    projection) and the rest return
    UNSUPPORTED_FEATURE naming the call."""
    assert lib.vckss_rust_centering_schema_v1() == 1
    assert lib.vckss_rust_numerical_schema_v1() == 1
    assert lib.vckss_rust_projection_centering_schema_v1() == 1
    for probe in ("numerical_schema_v2", "exact_execution_schema_v1",
                  "exact_legacy_execution_schema_v1", "exact_resolved_execution_schema_v2",
                  "component_inference_interface_version"):
        assert getattr(lib, "vckss_rust_" + probe)() == 0, probe
    called = 0
    for name, (res, args) in abi.UNSUPPORTED_SIGNATURES.items():
        if res is not abi.i32:
            continue
        zeros = [None if a is C.c_void_p else 0 for a in args]
        assert getattr(lib, name)(*zeros) == 11, name
        assert name[len("vckss_rust_"):].encode() in lib.vckss_rust_engine_last_error(), name
        assert lib.vckss_rust_session_last_error() == lib.vckss_rust_engine_last_error()
        called += 1
    assert called >= 70


def test_prepare_timings_split_the_preparation(lib):
    """The preparation's phase split: five non-negative phases that add up to
    the total, which the wall clock around the prepare call bounds."""
    import time

    from fevc_b200.panel import generate_panel

    e = abi.Engine(lib)
    panel = generate_panel(20_000, 1_000, 5, seed=5)
    t0 = time.perf_counter()
    e.prepare(panel)
    wall_ms = (time.perf_counter() - t0) * 1e3
    try:
        t = e.prepare_timings()
        phases = [t[k] for k in ("ingest_ms", "canonical_ms", "graph_ms", "compression_ms", "plan_ms")]
        assert all(p >= 0.0 for p in phases) and t["threads"] >= 1
        assert abs(sum(phases) - t["total_ms"]) < 1e-6 * max(1.0, t["total_ms"])
        assert 0.0 < t["total_ms"] <= wall_ms
        assert lib.fevcb_engine_prepare_timings_v1(e.generation, None, 0) == 20
    finally:
        e.release()


def test_setup_timings_need_a_device_engine(lib):
    """The device setup timings exist only once a solve has built the
    generation's device engine: before that the call is STALE_CONTEXT (80);
    a short output is an ABI mismatch (10)."""
    from make_golden import kat12

    e = abi.Engine(lib)
    e.prepare(kat12())
    try:
        t = abi.FevcbSetupTimingsV1()
        assert C.sizeof(t) == 176
        assert lib.fevcb_engine_setup_timings_v1(e.generation, C.byref(t), C.sizeof(t)) == 80
        assert lib.fevcb_engine_setup_timings_v1(e.generation, C.byref(t), 100) == 10
    finally:
        e.release()
