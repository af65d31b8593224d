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
    req = abi.SolveRequestV1()
    assert lib.vckss_rust_engine_default_solve_request_v1(C.byref(req), 8) == 20
    assert b"capacity" in lib.vckss_rust_engine_last_error()


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
