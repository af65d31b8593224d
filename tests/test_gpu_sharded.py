"""The library's shard entry points on one GPU: the ranges of a two-rank
split solved one after the other, accumulators summed and draws gathered on
the host, give the reference plugin's components (match, controls and
leave-observation-out)."""

import numpy as np
import pytest

from fevc_b200 import abi, sharded

import make_golden

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def request(e, rec, deletion=1):
    q = e.default_request_v5(deletion)
    v1 = q.v4.v3.v2.v1
    v1.seed = rec["seed"]
    v1.probes = rec["probes"]
    v1.pcg_tolerance = 1e-12
    v1.maximum_iterations = 20000
    q.v4.v3.v2.algorithm = 2
    q.v4.v3.engine = 2
    q.tolerance_supplied = 1
    return q


CASES = [("panels", "small_2k", make_golden.PANELS, 1), ("panels", "weighted_1500", make_golden.PANELS, 1),
         ("controls", "controls_2k", make_golden.CONTROL_PANELS, 1),
         ("observation", "obs_controls_duplicates_1500", make_golden.OBSERVATION_PANELS, 2)]


@pytest.mark.parametrize("section,name,panels,deletion", CASES)
@pytest.mark.parametrize("world", [2, 3])
def test_shards_reproduce_the_reference(lib, golden, section, name, panels, deletion, world):
    rec = golden["jla"][section][name][0]
    panel = panels[name]["build"]()
    e = abi.Engine(lib)
    e.prepare(panel, deletion_mode=deletion)
    be = sharded.DeviceBackend(e, request(e, rec, deletion), len(panel.controls))
    ranges = sharded.probe_ranges(rec["probes"], world)
    acc = sum(be.leverage(b, x) for b, x in ranges if x > b)
    draws = np.concatenate([be.target(b, x, acc) for b, x in ranges if x > b])
    res = be.finish(draws)
    e.release()
    for key in ("plugin", "correction", "corrected", "numerical_mcse"):
        assert rel(res[key], rec[key]) < 1e-8, (key, res[key], rec[key])


@pytest.mark.parametrize("section,name,panels,deletion", CASES[::3])
def test_device_accumulators_reproduce_the_reference(lib, golden, section, name, panels, deletion):
    """The accumulators in torch CUDA tensors: the library writes and reads
    them on the device (the path an NCCL all-reduce takes)."""
    import torch

    rec = golden["jla"][section][name][0]
    panel = panels[name]["build"]()
    e = abi.Engine(lib)
    e.prepare(panel, deletion_mode=deletion)
    be = sharded.DeviceBackend(e, request(e, rec, deletion), len(panel.controls), device=torch.device("cuda"))
    ranges = sharded.probe_ranges(rec["probes"], 2)
    accs = [be.leverage(b, x) for b, x in ranges if x > b]
    assert all(a.is_cuda for a in accs)
    acc = accs[0].clone()
    for a in accs[1:]:
        acc += a
    draws = np.concatenate([be.target(b, x, acc) for b, x in ranges if x > b])
    res = be.finish(draws)
    e.release()
    for key in ("plugin", "correction", "corrected", "numerical_mcse"):
        assert rel(res[key], rec[key]) < 1e-8, (key, res[key], rec[key])
