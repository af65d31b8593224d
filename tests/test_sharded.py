"""Probe sharding across ranks: the protocol (leverage accumulators summed by
an all-reduce, target draws gathered) run by two gloo ranks on CPU with the
oracle as the compute backend, against the single-process result and the
reference plugin's golden components."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from fevc_b200 import sharded


def test_probe_ranges_cover_and_align():
    for probes in (2, 5, 24, 200, 201):
        for world in (1, 2, 3, 8):
            r = sharded.probe_ranges(probes, world)
            assert r[0][0] == 0 and r[-1][1] == probes
            assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
            assert all(b % 4 == 0 for b, e in r if e > b)


class OracleBackend:
    def __init__(self, oracle_mod, view, probes, centering, seed):
        self.o, self.view = oracle_mod, view
        self.kw = dict(seed=seed, probes=probes, centering=centering)
        self.plugin = None

    def accumulators(self):
        return int(self.view.units) * 5

    def zeros(self):
        return np.zeros(self.accumulators())

    def leverage(self, b, e):
        io = np.zeros(self.accumulators())
        return self.o.shard(self.view, phase=1, probe_begin=b, probe_end=e, io=io, **self.kw)["io"]

    def target(self, b, e, acc):
        out = self.o.shard(self.view, phase=2, probe_begin=b, probe_end=e, io=acc.copy(), **self.kw)
        self.plugin = out["plugin"]
        return out["draws"]

    def finish(self, draws):
        return sharded.finish_components(self.plugin, draws)


def _rank(rank, world, port, name, which, q):
    import sys
    from pathlib import Path

    root = Path(__file__).resolve().parents[1]
    sys.path[:0] = [str(root), str(root / "tests" / "golden")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    import make_golden
    from fevc_b200 import abi
    from oracle import oracle as oracle_mod

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import json

        golden = json.loads((root / "tests" / "golden" / "jla_cases.json").read_text())
        rec = golden["panels"][name][which]
        lib = abi.load()
        e = abi.Engine(lib)
        e.prepare(make_golden.PANELS[name]["build"]())
        view = oracle_mod.problem_view(lib, e.generation)
        backend = OracleBackend(oracle_mod, view, rec["probes"], rec["centering"], rec["seed"])
        ar, ag = sharded.torch_collectives(None)
        res = sharded.solve_sharded(backend, rec["probes"], rank, world, ar, ag)
        e.release()
        q.put((rank, {k: list(v) for k, v in res.items()}, rec))
    finally:
        dist.destroy_process_group()


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("name,which", [("small_2k", 0), ("weighted_1500", 1)])
def test_two_gloo_ranks_reproduce_the_reference(name, which, oracle_mod):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, name, which, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, res, rec in out:
        for key in ("plugin", "correction", "corrected", "numerical_mcse"):
            a, b = np.array(res[key]), np.array(rec[key])
            assert np.max(np.abs(a - b)) / np.max(np.abs(b)) < 1e-10, (rank, key, a, b)
