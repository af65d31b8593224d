"""Probe-sharded decomposition across devices, one process per device.

Counter-V1 probes are schedule-invariant, so a decomposition splits by
probes: every rank prepares the same panel and solves a contiguous range of
the probes (ranges start on multiples of four, one Philox block).  The one
exchange of the leverage phase is an all-reduce (sum) of the leverage
accumulators; the target phase ends with a gather of every probe's four
draws.  The result equals the single-device decomposition of the same
request.

The compute side is a backend: ``DeviceBackend`` drives the library's shard
entry points on the rank's GPU; the tests drive the same protocol with the
oracle on CPU ranks (gloo).
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi

dptr = C.POINTER(C.c_double)


def probe_ranges(probes: int, world: int) -> list[tuple[int, int]]:
    """Contiguous probe ranges, each starting on a multiple of four."""
    blocks = (probes + 3) // 4
    per = -(-blocks // world)
    out = []
    for r in range(world):
        b, e = min(4 * per * r, probes), min(4 * per * (r + 1), probes)
        out.append((b, e))
    return out


def finish_components(plugin: np.ndarray, draws: np.ndarray) -> dict:
    """Correction (mean of the draws), corrected components and MCSE."""
    P = draws.shape[0]
    corr = draws.mean(axis=0)
    mcse = np.sqrt(((draws - corr) ** 2).sum(axis=0) / (P * (P - 1.0)))
    return {"plugin": tuple(plugin), "correction": tuple(corr), "corrected": tuple(plugin - corr),
            "numerical_mcse": tuple(mcse)}


def solve_sharded(backend, probes: int, rank: int, world: int, allreduce_sum, allgather) -> dict:
    """Run the sharded protocol; allreduce_sum(np.ndarray) -> np.ndarray and
    allgather(np.ndarray) -> list of every rank's array (rank order)."""
    b, e = probe_ranges(probes, world)[rank]
    acc = backend.leverage(b, e) if e > b else backend.zeros()
    acc = allreduce_sum(acc)
    draws = backend.target(b, e, acc) if e > b else np.zeros((0, 4))
    all_draws = np.concatenate(allgather(draws), axis=0)
    if all_draws.shape != (probes, 4):
        raise RuntimeError("gathered draws do not cover the probes")
    return backend.finish(all_draws)


class DeviceBackend:
    """The rank's GPU through the library's shard entry points.  With a torch
    CUDA ``device`` the leverage accumulators live in a device tensor that the
    library fills and reads directly, so the all-reduce runs on the device
    with no host round trip; otherwise they are numpy arrays."""

    def __init__(self, engine: abi.Engine, request, controls: int = 0, device=None):
        self.e, self.req, self.device = engine, request, device
        self.req.v4.v3.request_signature = abi.capability_signature_v3(request.v4, controls)
        n = C.c_uint64(0)
        engine.check(engine.lib.fevcb_engine_shard_size_v1(engine.generation, C.byref(n)))
        self.count = int(n.value)

    def accumulators(self) -> int:
        return self.count

    def zeros(self):
        if self.device is None:
            return np.zeros(self.count)
        import torch

        return torch.zeros(self.count, dtype=torch.float64, device=self.device)

    def _ptr(self, acc):
        if self.device is None:
            return acc.ctypes.data_as(dptr)
        return C.cast(C.c_void_p(acc.data_ptr()), dptr)

    def leverage(self, b: int, e: int):
        acc = self.zeros()
        self.e.check(self.e.lib.fevcb_engine_shard_leverage_v1(self.e.generation, C.byref(self.req), b, e,
                                                              self._ptr(acc), self.count))
        return acc

    def target(self, b: int, e: int, acc) -> np.ndarray:
        if self.device is None:
            acc = np.ascontiguousarray(acc, dtype=np.float64)
        else:
            acc = acc.contiguous()
        draws = np.zeros((e - b, 4))
        self.e.check(self.e.lib.fevcb_engine_shard_target_v1(self.e.generation, C.byref(self.req), b, e,
                                                            self._ptr(acc), self.count,
                                                            draws.ctypes.data_as(dptr)))
        return draws

    def finish(self, draws: np.ndarray) -> dict:
        d = np.ascontiguousarray(draws, dtype=np.float64)
        self.e.check(self.e.lib.fevcb_engine_shard_finish_v1(self.e.generation, C.byref(self.req),
                                                            d.ctypes.data_as(dptr)))
        return self.e.result()


def torch_collectives(device=None):
    """(allreduce_sum, allgather) over the default torch.distributed group;
    tensors live on `device` (a CUDA device for NCCL, None for gloo on CPU)."""
    import torch
    import torch.distributed as dist

    def allreduce_sum(a):
        if isinstance(a, torch.Tensor):  # a device tensor: reduced in place
            dist.all_reduce(a, op=dist.ReduceOp.SUM)
            return a
        t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64))
        if device is not None:
            t = t.to(device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return t.cpu().numpy()

    def allgather(a: np.ndarray) -> list[np.ndarray]:
        world = dist.get_world_size()
        n = torch.tensor([a.shape[0]], dtype=torch.int64, device=device)
        sizes = [torch.zeros_like(n) for _ in range(world)]
        dist.all_gather(sizes, n)
        m = int(max(s.item() for s in sizes))
        pad = np.zeros((m, 4))
        pad[:a.shape[0]] = a
        t = torch.from_numpy(pad)
        if device is not None:
            t = t.to(device)
        out = [torch.zeros_like(t) for _ in range(world)]
        dist.all_gather(out, t)
        return [o.cpu().numpy()[:int(s.item())] for o, s in zip(out, sizes)]

    return allreduce_sum, allgather
