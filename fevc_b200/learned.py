"""Learned preconditioner: training orchestration and parameter files.

The network and its training run in the library (CUDA kernels, see
``csrc/learned.cu``); this module drives them through the C ABI: it prepares
seeded training panels, hands their hybrid Laplacians to a device trainer
(which generates residual/error pairs by CMG-PCG), trains, and reads or
installs the parameter vector that preconditioner 3 uses.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import abi
from .panel import generate_panel

PARAMS_FILE = Path(__file__).resolve().parent / "learned_params.f32"
fp = C.POINTER(C.c_float)


class LearnedDumpV1(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("pairs", C.c_uint32), ("vertices", C.c_uint64),
                ("row_ptr", C.POINTER(C.c_uint32)), ("col", C.POINTER(C.c_uint32)),
                ("weight", C.POINTER(C.c_double)), ("diagonal", C.POINTER(C.c_double)),
                ("features", fp), ("basis", fp), ("error", fp), ("energy", fp)]


assert C.sizeof(LearnedDumpV1) == 80


def _check(lib, st: int) -> None:
    if st != 0:
        raise abi.EngineError(st, lib.vckss_rust_engine_last_error().decode())


def param_count(lib) -> int:
    n = C.c_uint64(0)
    _check(lib, lib.fevcb_learned_param_count_v1(C.byref(n)))
    return int(n.value)


def initial_params(lib, seed: int = 1) -> np.ndarray:
    p = np.zeros(param_count(lib), dtype=np.float32)
    _check(lib, lib.fevcb_learned_initial_params_v1(seed, p.ctypes.data_as(fp), p.size))
    return p


def install(lib, params: np.ndarray) -> None:
    """Make `params` the network of preconditioner 3 for engines built next."""
    p = np.ascontiguousarray(params, dtype=np.float32)
    _check(lib, lib.fevcb_learned_install_v1(p.ctypes.data_as(fp), p.size))


def load_params(path: Path = PARAMS_FILE) -> np.ndarray | None:
    return np.fromfile(path, dtype=np.float32) if Path(path).exists() else None


def save_params(params: np.ndarray, path: Path = PARAMS_FILE) -> None:
    np.ascontiguousarray(params, dtype=np.float32).tofile(path)


class Trainer:
    """A device trainer holding training graphs and the network parameters."""

    def __init__(self, lib, seed: int = 1):
        self.lib = lib
        h = C.c_uint64(0)
        _check(lib, lib.fevcb_learned_trainer_create_v1(seed, C.byref(h)))
        self.handle = h.value
        self.graphs = 0
        self.count = param_count(lib)

    def close(self) -> None:
        if self.handle:
            _check(self.lib, self.lib.fevcb_learned_trainer_destroy_v1(self.handle))
            self.handle = 0

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add_panel(self, panel, columns: int = 16, seed: int = 7) -> None:
        e = abi.Engine(self.lib)
        e.prepare(panel)
        try:
            _check(self.lib, self.lib.fevcb_learned_trainer_add_panel_v1(self.handle, e.generation, columns, seed))
        finally:
            e.release()
        self.graphs += 1

    def train(self, steps: int, lr: float = 3e-3) -> np.ndarray:
        out = np.zeros(steps)
        _check(self.lib, self.lib.fevcb_learned_trainer_train_v1(self.handle, steps, lr,
                                                                 out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def gradient(self, graph: int = 0) -> tuple[float, np.ndarray]:
        g = np.zeros(self.count, dtype=np.float32)
        loss = C.c_double(0)
        _check(self.lib, self.lib.fevcb_learned_trainer_gradient_v1(self.handle, graph, C.byref(loss),
                                                                    g.ctypes.data_as(fp), g.size))
        return loss.value, g

    @property
    def params(self) -> np.ndarray:
        p = np.zeros(self.count, dtype=np.float32)
        _check(self.lib, self.lib.fevcb_learned_trainer_params_v1(self.handle, p.ctypes.data_as(fp), p.size))
        return p

    @params.setter
    def params(self, value: np.ndarray) -> None:
        p = np.ascontiguousarray(value, dtype=np.float32)
        _check(self.lib, self.lib.fevcb_learned_trainer_set_params_v1(self.handle, p.ctypes.data_as(fp), p.size))

    def dump(self, graph: int = 0) -> dict:
        d = LearnedDumpV1()
        _check(self.lib, self.lib.fevcb_learned_trainer_dump_v1(self.handle, graph, C.byref(d), C.sizeof(d)))
        n, P = int(d.vertices), int(d.pairs)
        ptr = np.ctypeslib.as_array(d.row_ptr, shape=(n + 1,)).copy()
        nnz = int(ptr[-1])
        return {
            "n": n, "pairs": P, "ptr": ptr,
            "col": np.ctypeslib.as_array(d.col, shape=(nnz,)).copy(),
            "val": np.ctypeslib.as_array(d.weight, shape=(nnz,)).copy(),
            "diag": np.ctypeslib.as_array(d.diagonal, shape=(n,)).copy(),
            "X": np.ctypeslib.as_array(d.features, shape=(n, 8)).copy(),
            "Y": np.ctypeslib.as_array(d.basis, shape=(1, n, P)).copy(),
            "E": np.ctypeslib.as_array(d.error, shape=(n, P)).copy(),
            "ELE": np.ctypeslib.as_array(d.energy, shape=(P,)).copy(),
        }


def training_panels(count: int, workers: int = 20_000, firms: int = 1_500, seed: int = 20261203):
    """Seeded smaller panels of the benchmark generator (Pareto 1.2-1.5 sizes,
    mobility 0.08-0.12, some two-region panels)."""
    rng = np.random.default_rng(seed)
    for i in range(count):
        yield generate_panel(workers, firms, 5, move_p=float(rng.uniform(0.08, 0.12)),
                             pareto_shape=float(rng.uniform(1.2, 1.5)),
                             regions=2 if i % 4 == 3 else 1, cross_p=0.01, seed=seed + 1 + i)


def train_default(lib, panels: int = 24, steps: int = 600, lr: float = 3e-3, columns: int = 16,
                  workers: int = 20_000, firms: int = 1_500) -> tuple[np.ndarray, np.ndarray]:
    """Train on `panels` seeded panels; returns (parameters, losses)."""
    with Trainer(lib, seed=1) as t:
        for i, panel in enumerate(training_panels(panels, workers, firms)):
            t.add_panel(panel, columns=columns, seed=100 + i)
        losses = t.train(steps, lr)
        return t.params, losses


def main() -> None:
    """Train on seeded panels on the GPU and write the parameter file."""
    import argparse

    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--panels", type=int, default=64)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--columns", type=int, default=16)
    ap.add_argument("--workers", type=int, default=20_000)
    ap.add_argument("--firms", type=int, default=1_500)
    ap.add_argument("--out", default=str(PARAMS_FILE))
    args = ap.parse_args()
    lib = abi.load()
    params, losses = train_default(lib, args.panels, args.steps, args.lr, args.columns, args.workers, args.firms)
    save_params(params, Path(args.out))
    k = max(1, len(losses) // 20)
    print({"panels": args.panels, "steps": args.steps, "first_loss": float(np.mean(losses[:k])),
           "last_loss": float(np.mean(losses[-k:])), "out": args.out})


if __name__ == "__main__":
    main()
