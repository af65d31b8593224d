"""Seeded synthetic worker-firm panels.

The reference ships no generator with Pareto firm sizes, per-period mobility or
psi-rank sorting (its simulators are ``fevc/fevc__simulate_data.ado`` and
``fevc/benchmarks/five_way_scaling/generate_input.py``, fixed designs), so the
panels used by the tests and the benchmark come from this module.  The design:

* firm sizes ``s_f ~ Pareto(shape)`` with scale 1; every firm draw (initial
  assignment and move destination) is proportional to ``s_f``;
* worker effects ``alpha ~ N(0, 0.30^2)``, firm effects ``psi ~ N(0, 0.20^2)``;
* sorting: workers are ranked by a Gaussian-copula latent
  ``u = rho*z_alpha + sqrt(1-rho^2)*e`` and matched, rank for rank, to
  size-proportional initial firm draws ordered by ``psi``;
* each later period a worker moves with probability ``p`` to a
  size-proportional firm other than the current one (two-region panels keep
  the move inside the worker's region except with probability ``cross_p``);
* ``y = alpha + psi + eps (+ delta_t)``, ``eps ~ N(0, 0.25^2)``; year effects
  ``delta_t ~ N(0, 0.05^2)`` are added when year controls are requested, and
  the controls are the ``T-1`` year dummies (base year omitted);
* frequency 1, target weight 1, deletion identifier = the worker-firm match
  (or the row itself for leave-observation-out).

Identifiers are positive integers stored as binary64, which is the form the
plugin ABI takes (``VckssEngineColumnsV1``).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Panel:
    worker: np.ndarray
    firm: np.ndarray
    deletion: np.ndarray
    outcome: np.ndarray
    frequency: np.ndarray
    target_weight: np.ndarray
    controls: list = field(default_factory=list)
    info: dict = field(default_factory=dict)

    @property
    def rows(self) -> int:
        return int(self.worker.shape[0])


def _size_sampler(rng, sizes):
    cdf = np.cumsum(sizes)
    cdf /= cdf[-1]

    def draw(n):
        idx = np.searchsorted(cdf, rng.random(n), side="right")
        return np.minimum(idx, len(sizes) - 1)

    return draw


def generate_panel(
    workers: int,
    firms: int,
    periods: int,
    *,
    move_p: float = 0.10,
    pareto_shape: float = 1.5,
    rho: float = 0.2,
    sd_alpha: float = 0.30,
    sd_psi: float = 0.20,
    sd_eps: float = 0.25,
    year_controls: bool = False,
    sd_year: float = 0.05,
    deletion: str = "match",
    regions: int = 1,
    cross_p: float = 0.0,
    seed: int = 20261203,
) -> Panel:
    """Draw one panel of ``workers * periods`` rows (see the module docstring)."""
    if workers < 2 or firms < 2 or periods < 2:
        raise ValueError("panel needs at least two workers, firms and periods")
    if deletion not in ("match", "observation"):
        raise ValueError("deletion must be 'match' or 'observation'")
    rng = np.random.default_rng(seed)
    sizes = (1.0 - rng.random(firms)) ** (-1.0 / pareto_shape)
    psi = rng.normal(0.0, sd_psi, firms)
    alpha = rng.normal(0.0, sd_alpha, workers)

    if regions < 1 or firms % regions != 0:
        raise ValueError("firms must split evenly into regions")
    per_region = firms // regions
    region_of_worker = (np.arange(workers) % regions) if regions > 1 else np.zeros(workers, np.int64)

    # initial firm: size-proportional draws inside the worker's region, matched
    # rank-for-rank (psi order) to the copula latent of alpha
    z_alpha = alpha / sd_alpha
    latent = rho * z_alpha + np.sqrt(1.0 - rho * rho) * rng.standard_normal(workers)
    first = np.empty(workers, np.int64)
    samplers = []
    for region in range(regions):
        lo = region * per_region
        sampler = _size_sampler(rng, sizes[lo:lo + per_region])
        samplers.append((lo, sampler))
        members = np.flatnonzero(region_of_worker == region)
        draws = lo + sampler(members.size)
        draws = draws[np.argsort(psi[draws], kind="stable")]
        order = members[np.argsort(latent[members], kind="stable")]
        first[order] = draws
    global_sampler = _size_sampler(rng, sizes)

    firm_t = np.empty((workers, periods), np.int64)
    firm_t[:, 0] = first
    for t in range(1, periods):
        current = firm_t[:, t - 1].copy()
        moving = np.flatnonzero(rng.random(workers) < move_p)
        dest = np.empty(moving.size, np.int64)
        if regions > 1:
            crossing = rng.random(moving.size) < cross_p
        else:
            crossing = np.zeros(moving.size, bool)
        pending = np.arange(moving.size)
        while pending.size:
            w = moving[pending]
            cand = np.empty(pending.size, np.int64)
            cross = crossing[pending]
            if cross.any():
                cand[cross] = global_sampler(int(cross.sum()))
            for region in range(regions):
                sel = (~cross) & (region_of_worker[w] == region)
                if sel.any():
                    lo, sampler = samplers[region]
                    cand[sel] = lo + sampler(int(sel.sum()))
            dest[pending] = cand
            pending = pending[cand == current[w]]
        current[moving] = dest
        firm_t[:, t] = current

    year_effect = rng.normal(0.0, sd_year, periods) if year_controls else np.zeros(periods)
    worker_col = np.repeat(np.arange(workers, dtype=np.int64), periods)
    firm_col = firm_t.reshape(-1)
    period_col = np.tile(np.arange(periods, dtype=np.int64), workers)
    eps = rng.normal(0.0, sd_eps, worker_col.size)
    outcome = alpha[worker_col] + psi[firm_col] + eps + year_effect[period_col]

    rows = worker_col.size
    if deletion == "match":
        deletion_col = worker_col.astype(np.float64) * firms + firm_col + 1.0
    else:
        deletion_col = np.arange(1, rows + 1, dtype=np.float64)
    controls = []
    if year_controls:
        for t in range(1, periods):
            controls.append((period_col == t).astype(np.float64))

    realized = float(np.corrcoef(alpha[worker_col], psi[firm_col])[0, 1])
    return Panel(
        worker=(worker_col + 1).astype(np.float64),
        firm=(firm_col + 1).astype(np.float64),
        deletion=deletion_col,
        outcome=outcome.astype(np.float64),
        frequency=np.ones(rows, np.float64),
        target_weight=np.ones(rows, np.float64),
        controls=controls,
        info={
            "workers": workers,
            "firms": firms,
            "periods": periods,
            "move_p": move_p,
            "pareto_shape": pareto_shape,
            "rho_requested": rho,
            "rho_realized_rows": realized,
            "year_controls": year_controls,
            "deletion": deletion,
            "regions": regions,
            "cross_p": cross_p,
            "seed": seed,
        },
    )


# Named panels.  "cfg" numbers follow the order in which the workloads are
# described in the benchmark documentation: exact-leverage check, plain GPU
# form, batching, mixed precision, learned preconditioner.
PANELS = {
    "exact_20k": dict(workers=20_000, firms=1_000, periods=5, move_p=0.10, pareto_shape=1.5),
    "plain_1m": dict(workers=1_000_000, firms=50_000, periods=5, move_p=0.10, pareto_shape=1.5,
                     year_controls=True),
    "batched_3m": dict(workers=3_000_000, firms=150_000, periods=6, move_p=0.08, pareto_shape=1.3),
    "mixed_5m": dict(workers=5_000_000, firms=250_000, periods=6, move_p=0.10, pareto_shape=1.5,
                     regions=2, cross_p=0.001),
    "learned_10m": dict(workers=10_000_000, firms=1_000_000, periods=5, move_p=0.10,
                        pareto_shape=1.2, year_controls=True, deletion="observation"),
}


def named_panel(name: str, scale: float = 1.0, **overrides) -> Panel:
    """A named panel, optionally scaled down (workers and firms times ``scale``)."""
    spec = dict(PANELS[name])
    if scale != 1.0:
        spec["workers"] = max(50, int(spec["workers"] * scale))
        spec["firms"] = max(10, int(spec["firms"] * scale))
        if "regions" in spec and spec["firms"] % spec["regions"]:
            spec["firms"] -= spec["firms"] % spec["regions"]
    spec.update(overrides)
    return generate_panel(**spec)
