"""Preparation parity: retained masks, preparation receipts and error classes
equal the reference plugin's on every golden case (tests/golden/prep_cases.json,
made by tests/golden/make_golden.py)."""

import hashlib

import numpy as np
import pytest

from fevc_b200 import abi
from fevc_b200.panel import Panel

import make_golden


ALL_PANELS = {**make_golden.PANELS, **make_golden.CONTROL_PANELS, **make_golden.OBSERVATION_PANELS}


@pytest.mark.parametrize("name", list(ALL_PANELS))
def test_panel_preparation_matches_reference(lib, golden, name):
    """Match panels through the match-deletion graph; leave-observation-out
    panels through the observation graph (reference graph.rs:82-243)."""
    rec = golden["prep"]["panels"][name]
    panel = ALL_PANELS[name]["build"]()
    assert make_golden.panel_digest(panel) == rec["panel_sha256"], "panel generator drifted"
    e = abi.Engine(lib)
    e.prepare(panel, deletion_mode=rec.get("deletion_mode", 1))
    receipt = e.receipt()
    mask = e.retained_mask(panel.rows)
    e.release()
    assert hashlib.sha256(mask.tobytes()).hexdigest() == rec["mask_sha256"]
    for k, v in rec["receipt"].items():
        assert receipt[k] == v, (k, receipt[k], v)


@pytest.mark.parametrize("name", sorted(make_golden.error_cases()))
def test_error_cases_match_reference(lib, golden, name):
    rec = golden["prep"]["errors"][name]
    cols = {k: np.array([float(x) for x in v], dtype=np.float64) for k, v in rec["columns"].items()}
    panel = Panel(cols["worker"], cols["firm"], cols["deletion"], cols["outcome"], cols["frequency"],
                  cols["target_weight"])
    e = abi.Engine(lib)
    if rec["status"] == 0:
        e.prepare(panel)
        e.release()
        return
    with pytest.raises(abi.EngineError) as err:
        e.prepare(panel)
    assert err.value.code == rec["status"], err.value.message


def test_row_order_invariance(lib):
    """Permuting input rows changes neither dimensions nor the semantic plan
    (reference engine.rs:4188 batch/row-order invariance)."""
    from fevc_b200.panel import generate_panel
    from oracle import oracle

    p = generate_panel(1500, 100, 5, move_p=0.25, seed=8)
    perm = np.random.default_rng(0).permutation(p.rows)
    q = Panel(p.worker[perm], p.firm[perm], p.deletion[perm], p.outcome[perm], p.frequency[perm],
              p.target_weight[perm])
    views = []
    for panel in (p, q):
        e = abi.Engine(lib)
        e.prepare(panel)
        v = oracle.problem_view(lib, e.generation)
        views.append((v.cells, v.units, v.strata,
                      sorted(v.unit_rank[i] for i in range(v.units)),
                      sorted(v.stratum_rank[i] for i in range(v.strata))))
        e.release()
    assert views[0] == views[1]
