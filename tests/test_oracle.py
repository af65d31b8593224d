"""The oracle against the reference plugin's solved golden cases
(tests/golden/jla_cases.json): the four components, the correction and the MCSE."""

import json
from pathlib import Path

import numpy as np
import pytest

from fevc_b200 import abi

import make_golden


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("name", list(make_golden.PANELS))
@pytest.mark.parametrize("which", [0, 1])
def test_oracle_matches_reference(lib, oracle_mod, golden, name, which):
    rec = golden["jla"]["panels"][name][which]
    panel = make_golden.PANELS[name]["build"]()
    e = abi.Engine(lib)
    e.prepare(panel)
    out = oracle_mod.run(oracle_mod.problem_view(lib, e.generation), seed=rec["seed"], probes=rec["probes"],
                         centering=rec["centering"])
    e.release()
    for key, okey in (("plugin", "plugin"), ("correction", "correction"), ("corrected", "corrected"),
                      ("numerical_mcse", "mcse")):
        assert rel(out[okey], rec[key]) < 1e-11, (key, out[okey], rec[key])


@pytest.mark.parametrize("name", list(make_golden.CONTROL_PANELS))
@pytest.mark.parametrize("which", [0, 1])
def test_generic_oracle_matches_reference(lib, oracle_mod, golden, name, which):
    """The controlled (generic) estimator's restatement against the plugin."""
    rec = golden["jla"]["controls"][name][which]
    panel = make_golden.CONTROL_PANELS[name]["build"]()
    e = abi.Engine(lib)
    e.prepare(panel)
    out = oracle_mod.run(oracle_mod.problem_view(lib, e.generation), seed=rec["seed"], probes=rec["probes"],
                         centering=rec["centering"])
    e.release()
    for key, okey in (("plugin", "plugin"), ("correction", "correction"), ("corrected", "corrected"),
                      ("numerical_mcse", "mcse")):
        assert rel(out[okey], rec[key]) < 1e-10, (key, out[okey], rec[key])


@pytest.mark.parametrize("name", list(make_golden.OBSERVATION_PANELS))
@pytest.mark.parametrize("which", [0, 1])
def test_observation_oracle_matches_reference(lib, oracle_mod, golden, name, which):
    """Leave-observation-out (one Rademacher sign per physical copy, classes of
    equal semantic rank) restated against the plugin's generic engine."""
    rec = golden["jla"]["observation"][name][which]
    panel = make_golden.OBSERVATION_PANELS[name]["build"]()
    e = abi.Engine(lib)
    e.prepare(panel, deletion_mode=2)
    out = oracle_mod.run(oracle_mod.problem_view(lib, e.generation), seed=rec["seed"], probes=rec["probes"],
                         centering=rec["centering"])
    e.release()
    for key, okey in (("plugin", "plugin"), ("correction", "correction"), ("corrected", "corrected"),
                      ("numerical_mcse", "mcse")):
        assert rel(out[okey], rec[key]) < 1e-10, (key, out[okey], rec[key])


def test_observation_classes_number_copies_through_the_class(lib, oracle_mod):
    """Rows of equal semantic rank share one class entity; their copies are
    numbered consecutively in row order (reference generic_jla.rs:4158-4215)."""
    panel = make_golden.OBSERVATION_PANELS["obs_duplicates_1500"]["build"]()
    e = abi.Engine(lib)
    e.prepare(panel, deletion_mode=2)
    v = oracle_mod.problem_view(lib, e.generation)
    rank = np.ctypeslib.as_array(v.row_rank, shape=(v.rows,)).copy()
    off = np.ctypeslib.as_array(v.row_copy_offset, shape=(v.rows,)).copy()
    freq = np.ctypeslib.as_array(v.row_frequency, shape=(v.rows,)).copy()
    e.release()
    assert v.deletion_mode == 2
    assert len(np.unique(rank)) < v.rows  # the panel repeats rows
    for r_ in np.unique(rank)[:400]:
        rows = np.flatnonzero(rank == r_)
        assert np.array_equal(off[rows], np.concatenate([[0], np.cumsum(freq[rows])[:-1]]))


def test_kat_unit_detail(lib, oracle_mod):
    """Per-unit shares of the 12-row known-answer design sum to one and the
    cell weights are finite (reference rust_mata_shared_atoms.rs:108-194)."""
    e = abi.Engine(lib)
    e.prepare(make_golden.kat12())
    out = oracle_mod.run(oracle_mod.problem_view(lib, e.generation), probes=5)
    e.release()
    assert np.allclose(out["projection_share"] + out["residual_share"], 1.0, atol=1e-14)
    assert out["projection_share"].shape == (8,) and out["cell_correction_weight"].shape == (4,)
    assert np.all(np.isfinite(out["deleted_mass"]))


EXACT = json.loads((Path(__file__).resolve().parent / "golden" / "exact_cases.json").read_text())["cases"]


@pytest.mark.parametrize("name", sorted(EXACT))
@pytest.mark.parametrize("which", [0, 1])
def test_exact_oracle_matches_the_plugin_exact_estimator(lib, oracle_mod, name, which):
    """The numpy restatement of the exact estimator against the plugin's own
    (algorithm EXACT) on the same prepared problem."""
    case = EXACT[name]
    rec = case["records"][which]
    panel = make_golden.EXACT_PANELS[name]["build"]()
    assert make_golden.panel_digest(panel) == case["panel_sha256"]
    e = abi.Engine(lib)
    e.prepare(panel)
    try:
        got = oracle_mod.exact(oracle_mod.problem_view(lib, e.generation), centering=rec["centering"])
    finally:
        e.release()
    for key in ("plugin", "correction", "corrected"):
        want = np.array(rec[key])
        assert np.max(np.abs(got[key] - want)) <= 1e-9 * max(np.max(np.abs(want)), 1e-12), (key, got[key], want)
