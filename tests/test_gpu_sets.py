"""Independent probe sets in one call (fevcb_engine_solve_sets_v1): every
set's components equal a separate V5 solve with that seed and probe count,
on the compressed engine, with controls and with leave-observation-out
deletion; the generation's result is the first set's."""

import numpy as np
import pytest

from fevc_b200 import abi
from fevc_b200.panel import generate_panel

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def request(e, deletion, seed, probes):
    q = e.default_request_v5(deletion)
    v1 = q.v4.v3.v2.v1
    v1.seed = seed
    v1.probes = probes
    v1.pcg_tolerance = 1e-12
    v1.maximum_iterations = 20000
    q.v4.v3.v2.algorithm = 2
    q.tolerance_supplied = 1
    return q


CASES = {
    "match": (lambda: generate_panel(2000, 150, 5, move_p=0.2, seed=11), 1),
    "controls": (lambda: generate_panel(2000, 150, 5, move_p=0.2, year_controls=True, seed=11), 1),
    "observation": (lambda: generate_panel(2000, 150, 5, move_p=0.2, seed=12), 2),
}
SETS = [(8675309, 24), (8675310, 16), (8675311, 20), (8675312, 8)]


@pytest.mark.parametrize("name", sorted(CASES))
def test_sets_equal_separate_solves(lib, name):
    build, deletion = CASES[name]
    panel = build()
    controls = len(panel.controls)
    e = abi.Engine(lib)
    e.prepare(panel, deletion_mode=deletion)
    got = e.solve_sets(request(e, deletion, 1, 2), SETS, controls_count=controls)
    head = e.result()
    e.release()
    assert head == got[0]
    for (seed, probes), res in zip(SETS, got):
        f = abi.Engine(lib)
        f.prepare(panel, deletion_mode=deletion)
        f.solve_v5(request(f, deletion, seed, probes), controls_count=controls)
        want = f.result()
        f.release()
        for key in ("plugin", "correction", "corrected", "numerical_mcse"):
            assert rel(res[key], want[key]) < 1e-9, (name, seed, key, res[key], want[key])


def test_sets_refuse_bad_input(lib):
    panel = generate_panel(2000, 150, 5, move_p=0.2, seed=11)
    e = abi.Engine(lib)
    e.prepare(panel)
    with pytest.raises(abi.EngineError) as err:
        e.solve_sets(request(e, 1, 1, 2), [(5, 1)])
    assert err.value.code == 20
    e.release()
