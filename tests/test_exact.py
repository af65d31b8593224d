"""The exact-estimator request gates through the C ABI (no GPU): the
reference's option ranges and its identified-dimension limit, and the
B200 ceiling that lifts that limit for a generation."""

import pytest

from fevc_b200 import abi
from fevc_b200.panel import generate_panel


def prepared(lib):
    e = abi.Engine(lib)
    e.prepare(generate_panel(400, 60, 5, move_p=0.3, seed=3))
    return e


def test_exact_limit_outside_the_reference_range_is_invalid(lib):
    e = prepared(lib)
    try:
        for limit in (1, 2001):
            with pytest.raises(abi.EngineError) as err:
                e.solve_v5(e.exact_request_v5(limit))
            assert err.value.code == 20 and "exact limit" in err.value.message
    finally:
        e.release()


def test_identified_dimension_above_the_limit_is_a_resource_limit(lib):
    e = prepared(lib)
    try:
        with pytest.raises(abi.EngineError) as err:
            e.solve_v5(e.exact_request_v5(10))
        assert err.value.code == 40 and "exact_limit" in err.value.message
    finally:
        e.release()


def test_exact_ceiling_is_range_checked(lib):
    e = prepared(lib)
    try:
        with pytest.raises(abi.EngineError) as err:
            e.exact_ceiling(2_000_000)
        assert err.value.code == 20
        e.exact_ceiling(0)
    finally:
        e.release()


def test_exact_request_on_a_controls_panel_is_refused(lib):
    e = abi.Engine(lib)
    e.prepare(generate_panel(400, 60, 5, move_p=0.3, year_controls=True, seed=3))
    try:
        with pytest.raises(abi.EngineError) as err:
            e.solve_v5(e.exact_request_v5(2000), controls_count=4)
        assert err.value.code == 11
    finally:
        e.release()
