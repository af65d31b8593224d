"""The allocation-free atom entry point against the allocating one.

fevcb_counter_atoms_noalloc_v1 serves callers that cannot allocate device
memory (their own framework already holds the device's memory, or their
memory plan is fixed at start-up): it stages inputs and outputs in one fixed
8 MiB device array instead of cudaMalloc.  This file is collected last so a
failure here leaves every other test already run; it passes alone in a fresh
process and after the rest of the suite.
"""

import numpy as np
import pytest

from fevc_b200 import abi

pytestmark = pytest.mark.gpu

LIMIT = 8 << 20


def scratch_need(count: int, columns: int) -> int:
    """Bytes of the fixed array a request uses: entities, trials and atoms,
    each rounded up to 256 bytes."""
    r = lambda b: (b + 255) & ~255  # noqa: E731
    return 2 * r(count * 8) + r(count * columns * 8)


def test_no_alloc_atoms_equal_the_allocating_entry_point(lib):
    rng = np.random.default_rng(2024)
    # two calls in a row with different inputs, the second larger than the
    # first, so atoms left in the array by the first call would show up in
    # the second's output if the output region were not cleared
    for call, (count, columns, first) in enumerate(((1200, 9, 13), (5000, 16, 0))):
        entity = rng.integers(1, 2**50, count, dtype=np.uint64)
        trials = rng.integers(1, 300, count).astype(np.uint64)
        for tag in (abi.TAG_LEVERAGE, abi.TAG_TARGET):
            want = abi.device_atoms(lib, 8675309 + call, tag, first, columns, entity, trials)
            got = abi.device_atoms(lib, 8675309 + call, tag, first, columns, entity, trials, no_alloc=True)
            # integer atoms: the tolerance of the other atom tests is exact equality
            assert np.array_equal(got, want), (call, tag)


def test_no_alloc_accepts_a_request_of_exactly_the_array_size(lib):
    count, columns = 65536, 14
    assert scratch_need(count, columns) == LIMIT
    rng = np.random.default_rng(7)
    entity = rng.integers(1, 2**40, count, dtype=np.uint64)
    trials = rng.integers(1, 50, count).astype(np.uint64)
    for _ in range(2):
        want = abi.device_atoms(lib, 99, abi.TAG_LEVERAGE, 4, columns, entity, trials)
        got = abi.device_atoms(lib, 99, abi.TAG_LEVERAGE, 4, columns, entity, trials, no_alloc=True)
        assert np.array_equal(got, want)


def test_no_alloc_rejects_requests_beyond_the_array(lib):
    # 256 bytes above the array: refused before anything is copied
    count, columns = 349505, 1
    assert scratch_need(count, columns) == LIMIT + 256
    entity = np.arange(1, count + 1, dtype=np.uint64)
    trials = np.ones(count, np.uint64)
    with pytest.raises(abi.EngineError) as err:
        abi.device_atoms(lib, 1, abi.TAG_LEVERAGE, 0, columns, entity, trials, no_alloc=True)
    assert err.value.code == 40 and "scratch" in err.value.message
