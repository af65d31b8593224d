"""Counter-V1 restatement in the oracle and in the library's host self-test,
pinned to the reference's permanent vectors (rust/crates/vckss-core/src/rng.rs:366-419,
rust/RNG_CONTRACT.md:5-41)."""

import pytest

TAG_LEVERAGE = 0x4C45564552414745
TAG_TARGET = 0x0054415247455401
TAG_COMPONENT = 0x434F4D50494E4601
TAG_CRITICAL = 0x434F4D5051435201
TAG_FOLD = 0x434F4D5056464C01
TAG_RESIDUAL = 0x4F4253524D4F4D01


def word(o, seed, tag, probe, entity, w):
    return o.philox_block(seed, tag, probe // 4, entity, w)[probe % 4]


def test_philox_block_vector(oracle_mod):
    assert oracle_mod.philox_block(123_456_789, TAG_LEVERAGE, 17, 99, 3) == [
        0x9F4B6EA90B26B57D, 0x529B58B961489B78, 0x9D84FAB11898A6A0, 0x469459830D836D27]


@pytest.mark.parametrize("tag,expected", [
    (TAG_LEVERAGE, 0x40CE71BF068D1E52), (TAG_TARGET, 0x46E2BF28FAB1EA2C), (TAG_COMPONENT, 0x1C2FDA9DD5D4F916),
    (TAG_CRITICAL, 0x63A164B2C1229856), (TAG_FOLD, 0x7B4FB67CD3FCEB3C), (TAG_RESIDUAL, 0xDA875EA1EBD7ED3E)])
def test_domain_words(oracle_mod, tag, expected):
    assert word(oracle_mod, 123, tag, 5, 7, 0) == expected


@pytest.mark.parametrize("trials,expected", [(1, -1), (5, -1), (20, 0), (64, -4), (65, -5), (100, 4)])
def test_compressed_sums(oracle_mod, trials, expected):
    assert oracle_mod.rademacher_sum(123, TAG_LEVERAGE, 5, 7, trials) == expected


def test_sum_is_popcount_of_selected_bits(oracle_mod):
    for trials in (1, 63, 64, 65, 127, 128, 200):
        pos = 0
        for w in range((trials + 63) // 64):
            bits = word(oracle_mod, 987_654_321, TAG_TARGET, 9, 29, w)
            n = min(64, trials - 64 * w)
            pos += bin(bits & ((1 << n) - 1)).count("1")
        assert oracle_mod.rademacher_sum(987_654_321, TAG_TARGET, 9, 29, trials) == 2 * pos - trials


def test_zero_trials_rejected(oracle_mod):
    with pytest.raises(ValueError):
        oracle_mod.rademacher_sum(1, TAG_LEVERAGE, 0, 0, 0)


def test_library_selftest(lib):
    assert lib.vckss_rust_selftest() == 0
