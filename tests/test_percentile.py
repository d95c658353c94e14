"""The line-source quantile table (physics/src/percentile.rs): the oracle's restatement of the
reference's own seeded simulation (physics/src/percentile_tests.rs:1-102) regenerates the table
the reference ships (physics/src/percentile_table.rs, read in place, never copied) bit for bit."""

import re

import numpy as np
import pytest

from conftest import reference_file
from oracle import oracle


@pytest.fixture(scope="module")
def table():
    return oracle.percentile_table(41)


def test_the_simulation_regenerates_the_reference_table_bit_for_bit(table):
    text = open(reference_file("physics/src/percentile_table.rs")).read()
    rows = re.findall(r"\[([^\[\]]+)\]", text)
    ref = np.array([[np.float32(v) for v in r.split(",") if v.strip()] for r in rows], dtype=np.float32)
    assert ref.shape == (41, 100)
    np.testing.assert_array_equal(table, ref)


def test_rows_ascend_and_keep_their_scale(table):
    assert np.all(np.diff(table, axis=1) >= 0.0)
    # A dense line hums at its mean: lambda 10's middle quantile is within a few per cent of 1.
    assert abs(table[40, 50] - 1.0) < 0.05
    # A sparse line is quiet most of the time: lambda 1e-4's median is far below its mean.
    assert table[0, 50] < 0.01


def _splitmix_uniforms(seed, n):
    """n draws of the tests' SplitMix64 generator (percentile_tests.rs:5-21), vectorised: the
    i-th draw's state is the seed plus i + 1 increments."""
    gamma = np.uint64(0x9E37_79B9_7F4A_7C15)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + gamma * np.arange(1, n + 1, dtype=np.uint64)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58_476D_1CE4_E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D0_49BB_1331_11EB)
    return ((z ^ (z >> np.uint64(31))) >> np.uint64(11)).astype(np.float64) / float(1 << 53)


def test_sparse_lines_are_quiet_most_of_the_time_and_dense_ones_hum():
    """percentile_tests.rs:104-129."""
    l90 = lambda lam: 50.0 + 10.0 * np.log10(oracle.relative_intensity(lam, 0.1))
    l10 = lambda lam: 50.0 + 10.0 * np.log10(oracle.relative_intensity(lam, 0.9))
    for lam in (1e-4, 1e-3):
        x = 0.105 / (2.0 * lam)
        expected = 50.0 + 10.0 * np.log10(1.0 / (1.0 + x * x) / (lam * np.pi))
        assert abs(l10(lam) - expected) < 1.0, (lam, l10(lam), expected)
    assert l90(1e-3) < l10(1e-3)
    assert abs(l10(100.0) - 50.0) < 1.0 and abs(l90(100.0) - 50.0) < 1.0
    assert l10(np.inf) == 50.0
    for lam in (1e-4, 1e-2, 0.3, 3.0, 9.9, 10.0, 30.0):
        assert l90(lam) <= l10(lam), lam


def test_every_line_keeps_its_mean():
    """percentile_tests.rs:131-155: within 5 % at every row of the table, halfway between, and
    for lines sparser than it; the rare passes above the last quantile carry the sparse lines."""
    body_p = (np.arange(20_000) + 0.5) / 20_000.0
    last = 1.0 - 1.0 / 20_000.0
    tail_p = last + (np.arange(200_000) + 0.5) / 200_000.0 / 20_000.0
    lambdas = [1e-6, 1e-5] + [1e-4 * 10.0 ** (h / 2.0 / 8.0) for h in range(0, 2 * 41 - 1)]
    for lam in lambdas:
        body = oracle.relative_intensity(lam, body_p).sum() / 20_000.0
        at_last = oracle.relative_intensity(lam, last + 0.5 / 20_000.0)
        tail = (oracle.relative_intensity(lam, tail_p) - at_last).sum() / 200_000.0 / 20_000.0
        assert abs(body + tail - 1.0) < 0.05, (lam, body + tail)


def test_a_line_without_emitters_is_silent():
    """percentile_tests.rs:157-163."""
    for p in (0.001, 0.5, 0.995, 0.9999):
        assert oracle.relative_intensity(0.0, p) == 0.0


def test_independent_sparse_lines_add_up_to_a_denser_one():
    """percentile_tests.rs:165-195: ten and a hundred lines of 1e-4 and ten of 1e-5 sampled line by
    line have the normalised L10 and L5 of one line of the summed density within 0.3 dB."""
    draws = _splitmix_uniforms(0x5EED_2026, 200_000 * (10 + 100 + 10))
    at = 0
    for lines, lam in ((10, 1e-4), (100, 1e-4), (10, 1e-5)):
        u = draws[at:at + 200_000 * lines]
        at += 200_000 * lines
        sums = np.sort(oracle.relative_intensity(lam, u).reshape(200_000, lines).sum(axis=1) / lines)
        for exceeded in (0.1, 0.05):
            sampled = sums[int((1.0 - exceeded) * len(sums))]
            one = oracle.relative_intensity(lam * lines, 1.0 - exceeded)
            assert abs(10.0 * np.log10(sampled / one)) < 0.3, (lines, lam, exceeded)


def test_the_library_builds_the_same_table(table):
    from quietmap_b200 import native
    np.testing.assert_array_equal(native.line_level_table(), table)
