"""The library's level distributions (qm_distribution.cuh: one source for the host and the
device), run on the host through the C ABI: adding lines to distributions and reading exceeded
levels equal the oracle's restatement (pinned to the reference's distribution tests) to the bit
on 0.1, 0.5 and 2 dB grids; the reference's own properties hold through the library (passes
fill the time and keep the mean; many quiet lines keep their energy); line and pass values
match the oracle's; and the entry points reject what the reference cannot take."""

import math

import numpy as np
import pytest

from oracle import distribution as dist
from oracle import oracle
from quietmap_b200 import abi, native


def _bins(d):
    return np.array(d.bins, dtype=np.float64).reshape(-1, 2)


def _pairs(line):
    return np.array(line.pairs, dtype=np.float64).reshape(-1, 2)


def _lines(rng):
    """Lines of every kind the reference adds: Kurze lines sparse to dense, events over a duty,
    passes, steady sounds, values at zero, equal values, and random sets."""
    out = [(dist.line_values(lam), 10.0 ** rng.uniform(0.0, 7.0)) for lam in (1e-5, 1e-3, 0.05, 0.5, 3.0, 30.0)]
    out += [(dist.line_values(0.0, duty=d), 10.0 ** rng.uniform(0.0, 7.0)) for d in (0.001, 0.02, 0.5, 1.0)]
    out += [(dist.pass_values(m), 10.0 ** rng.uniform(0.0, 7.0)) for m in (1e-6, 0.01, 0.7, 5.0, 60.0)]
    out += [(dist.LineValues([(4e4, 1.0)]), 1.0), (dist.LineValues([(0.0, 0.3), (0.0, 0.7)]), 1.0),
            (dist.LineValues([(2.0, 0.25), (2.0, 0.25), (0.5, 0.5)]), 3.0)]
    for _ in range(10):
        n = int(rng.integers(1, 40))
        values = 10.0 ** rng.uniform(-3.0, 3.0, n) * (rng.random(n) > 0.1)
        shares = rng.dirichlet(np.ones(n))
        out.append((dist.LineValues(list(zip(values, shares))), 10.0 ** rng.uniform(-2.0, 9.0)))
    return out


@pytest.mark.parametrize("bin_db", [0.1, 0.5, 2.0])
def test_adding_lines_matches_the_oracle_to_the_bit(bin_db):
    rng = np.random.default_rng(int(bin_db * 10))
    ours = dist.Distribution(bin_db)
    ours.silent = 1.0
    bins, silent = _bins(ours), 1.0
    for line, scale in _lines(rng):
        want = ours.with_line(line, scale)
        got_bins, got_silent = native.distribution_with_line(bin_db, bins, silent, _pairs(line), scale)
        assert np.array_equal(got_bins, _bins(want)) and got_silent == want.silent
        for exceeded in (0.0, 0.01, 0.1, 0.5, 0.9, 0.999, 1.0):
            assert native.distribution_exceeded_db(bin_db, got_bins, exceeded) == want.exceeded_db(exceeded)
        # Values handed over in any order add the same: the library sorts them as the reference
        # does, equal values keeping their order.
        shuffled = _pairs(line)[rng.permutation(len(line.pairs))]
        again, again_silent = native.distribution_with_line(bin_db, bins, silent, shuffled, scale)
        assert np.allclose(again, got_bins, rtol=1e-12, atol=0.0) and abs(again_silent - got_silent) <= 1e-12
        ours, bins, silent = want, got_bins, got_silent
    assert np.count_nonzero(bins[:, 0]) > 10


def test_passes_in_progress_fill_the_time_and_keep_the_mean():
    """distribution.rs:308-338 through the library, and the values equal the oracle's."""
    for mean in (2.2250738585072014e-308, 1e-18, 1e-4, 0.03, 0.7, 5.0, 60.0, 700.0):
        values = native.distribution_pass_values(mean)
        assert np.all(np.isfinite(values)) and np.all(values[:, 1] >= 0.0), mean
        assert abs(values[:, 1].sum() - 1.0) < 1e-9 and abs((values[:, 0] * values[:, 1]).sum() - 1.0) < 1e-9, mean
        order = np.argsort(values[:, 0], kind="stable")
        assert np.array_equal(values[order], _pairs(dist.pass_values(mean))), mean
    sparse = native.distribution_pass_values(0.01)
    assert abs(sparse[0, 1] - 0.99005) < 1e-5 and sparse[1, 0] == 100.0


def test_many_quiet_lines_keep_their_energy():
    """distribution.rs:340-361 through the library: 500 lines at lambda 0.5 added one by one."""
    values = native.distribution_line_values(0.5)
    mean = float((values[:, 0] * values[:, 1]).sum())
    bins = np.zeros((native.distribution_bins(0.5), 2))
    silent = 1.0
    for _ in range(500):
        bins, silent = native.distribution_with_line(0.5, bins, silent, values)
    energy = float(bins[:, 1].sum())
    assert abs(energy / (500.0 * mean) - 1.0) < 1e-9, energy


def test_line_values_match_the_oracle():
    """Kurze lines by the library's sampler equal the oracle's within the sampler's 1e-12; events
    over a duty exactly; the node shares exactly."""
    for lam in (0.0, 1e-6, 1e-4, 2e-3, 0.5, 9.99, 10.0, 400.0, math.inf):
        got = native.distribution_line_values(lam)
        want = _pairs(dist.line_values(lam))
        nodes = np.array(dist.node_probabilities())
        assert len(got) == abi.DISTRIBUTION_LINE_NODES == len(nodes)
        assert np.array_equal(got[:, 1], nodes[:, 1])
        relative = np.array(oracle.relative_intensity(lam, list(nodes[:, 0])))
        assert np.allclose(got[:, 0], relative, rtol=1e-12, atol=0.0), lam
        assert np.allclose(np.sort(got[:, 0]), want[:, 0], rtol=1e-12, atol=0.0), lam
    for duty in (1e-3, 0.25, 1.0):
        assert np.array_equal(native.distribution_line_values(0.0, duty=duty), [[0.0, 1.0 - duty], [1.0 / duty, duty]])


def test_errors():
    bins = np.zeros((360, 2))
    for bin_db in (0.0, -1.0, math.nan, math.inf, 0.05, 400.0):
        with pytest.raises(native.QmError) as err:
            native.distribution_bins(bin_db)
        assert err.value.status == abi.QM_ERR_ARGUMENT, bin_db
    assert native.distribution_bins(0.1) == 1800 and native.distribution_bins(2.0) == 90
    for values in ([[-1.0, 1.0]], [[1.0, -0.5]], [[math.nan, 1.0]]):
        with pytest.raises(native.QmError) as err:
            native.distribution_with_line(0.5, bins, 1.0, values)
        assert err.value.status == abi.QM_ERR_ARGUMENT and "value 0" in str(err.value)
    with pytest.raises(native.QmError) as err:
        native.distribution_with_line(0.5, bins, 1.0, [[1.0, 1.0]], scale=0.0)
    assert err.value.status == abi.QM_ERR_ARGUMENT
    with pytest.raises(native.QmError) as err:
        native.distribution_pass_values(800.0)
    assert err.value.status == abi.QM_ERR_ARGUMENT and "700" in str(err.value)
    with pytest.raises(native.QmError) as err:
        native.distribution_pass_values(60.0, cap=3)
    assert err.value.status == abi.QM_ERR_CAPACITY
    with pytest.raises(native.QmError) as err:
        native.distribution_line_values(0.5, duty=1.5)
    assert err.value.status == abi.QM_ERR_ARGUMENT
    # A line of no values holds no time, so no moment survives the sum (as in the reference).
    start = np.zeros((360, 2))
    start[100] = (0.5, 0.5 * dist.energy(-30.0 + 100 * 0.5))
    out, silent = native.distribution_with_line(0.5, start, 0.5, np.zeros((0, 2)))
    assert np.array_equal(out, np.zeros((360, 2))) and silent == 0.0
