"""Level distributions over time (popup/src/distribution.rs) restated in the oracle, pinned to
the reference's own tests (distribution.rs:300-407): Poisson passes in progress filling the time
and keeping the mean, many quiet lines keeping their energy, runs putting each sum in its bin."""

import math

from oracle import distribution as dist


def test_passes_in_progress_fill_the_time_and_keep_the_mean():
    for mean in (2.2250738585072014e-308, 1e-18, 1e-4, 0.03, 0.7, 5.0, 60.0):
        values = dist.pass_values(mean)
        assert all(math.isfinite(v) and s >= 0.0 for v, s in values.pairs), mean
        shares = sum(s for _, s in values.pairs)
        energy = sum(s * v for v, s in values.pairs)
        assert abs(shares - 1.0) < 1e-9 and abs(energy - 1.0) < 1e-9, mean
    sparse = dist.pass_values(0.01)
    assert abs(sparse.pairs[0][1] - 0.99005) < 1e-5
    assert sparse.pairs[1][0] == 100.0
    dense = dist.pass_values(60.0)
    within = sum(s for v, s in dense.pairs if 0.75 <= v <= 1.25)
    assert within > 0.94, within


def test_many_quiet_lines_keep_their_energy():
    total = dist.Distribution(0.5)
    total.silent = 1.0
    values = dist.line_values(0.5)
    mean = sum(v * s for v, s in values.pairs)
    for _ in range(500):
        total = total.with_line(values)
    energy = sum(i * s for i, s in total.intensities())
    assert abs(energy / (500.0 * mean) - 1.0) < 1e-9, energy


def test_runs_put_each_sum_in_the_bin_of_its_level():
    lines = [(dist.line_values(1e-3), 1e3), (dist.line_values(0.5), 1e5), (dist.line_values(30.0), 2e4),
             (dist.line_values(0.0, duty=0.02), 1e6), (dist.LineValues([(0.0, 0.3), (0.0, 0.7)]), 1.0),
             (dist.LineValues([(4e4, 1.0)]), 1.0)]
    for bin_db in (0.5, 1.0):
        grid = dist.Distribution(bin_db)
        n = grid.bin_count()
        for line, scale in lines:
            for intensity in (0.0, 1e-7, 3.3e3, 1e5, 2.2e7, 1e19):
                ours = [None] * (n + 1)

                def visit(b, sums):
                    at = n if b is None else b
                    assert ours[at] is None, "a bin visited twice"
                    ours[at] = sums

                grid.runs(intensity, line, scale, visit)
                expected = [[0.0, 0.0] for _ in range(n + 1)]
                for relative, share in line.pairs:
                    value = scale * relative
                    total = intensity + value
                    at = grid.bin(10.0 * math.log10(total)) if total > 0.0 else n
                    expected[at][0] += share
                    expected[at][1] += share * value
                for at, (e_share, e_weighted) in enumerate(expected):
                    shares, weighted = ours[at] if ours[at] is not None else (0.0, 0.0)
                    close = lambda a, b: abs(a - b) <= 1e-12 * max(abs(b), 1e-300)
                    assert close(shares, e_share) and close(weighted, e_weighted), (bin_db, intensity, at)
