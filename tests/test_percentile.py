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
