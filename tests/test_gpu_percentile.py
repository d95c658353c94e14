"""Line-source levels in time on the device (qm_line_level_quantiles) against the oracle's
sampler (physics/src/percentile.rs): every regime, FP64 within 1e-12 relative (the device's and
the host's logarithms and exponentials may differ in the last bits)."""

import numpy as np
import pytest

from oracle import oracle
from quietmap_b200 import native

pytestmark = pytest.mark.gpu


def test_device_levels_match_the_oracle():
    ctx = native.Context(0)
    probabilities = np.concatenate([(np.arange(99) + 0.5) / 100.0, 1.0 - 10.0 ** (-2.0 - 0.25 * np.arange(25)),
                                    [0.001, 0.0049, 0.995, 0.9951, 1.0 - 0.5e-8]])
    lambdas = [0.0, 1e-7, 3e-5, 1e-4, 1.3e-4, 0.01, 0.37, 1.0, 9.99, 10.0, 31.0, np.inf]
    lam = np.repeat(lambdas, len(probabilities))
    p = np.tile(probabilities, len(lambdas))
    got = ctx.line_level_quantiles(lam, p)
    want = np.concatenate([oracle.relative_intensity(l, probabilities) for l in lambdas])
    assert np.array_equal(got == 0.0, want == 0.0)
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=0.0)
    ctx.close()
