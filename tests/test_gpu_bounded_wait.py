"""The bounded waits on the device (the bulk copies' mbarriers in the painter, the flight kernel and
the tcgen05 network all wait through one function, which gives up after its limit): a kernel waits
on an mbarrier that nothing completes, and must give up no sooner than its limit and soon after it,
report that to the host, and leave the context usable. No fault is involved: nothing is in flight
when the waiting thread returns."""

import numpy as np
import pytest

from quietmap_b200 import native

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("limit_ms", [50.0, 1000.0])
def test_a_wait_that_nothing_completes_gives_up_at_its_limit(limit_ms):
    ctx = native.Context(0)
    waited = ctx.check_bounded_wait(limit_ms)
    assert limit_ms <= waited < limit_ms + 250.0, waited
    # The context still works: a Zwicker call on a flat spectrum.
    sone = ctx.zwicker(np.full((2, 28), 60.0, np.float32))
    assert np.all(np.isfinite(sone)) and np.all(sone > 0.0)
    ctx.close()


def test_limits_outside_the_range_are_refused():
    ctx = native.Context(0)
    with pytest.raises(RuntimeError, match="limit_ms"):
        ctx.check_bounded_wait(0.0)
    with pytest.raises(RuntimeError, match="limit_ms"):
        ctx.check_bounded_wait(5000.0)
    ctx.close()
