"""Batch::loudness on the device (qm_pixel_loudness) against the host composition.

Packed pixels (paint/src/sone.rs's format, packed by the format's rule) are read, composed and
read on their curves by the device kernel; the host form of the same path, qm_pixel_ndens (equal to
the oracle's composition bit for bit, tests/test_pixel_read.py), with curves of the oracle's Zwicker
in double, is the checker. The device takes its curves from the pixel's shapes with its own FP32
Zwicker and adds a line's runs in shared memory in any order, so Nden agrees to 1e-4 relative, far
inside the 0.5 % of the reference's loudness check (about 5e-7 is seen); a layer without a shape
reads 0 on both.
"""

import numpy as np
import pytest

from oracle import oracle
from quietmap_b200 import native
from test_pixel_read import LAYERS, _pack, _pixel

pytestmark = pytest.mark.gpu

REL = 1e-4


def _host_ndens(packed, curves, shares, runs):
    tables = np.zeros((LAYERS + 1, 3, 191))
    for c in range(LAYERS + 1):
        for p in range(3):
            shape = curves[c][p]
            if shape is not None:
                shape32 = np.float32(shape).astype(np.float64)
                tables[c, p] = oracle.zwicker_many([shape32 + (-30.0 + step) for step in range(191)])
    return native.pixel_ndens(packed, LAYERS, 2.0, tables, shares, runs)


@pytest.fixture(scope="module")
def ctx():
    c = native.Context(0)
    yield c
    c.close()


def _pixels(seed, n, profiled=True):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        layers, curves = _pixel(rng)
        if not profiled:
            for _, lines in layers:
                for line in lines:
                    line["profile"] = None
        if rng.random() < 0.3:
            curves[int(rng.integers(0, LAYERS + 1))] = [None, None, None]
        out.append((_pack(layers, curves), curves))
    return out


@pytest.mark.parametrize("profiled", [True, False])
def test_device_ndens_match_the_host_composition(ctx, profiled):
    rng = np.random.default_rng(31)
    shares = rng.uniform(0.3, 9.0, (12, 24))
    runs = [4, 1, 3]
    pixels = _pixels(41 if profiled else 43, 48, profiled)
    got, ms = ctx.pixel_loudness([p for p, _ in pixels], LAYERS, 2.0, shares, runs, stats=True)
    worst = 0.0
    for k, (packed, curves) in enumerate(pixels):
        want = _host_ndens(packed, curves, shares, runs)
        for c in range(LAYERS + 1):
            if want[c] == 0.0:
                assert got[k, c] == 0.0, (k, c, got[k], want)
                continue
            rel = abs(float(got[k, c]) - want[c]) / want[c]
            worst = max(worst, rel)
            assert rel < REL, (k, c, float(got[k, c]), want[c])
    print(f"pixel loudness: {len(pixels)} pixels, worst relative Nden error {worst:.2e}, kernel {ms:.2f} ms")


def test_device_loudness_refuses_a_malformed_pixel_by_its_index(ctx):
    pixels = [p for p, _ in _pixels(47, 3, False)]
    pixels[1] = pixels[1][:-5]  # its curves cut short
    with pytest.raises(native.QmError, match="pixel 1"):
        ctx.pixel_loudness(pixels, LAYERS, 2.0)


def test_device_loudness_refuses_a_grid_finer_than_its_limit(ctx):
    pixels = [p for p, _ in _pixels(53, 1, False)]
    with pytest.raises(native.QmError, match="bins"):
        ctx.pixel_loudness(pixels, LAYERS, 0.5)
