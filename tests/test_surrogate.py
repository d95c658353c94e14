"""The surrogate's CPU side: the FP64 network oracle checked against finite differences, and the
oracle's feature extraction and eligibility on hand-built paths."""

import numpy as np

from helpers import Stock, point_sources, square
from oracle import mlp, oracle
from quietmap_b200 import abi, native, scenes


def _small_net(seed=3):
    p = native.init_params(seed).astype(np.float64)
    q = abi.SURR_WEIGHTS
    rng = np.random.default_rng(seed)
    p[q:q + 32] = rng.normal(0, 0.1, 32)            # in_shift
    p[q + 32:q + 64] = rng.uniform(0.5, 2.0, 32)    # in_scale
    p[q + 64:q + 72] = rng.uniform(5, 15, 8)        # out_shift
    p[q + 72:q + 80] = rng.uniform(2, 6, 8)         # out_scale
    # biases away from zero so every term of the gradient is exercised
    o = 0
    for k in range(5):
        o += abi.SURR_DIMS[k + 1] * abi.SURR_DIMS[k]
        p[o:o + abi.SURR_DIMS[k + 1]] = rng.normal(0, 0.1, abi.SURR_DIMS[k + 1])
        o += abi.SURR_DIMS[k + 1]
    return p


def test_parameter_layout():
    assert abi.SURR_WEIGHTS == mlp.WEIGHTS == 207880
    assert abi.SURR_PARAMS == abi.SURR_WEIGHTS + 161


def test_oracle_gradient_matches_finite_differences():
    p = _small_net()
    rng = np.random.default_rng(5)
    x = rng.normal(0, 1, (16, 32))
    y = rng.normal(10, 4, (16, 8))
    g, loss = mlp.gradients(p, x, y)
    assert loss > 0
    idx = np.concatenate([rng.choice(abi.SURR_WEIGHTS, 24, replace=False),
                          [0, 8192, 8192 + 256, abi.SURR_WEIGHTS - 1, abi.SURR_WEIGHTS - 9]])
    for i in idx:
        h = 1e-6 * max(1.0, abs(p[i]))
        a, b = p.copy(), p.copy()
        a[i] += h
        b[i] -= h
        num = (mlp.gradients(a, x, y)[1] - mlp.gradients(b, x, y)[1]) / (2 * h)
        assert abs(num - g[i]) <= 1e-6 + 1e-4 * abs(num), (i, num, g[i])


def test_bf16_rounding_is_round_to_nearest_even():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.0e38], np.float32)
    r = mlp.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == -2.5


def _one_building_scene():
    stock = Stock(side_m=400.0, offset_m=200.0)
    stock.building(7, 12.0, [square(0.0, 0.0, 5.0)])
    sources = point_sources(stock, [(-60.0, 0.0), (-60.0, 80.0)])
    return stock, stock.scene(sources=sources)


def test_oracle_features_of_a_path_over_one_building():
    stock, scene = _one_building_scene()
    ora = oracle.OracleScene(scene)
    r = stock.steps((40.0, 0.0))
    grid = scenes.Grid(origin=(int(r[0]), int(r[1])), spacing=32, nx=1, ny=1)
    f, lab, ok = ora.surrogate_samples(grid)
    assert ok.all()
    # source (-60, 0) -> receiver (40, 0): 100 m, the building spans x in [-5, 5] at 12 m.
    a = f[0]
    assert abs(a[0] - 0.1) < 1e-12
    assert abs(a[1] - 0.005) < 1e-8 and abs(a[2] - 0.4) < 1e-8 and a[3] == 0.0
    assert a[5] == a[6] == a[7] == 0.5
    assert abs(a[8] - 0.55) < 1e-9 and abs(a[9] - 0.65) < 1e-9 and abs(a[10] - 1.2) < 1e-9
    assert np.all(a[11:] == 0.0)
    # the second source sees the receiver past the building: no roof, ground attenuation only
    b = f[1]
    assert np.all(b[8:] == 0.0)
    assert np.all(lab[0] > lab[1])  # the screened path is attenuated more in every band


def test_oracle_eligibility_limits_roofs_to_eight():
    stock = Stock(side_m=600.0, offset_m=300.0)
    for i in range(9):
        stock.building(i + 1, 8.0, [square(-100.0 + 20.0 * i, 0.0, 4.0)])
    sources = point_sources(stock, [(-140.0, 0.0), (-140.0, 30.0)])
    scene = stock.scene(sources=sources)
    ora = oracle.OracleScene(scene)
    r = stock.steps((100.0, 0.0))
    grid = scenes.Grid(origin=(int(r[0]), int(r[1])), spacing=32, nx=1, ny=1)
    f, lab, ok = ora.surrogate_samples(grid)
    assert not ok[0]  # nine roofs on the way
    assert ok[1]      # the oblique path misses them
