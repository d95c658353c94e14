"""The learned surrogate on the GPU: exact training samples, the network's forward pass and
gradients against the FP64 oracle, and a trained network painting against the exact painter."""

import numpy as np
import pytest

from oracle import mlp, oracle
from quietmap_b200 import abi, native, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return native.Context(0)


@pytest.fixture(scope="module")
def road():
    return scenes.road_square()


def _coarse_grid(full, n, offset, source_end=0):
    sp = full.spacing * (full.nx // n)
    return scenes.Grid(origin=(offset, offset), spacing=sp, nx=n, ny=n, source_begin=0, source_end=source_end)


def _random_params(seed, features):
    """He-initialised weights with the normalisation of a feature sample."""
    p = native.init_params(seed)
    q = abi.SURR_WEIGHTS
    mean, sd = features.mean(axis=0), features.std(axis=0)
    p[q:q + 32] = mean
    p[q + 32:q + 64] = np.where(sd > 1e-6, 1.0 / np.maximum(sd, 1e-6), 1.0)
    p[q + 64:q + 72] = 10.0
    p[q + 72:q + 80] = 4.0
    rng = np.random.default_rng(seed)
    o = 0
    for k in range(5):
        o += abi.SURR_DIMS[k + 1] * abi.SURR_DIMS[k]
        p[o:o + abi.SURR_DIMS[k + 1]] = rng.normal(0, 0.1, abi.SURR_DIMS[k + 1])
        o += abi.SURR_DIMS[k + 1]
    return p


def test_samples_match_the_oracle(ctx, road):
    scene, full = road
    grid = _coarse_grid(full, 4, 1000, source_end=3000)
    dev = ctx.scene(scene)
    f, lab, ok = dev.surrogate_samples(grid)
    ora = oracle.OracleScene(scene)
    rf, rlab, rok = ora.surrogate_samples(grid)
    assert np.array_equal(ok, rok), (ok.sum(), rok.sum())
    assert ok.mean() > 0.5
    # Features matter on eligible paths only (the others run the exact path).
    df = np.abs(f[ok] - rf[ok])
    assert df.max() < 2e-4, (df.max(axis=0), np.argwhere(df > 2e-4)[:5])
    err = np.abs(lab - rlab)[ok]
    assert np.percentile(err, 99) <= 0.05 and np.median(err) < 0.005, (np.percentile(err, 99), err.max())


def test_forward_matches_the_oracle(ctx, road):
    scene, full = road
    dev = ctx.scene(scene)
    f, lab, ok = dev.surrogate_samples(_coarse_grid(full, 2, 3000, source_end=700))
    x = f[ok][:1000]
    p = _random_params(7, x)
    net = native.Surrogate(ctx, p)
    out = net.forward(x)
    ref = mlp.forward(p, x, bf16_round=True)
    d = np.abs(out - ref) / 4.0  # in units of the output scale
    assert np.percentile(d, 99) < 0.01 and d.max() < 0.05, (np.percentile(d, 99), d.max())
    # rows beyond a whole tile and a single row give the same answers
    np.testing.assert_allclose(net.forward(x[:1]), out[:1], rtol=0, atol=1e-6)
    np.testing.assert_allclose(net.forward(x[:131]), out[:131], rtol=0, atol=1e-6)


def test_tensor_memory_and_mma_sync_kernels_agree(ctx, road):
    """The tcgen05 inference kernel (the default) and the mma.sync one on the same rows, including a
    ragged last tile."""
    scene, full = road
    dev = ctx.scene(scene)
    f, lab, ok = dev.surrogate_samples(_coarse_grid(full, 2, 3000, source_end=700))
    x = f[ok][:1000]
    net = native.Surrogate(ctx, _random_params(13, x))
    a = net.forward(x)
    net.set_kernel(1)
    b = net.forward(x)
    net.set_kernel(0)
    d = np.abs(a - b) / 4.0
    assert np.percentile(d, 99) < 0.005 and d.max() < 0.02, (np.percentile(d, 99), d.max())


def test_gradients_match_the_oracle(ctx, road):
    scene, full = road
    dev = ctx.scene(scene)
    f, lab, ok = dev.surrogate_samples(_coarse_grid(full, 2, 3000, source_end=700))
    x, y = f[ok][:512], lab[ok][:512]
    p = _random_params(11, x)
    net = native.Surrogate(ctx, p)
    g, loss = net.gradients(x, y)
    rg, rloss = mlp.gradients(p, x, y, bf16_round=True)
    assert abs(loss - rloss) <= 2e-3 * rloss + 1e-6, (loss, rloss)
    o = 0
    for k in range(5):
        for part, n in (("w", abi.SURR_DIMS[k + 1] * abi.SURR_DIMS[k]), ("b", abi.SURR_DIMS[k + 1])):
            a, b = g[o:o + n].astype(np.float64), rg[o:o + n]
            rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
            cos = float(a @ b / max(np.linalg.norm(a) * np.linalg.norm(b), 1e-30))
            assert rel < 0.03 and cos > 0.999, (k, part, rel, cos)
            o += n


@pytest.fixture(scope="module")
def trained(ctx, road):
    scene, full = road
    dev = ctx.scene(scene)
    net = native.Surrogate(ctx, seed=1)
    grids = [_coarse_grid(full, 16, 37), _coarse_grid(full, 16, 211)]
    hist, n = net.train(dev, grids, epochs=4, batch=8192, learning_rate=2e-3, seed=3, max_samples=4_000_000)
    return dev, net, hist, n


def test_training_lowers_the_loss(trained):
    dev, net, hist, n = trained
    assert n == 4_000_000
    assert np.all(np.isfinite(hist)) and hist[-1] < 0.5 * hist[0], hist
    p = net.params()
    assert np.all(np.isfinite(p))


def test_trained_network_beats_the_mean_predictor(ctx, road, trained):
    """The ablation: on held-out paths the trained network's error against the exact labels,
    against the same painter without the learned part (every band predicted as its mean label)."""
    scene, full = road
    dev, net, hist, n = trained
    f, lab, ok = dev.surrogate_samples(_coarse_grid(full, 4, 555, source_end=20000))
    x, y = f[ok], lab[ok]
    pred = net.forward(x)
    err = np.abs(pred - y)
    base = np.abs(y.mean(axis=0) - y)
    p50, p99 = np.percentile(err, 50), np.percentile(err, 99)
    b99 = np.percentile(base, 99)
    print(f"surrogate |A| error p50 {p50:.3f} dB p99 {p99:.3f} dB; mean predictor p99 {b99:.3f} dB")
    assert p99 < 0.5 * b99


def test_surrogate_painter_matches_the_exact_painter(ctx, road, trained):
    scene, full = road
    dev, net, hist, n = trained
    tile = scenes.Grid(origin=(full.origin[0] + 40 * full.spacing, full.origin[1] + 70 * full.spacing),
                       spacing=full.spacing, nx=16, ny=8)
    eb, edba, elden, ehist, est = dev.paint_grid(tile)
    sb, sdba, slden, shist, sst = dev.paint_grid_surrogate(tile, net)
    assert sst["paths"] == est["paths"]
    assert sst["surrogate_paths"] > 0.5 * sst["paths"], sst
    d = np.abs(sdba - edba)
    print(f"cells dBA |surrogate - exact| p50 {np.median(d):.4f} p99 {np.percentile(d, 99):.4f} max {d.max():.4f}; "
          f"surrogate paths {sst['surrogate_paths']} of {sst['paths']}")
    assert np.percentile(d, 99) < 0.5


@pytest.fixture(scope="module")
def terrain():
    return scenes.terrain_square(scale=0.25)


def test_terrain_samples_match_the_oracle(ctx, terrain):
    scene, full = terrain
    dev = ctx.scene(scene)
    sp = full.spacing * (full.nx // 3)
    grid = scenes.Grid(origin=(full.origin[0] + 7, full.origin[1] + 11), spacing=sp, nx=3, ny=3, source_begin=0,
                       source_end=1200)
    f, lab, ok = dev.surrogate_samples(grid)
    rf, rlab, rok = oracle.OracleScene(scene).surrogate_samples(grid)
    assert len(f) == 2 * 9 * 1200
    assert np.array_equal(ok, rok), (ok.sum(), rok.sum())
    assert ok.mean() > 0.3
    assert np.array_equal(f[:, 4], np.tile([0.0, 1.0], len(f) // 2))
    df = np.abs(f[ok] - rf[ok])
    assert df.max() < 2e-3, (df.max(axis=0), np.argwhere(df > 2e-3)[:5])
    err = np.abs(lab - rlab)[ok]
    assert np.percentile(err, 99) <= 0.05 and np.median(err) < 0.005, (np.percentile(err, 99), err.max())


def test_terrain_surrogate_trains_and_paints(ctx, terrain):
    scene, full = terrain
    dev = ctx.scene(scene)
    net = native.Surrogate(ctx, seed=2)
    grids = [scenes.Grid(origin=(full.origin[0] + 13 * k, full.origin[1] + 29 * k), spacing=full.spacing * 32,
                         nx=16, ny=16) for k in range(2)]
    # The painter's recipe: paths within 200 m stay exact (the near field carries a cell's energy).
    hist, n = net.train(dev, grids, epochs=3, batch=8192, learning_rate=2e-3, seed=5, max_samples=3_000_000,
                        exact_within_m=200.0)
    assert hist[-1] < 0.8 * hist[0], hist
    tile = scenes.Grid(origin=(full.origin[0] + 100 * full.spacing, full.origin[1] + 60 * full.spacing),
                       spacing=full.spacing, nx=16, ny=8)
    _, edba, _, _, est = dev.paint_grid(tile)
    _, sdba, _, _, sst = dev.paint_grid_surrogate(tile, net)
    d = np.abs(sdba - edba)
    # The north star's bar: the surrogate painter's cells within 0.5 dB at p99 of the FP64 oracle, here
    # on a seeded row of the tile against every source.
    row = int(np.random.default_rng(25).integers(0, tile.ny))
    e, _, _ = oracle.OracleScene(scene).paint_grid(tile, row * tile.nx, (row + 1) * tile.nx)
    vs_oracle = np.abs(sdba[row * tile.nx:(row + 1) * tile.nx] - 10.0 * np.log10(e.sum(axis=1)))
    print(f"terrain: samples {n}, loss {hist}, surrogate paths {sst['surrogate_paths']} of {sst['paths']}, cell dBA "
          f"vs exact p50 {np.median(d):.3f} p99 {np.percentile(d, 99):.3f} max {d.max():.3f}; vs oracle p99 "
          f"{np.percentile(vs_oracle, 99):.3f} max {vs_oracle.max():.3f}; exact {est['kernel_ms']:.1f} ms, "
          f"surrogate {sst['kernel_ms']:.1f} ms")
    assert sst["paths"] == est["paths"]
    assert sst["surrogate_paths"] > 0.3 * sst["paths"]
    assert np.percentile(d, 99) < 0.5
    assert np.percentile(vs_oracle, 99) <= 0.5, vs_oracle
    # a flat network refuses terrain scenes
    flat = native.Surrogate(ctx, seed=3)
    with pytest.raises(native.QmError):
        dev.paint_grid_surrogate(tile, flat)


def test_paths_inside_the_exact_radius_stay_exact(ctx, terrain):
    """A network trained with exact_within_m leaves every shorter path to the exact path: its
    eligible range starts at that length, and on a tile the network takes no path that short."""
    scene, full = terrain
    dev = ctx.scene(scene)
    net = native.Surrogate(ctx, seed=4)
    radius = 150.0
    grid = scenes.Grid(origin=(full.origin[0] + 17, full.origin[1] + 23), spacing=full.spacing * 32, nx=16, ny=16,
                       source_begin=0, source_end=20000)
    net.train(dev, [grid], epochs=2, batch=8192, learning_rate=2e-3, seed=6, max_samples=1_000_000,
              exact_within_m=radius)
    lo0 = net.params()[abi.SURR_WEIGHTS + 32 + 32 + 8 + 8]
    assert lo0 >= radius * 1e-3, lo0
    tile = scenes.Grid(origin=(full.origin[0] + 100 * full.spacing, full.origin[1] + 60 * full.spacing),
                       spacing=full.spacing, nx=16, ny=8)
    _, edba, _, _, est = dev.paint_grid(tile)
    _, sdba, _, _, sst = dev.paint_grid_surrogate(tile, net)
    # Paths shorter than the radius, counted on the host (a small margin for float rounding).
    rx = (tile.origin[0] + tile.spacing * np.arange(tile.nx))[None, :].repeat(tile.ny, 0).ravel()
    ry = (tile.origin[1] + tile.spacing * np.arange(tile.ny))[:, None].repeat(tile.nx, 1).ravel()
    sx = scene.sources["x"].astype(np.float64)
    sy = scene.sources["y"].astype(np.float64)
    short = 0
    for x, y in zip(rx, ry):
        short += int(np.count_nonzero(np.hypot((x - sx) * scene.step_m, (y - sy) * scene.step_m) < radius - 0.01))
    assert short > 0
    assert sst["surrogate_paths"] <= sst["paths"] - short, (sst["surrogate_paths"], sst["paths"], short)
    d = np.abs(sdba - edba)
    assert np.percentile(d, 99) < 0.5, np.percentile(d, [50, 99, 100])
