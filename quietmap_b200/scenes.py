"""Seeded synthetic scenes of the painter workloads (there are no real tiles on this box).

Every scene comes from one `numpy.random.default_rng(seed)` stream. Positions are lattice steps
(x east, y north) of `step_m` metres; obstacle vertices, receivers and source points are lattice
points, so crossing tests are exact integer arithmetic (the reference stores obstacle vertices
as exact integers of its lattice too: popup/src/obstacles/mod.rs:5-8).

Workloads:
- `road_square` — 1 km x 1 km, flat ground G = 0.5, homogeneous air, 400 straight roads split
  into 1 m point sources at 0.05 m, 300 rotated rectangular buildings; 128 x 128 receivers at
  7.8125 m, 4 m high.
- `terrain_square` — the 16 km^2 terrain square: 2048 x 2048 receivers at 1.953125 m, fBm DEM
  (Hurst 0.8, 5 m posts, +-40 m), Voronoi ground factor (200 cells, G in {0, 0.5, 1}), 20,000 road
  and rail segments at 1 m points, 30,000 polygon buildings of 4-12 vertices (log-normal heights,
  median 9 m, sigma 0.6), favourable probability 0.5 in every sector. `scale` shrinks the side and
  every count with the area, keeping the densities.
"""

from dataclasses import dataclass, field

import numpy as np

from . import abi
from .physics import alpha_bands

# A-weighted octave shapes (dB relative to the base level), 63 Hz .. 8 kHz: a road's rolling
# noise and a railway's, each an unweighted shape plus the A-weighting of the bands
# (physics/src/bands.rs:11).
A_WEIGHTING_DB = np.array([-26.2, -16.1, -8.6, -3.2, 0.0, 1.2, 1.0, -1.1])
ROAD_SHAPE_DB = np.array([-7.0, -6.0, -5.0, -4.0, -3.0, -5.0, -8.0, -12.0]) + A_WEIGHTING_DB
RAIL_SHAPE_DB = np.array([-9.0, -7.0, -5.0, -3.0, -2.0, -3.0, -6.0, -11.0]) + A_WEIGHTING_DB
# Evening and night emissions relative to the day (dB).
PERIOD_OFFSETS_DB = np.array([0.0, -3.0, -8.0])


@dataclass
class Scene:
    step_m: float
    cell_steps: int
    extent_steps: tuple
    vertices: np.ndarray            # [n][2] int32
    outlines: np.ndarray            # OUTLINE_DTYPE
    sources: np.ndarray             # SOURCE_DTYPE
    favourable: np.ndarray          # [3][16]
    alpha_db_per_km: np.ndarray     # [8]
    flat_altitude_m: float = 0.0
    flat_ground_factor: float = 0.5
    dem_altitude: np.ndarray = None  # [ny][nx] float32
    dem_ground_factor: np.ndarray = None
    dem_origin: tuple = (0, 0)
    dem_spacing: int = 0
    name: str = ""
    info: dict = field(default_factory=dict)


@dataclass
class Grid:
    origin: tuple
    spacing: int
    nx: int
    ny: int
    height_m: float = 4.0
    source_begin: int = 0
    source_end: int = 0
    level_min_db: float = -30.0
    bin_db: float = 0.1
    n_bins: int = 1800

    @property
    def cells(self):
        return self.nx * self.ny

    def receiver_xy(self):
        """[cells][2] lattice steps in cell order j*nx + i."""
        j, i = np.divmod(np.arange(self.cells, dtype=np.int64), self.nx)
        return np.stack([self.origin[0] + i * self.spacing, self.origin[1] + j * self.spacing], axis=1)


def _outlines(records):
    out = np.zeros(len(records), dtype=abi.OUTLINE_DTYPE)
    for k, (first, count, fp, height, building) in enumerate(records):
        out[k] = (first, count, fp, height, building)
    return out


def _rectangle(rng, centre, sides, angle):
    c, s = np.cos(angle), np.sin(angle)
    hx, hy = sides[0] / 2, sides[1] / 2
    corners = np.array([[-hx, -hy], [hx, -hy], [hx, hy], [-hx, hy]])
    rot = np.array([[c, -s], [s, c]])
    return corners @ rot.T + centre


def _convex_polygon(rng, centre, radius, n):
    angles = np.sort(rng.uniform(0, 2 * np.pi, n))
    # Spread the angles so no two vertices nearly coincide.
    angles = np.sort((angles + np.linspace(0, 2 * np.pi, n, endpoint=False)) / 2 % (2 * np.pi))
    r = radius * rng.uniform(0.75, 1.0, n)
    return centre + np.stack([r * np.cos(angles), r * np.sin(angles)], axis=1)


def _signed_area2(p):
    x, y = p[:, 0], p[:, 1]
    return float(np.sum(x * np.roll(y, -1) - np.roll(x, -1) * y))


def _place_buildings(rng, n, side_m, make, min_gap_m, margin_m):
    """Rejection-sampled non-overlapping footprints: bounding circles kept `min_gap_m` apart."""
    cell = 48.0
    grid = {}
    placed = []
    attempts = 0
    while len(placed) < n and attempts < 200 * n:
        attempts += 1
        polygon, radius = make(rng)
        centre = rng.uniform(margin_m + radius, side_m - margin_m - radius, 2)
        key = (int(centre[0] // cell), int(centre[1] // cell))
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for (oc, orad) in grid.get((key[0] + dx, key[1] + dy), ()):
                    if np.hypot(*(oc - centre)) < radius + orad + min_gap_m:
                        ok = False
                        break
                if not ok:
                    break
            if not ok:
                break
        if not ok:
            continue
        grid.setdefault(key, []).append((centre, radius))
        placed.append(polygon + centre)
    return placed


def _rings_to_arrays(polygons, heights, step_m, first_id=1):
    verts, records = [], []
    total = 0  # vertices so far: the next ring's first vertex
    for k, (poly, height) in enumerate(zip(polygons, heights)):
        pts = np.round(poly / step_m).astype(np.int64)
        # Counter-clockwise, distinct consecutive vertices, closed by repeating the first.
        keep = [pts[0]]
        for p in pts[1:]:
            if not np.array_equal(p, keep[-1]):
                keep.append(p)
        if np.array_equal(keep[-1], keep[0]) and len(keep) > 1:
            keep.pop()
        pts = np.array(keep)
        if len(pts) < 3:
            continue
        if _signed_area2(pts.astype(np.float64)) < 0:
            pts = pts[::-1]
        ring = np.vstack([pts, pts[:1]])
        records.append((total, len(ring), first_id + k, float(height), 1))
        verts.append(ring)
        total += len(ring)
    vertices = np.vstack(verts).astype(np.int32) if verts else np.zeros((0, 2), np.int32)
    return vertices, _outlines(records)


def _segments_to_points(rng, n_segments, side_m, step_m, kind_of, base_of, margin_m=1.0, origin_m=(0.0, 0.0),
                        max_points=None, kept=None):
    """Straight segments with ends uniform in the square, length clipped to [20, 200] m, split
    into 1 m point sources at their piece centres (snapped to the lattice). The square starts at
    `origin_m`; past `max_points` points no further segment is added (`kept`, a list, receives
    the count of segments kept)."""
    xs, ys, hs, energy, layers = [], [], [], [], []
    total = 0
    for k in range(n_segments):
        if max_points is not None and total >= max_points:
            break
        a = rng.uniform(margin_m, side_m - margin_m, 2)
        b = rng.uniform(margin_m, side_m - margin_m, 2)
        d = b - a
        length = float(np.hypot(*d))
        if length < 1e-9:
            d, length = np.array([1.0, 0.0]), 1.0
        target = min(max(length, 20.0), 200.0)
        b = np.clip(a + d * (target / length), margin_m, side_m - margin_m)
        d = b - a
        length = float(np.hypot(*d))
        count = max(int(round(length)), 1)
        kind = kind_of(k)
        base = base_of(kind)
        shape = ROAD_SHAPE_DB if kind == 0 else RAIL_SHAPE_DB
        levels = base + shape + rng.normal(0.0, 2.0, 8)  # per metre, A-weighted
        f = (np.arange(count) + 0.5) / count
        pts = a + f[:, None] * d + np.asarray(origin_m)
        total += count
        if kept is not None:
            kept.append(k)
        xs.append(np.round(pts[:, 0] / step_m))
        ys.append(np.round(pts[:, 1] / step_m))
        piece_m = length / count
        e_day = 10.0 ** (levels / 10.0) * piece_m
        energy.append(np.repeat(e_day[None, :], count, axis=0))
        hs.append(np.full(count, 0.05 if kind == 0 else 0.5))
        layers.append(np.full(count, kind))
    x = np.concatenate(xs).astype(np.int32)
    y = np.concatenate(ys).astype(np.int32)
    e = np.concatenate(energy)
    src = np.zeros(len(x), dtype=abi.SOURCE_DTYPE)
    src["x"], src["y"] = x, y
    src["height_m"] = np.concatenate(hs)
    src["ground_factor"] = -1.0
    src["layer"] = np.concatenate(layers)
    for p in range(abi.PERIODS):
        src["energy"][:, p, :] = e * 10.0 ** (PERIOD_OFFSETS_DB[p] / 10.0)
    return src


def road_square(seed=1, n_roads=400, n_buildings=300, side_m=1000.0, receivers=128,
                cell_steps=1024):
    """The plain CNOSSOS road painter: flat G = 0.5, homogeneous conditions, 15 C / 70 %."""
    rng = np.random.default_rng(seed)
    step_m = 1.0 / 32.0
    extent = int(round(side_m / step_m))

    def rect(rng):
        sides = rng.uniform(8.0, 40.0, 2)
        poly = _rectangle(rng, np.zeros(2), sides, rng.uniform(0, np.pi))
        return poly, float(np.hypot(*sides) / 2)

    polys = _place_buildings(rng, n_buildings, side_m, rect, 1.0, 1.0)
    heights = rng.uniform(3.0, 30.0, len(polys))
    vertices, outlines = _rings_to_arrays(polys, heights, step_m)
    sources = _segments_to_points(rng, n_roads, side_m, step_m, lambda k: 0,
                                  lambda kind: rng.uniform(70.0, 100.0))
    scene = Scene(step_m=step_m, cell_steps=cell_steps, extent_steps=(extent, extent),
                  vertices=vertices, outlines=outlines, sources=sources,
                  favourable=np.zeros((3, 16)), alpha_db_per_km=alpha_bands(15.0, 70.0),
                  flat_altitude_m=0.0, flat_ground_factor=0.5, name="road_square",
                  info=dict(seed=seed, side_m=side_m, roads=n_roads, buildings=len(polys)))
    spacing = extent // receivers
    grid = Grid(origin=(spacing // 2, spacing // 2), spacing=spacing, nx=receivers, ny=receivers)
    return scene, grid


def fbm_dem(rng, n, hurst, relief_m):
    """Fractional Brownian surface by spectral synthesis: amplitude ~ k^-(H+1), scaled to
    +-relief_m."""
    size = 1 << int(np.ceil(np.log2(n)))
    kx = np.fft.fftfreq(size)[:, None]
    ky = np.fft.fftfreq(size)[None, :]
    k = np.sqrt(kx * kx + ky * ky)
    k[0, 0] = 1.0
    amplitude = k ** (-(hurst + 1.0))
    amplitude[0, 0] = 0.0
    phase = rng.uniform(0, 2 * np.pi, (size, size))
    field_ = np.real(np.fft.ifft2(amplitude * np.exp(1j * phase)))[:n, :n]
    field_ -= field_.mean()
    field_ *= relief_m / np.max(np.abs(field_))
    return field_.astype(np.float32)


def voronoi_ground(rng, n, cells, spacing_m):
    sites = rng.uniform(0, (n - 1) * spacing_m, (cells, 2))
    values = rng.choice(np.array([0.0, 0.5, 1.0]), cells)
    ys, xs = np.mgrid[0:n, 0:n].astype(np.float64) * spacing_m
    out = np.empty((n, n), np.float32)
    # Nearest site, row by row (n x cells each).
    for j in range(n):
        d = (xs[j][:, None] - sites[None, :, 0]) ** 2 + (ys[j][:, None] - sites[None, :, 1]) ** 2
        out[j] = values[np.argmin(d, axis=1)]
    return out


def terrain_square(seed=2, scale=1.0, n_segments=20000, n_buildings=30000, side_m=4000.0,
                   receivers=2048, cell_steps=1024, rail_share=0.2):
    """The exact painter on terrain. `scale` (0 < scale <= 1) multiplies the square's side and
    the receiver count per axis, and the segment, building and ground-cell counts by scale^2."""
    rng = np.random.default_rng(seed)
    step_m = 1.0 / 64.0
    side = side_m * scale
    area = scale * scale
    n_segments = max(int(round(n_segments * area)), 1)
    n_buildings = max(int(round(n_buildings * area)), 1)
    receivers = max(int(round(receivers * scale)), 2)
    extent = int(round(side / step_m))
    dem_spacing_m = 5.0
    nodes = int(round(side / dem_spacing_m)) + 1
    dem = fbm_dem(rng, nodes, 0.8, 40.0)
    gf = voronoi_ground(rng, nodes, max(int(round(200 * area)), 2), dem_spacing_m)

    def poly(rng):
        n = int(rng.integers(4, 13))
        radius = float(rng.uniform(4.0, 11.0))
        return _convex_polygon(rng, np.zeros(2), radius, n), radius

    polys = _place_buildings(rng, n_buildings, side, poly, 1.0, 1.0)
    heights = rng.lognormal(np.log(9.0), 0.6, len(polys))
    vertices, outlines = _rings_to_arrays(polys, heights, step_m)
    rail_cut = int(round(n_segments * (1.0 - rail_share)))
    sources = _segments_to_points(
        rng, n_segments, side, step_m, lambda k: 0 if k < rail_cut else 1,
        lambda kind: rng.uniform(70.0, 100.0) if kind == 0 else rng.uniform(80.0, 105.0))
    scene = Scene(step_m=step_m, cell_steps=cell_steps, extent_steps=(extent, extent),
                  vertices=vertices, outlines=outlines, sources=sources,
                  favourable=np.full((3, 16), 0.5), alpha_db_per_km=alpha_bands(15.0, 70.0),
                  dem_altitude=dem, dem_ground_factor=gf, dem_origin=(0, 0),
                  dem_spacing=int(round(dem_spacing_m / step_m)), name="terrain_square",
                  info=dict(seed=seed, scale=scale, side_m=side, segments=n_segments,
                            buildings=len(polys)))
    spacing = int(round(side / receivers / step_m))
    grid = Grid(origin=(spacing // 2, spacing // 2), spacing=spacing, nx=receivers, ny=receivers)
    return scene, grid


def terrain_tile_steps(full, n_sources, seed=1000, tiles=8, slices=8, tile=(16, 8)):
    """Seeded receiver tiles of the terrain square's grid, each painted against the source list in
    `slices` consecutive slices: a list of Grids, tile after tile, slice after slice. Painting the
    whole square is ~10^13 paths; these tiles are the sample a timing step paints."""
    tile_w, tile_h = tile
    per = (n_sources + slices - 1) // slices
    rng = np.random.default_rng(seed)
    steps = []
    for _ in range(tiles):
        tx = int(rng.integers(0, full.nx // tile_w))
        ty = int(rng.integers(0, full.ny // tile_h))
        for s in range(slices):
            b, e = s * per, min((s + 1) * per, n_sources)
            if b >= e:
                continue
            steps.append(Grid(origin=(full.origin[0] + tx * tile_w * full.spacing,
                                      full.origin[1] + ty * tile_h * full.spacing),
                              spacing=full.spacing, nx=tile_w, ny=tile_h, source_begin=b, source_end=e))
    return steps


# ---------------------------------------------------------------------------------------------
# Aircraft: Doc 29 flights over a receiver grid.

NPD_DISTANCES_FT = np.array([200.0, 400.0, 630.0, 1000.0, 2000.0, 4000.0, 6300.0, 10000.0, 16000.0, 25000.0])


@dataclass
class FlightScene:
    types: np.ndarray       # AIRCRAFT_TYPE_DTYPE
    segments: np.ndarray    # FLIGHT_SEGMENT_DTYPE
    grid: dict              # origin_m, spacing_m, nx, ny, receiver_height_m, reach_m, duration_s
    epnl_db: np.ndarray = None  # [types][2][10][10] EPNL-like curves (the NPD's third metric)
    la_db: np.ndarray = None    # [types][2][10][10] LA curves (the fourth)
    info: dict = field(default_factory=dict)


def flights_square(seed=3, n_flights=2000, segments_per_flight=50, n_types=10, receivers=1024, spacing_m=100.0,
                   segment_m=1000.0, reach_m=25000.0):
    """Doc 29 aircraft: `n_flights` 3D polyline tracks of `segments_per_flight` segments (departures
    climbing from 0 to up to 3000 m, approaches descending, 70-250 m/s), `n_types` types with seeded
    NPD tables (10 powers x 10 distances x 4 metrics, monotone: ~ -20 lg d - 0.005 dB/m) and 28-band
    spectra, over `receivers`^2 cells at `spacing_m`."""
    from . import abi
    rng = np.random.default_rng(seed)
    side = receivers * spacing_m
    d_m = NPD_DISTANCES_FT * 0.3048
    types = np.zeros(n_types, dtype=abi.AIRCRAFT_TYPE_DTYPE)
    epnl = np.zeros((n_types, 2, 10, 10), np.float32)
    la = np.zeros((n_types, 2, 10, 10), np.float32)
    bands = np.arange(28)
    for t in range(n_types):
        base = rng.uniform(85.0, 100.0)
        for op in range(2):
            for r in range(10):
                level0 = base + (1.4 * r if op == 1 else 0.8 * r) - (4.0 if op == 0 else 0.0)
                sel = level0 - 20.0 * np.log10(d_m / d_m[0]) - 0.005 * (d_m - d_m[0]) + rng.normal(0, 0.15, 10)
                sel = np.minimum.accumulate(sel)  # monotone decreasing in distance
                duration = 6.0 + 3.0 * np.log10(d_m / d_m[0]) + rng.uniform(-0.5, 0.5)
                types[t]["sel_db"][op, r] = sel
                types[t]["lamax_db"][op, r] = sel - duration
                epnl[t, op, r] = sel + 2.0
                la[t, op, r] = sel - duration - 2.0
        types[t]["v_ref_kt"] = rng.uniform(140.0, 180.0)
        types[t]["installation"] = rng.integers(0, 3)
        peak = rng.uniform(12.0, 18.0)
        types[t]["spectrum_db"] = -0.35 * (bands - peak) ** 2 / 4.0 + rng.normal(0, 1.0, 28)
    segs = np.zeros(n_flights * segments_per_flight, dtype=abi.FLIGHT_SEGMENT_DTYPE)
    k = 0
    for f in range(n_flights):
        departure = int(rng.integers(0, 2))
        ty = int(rng.integers(0, n_types))
        p = rng.uniform(0.1 * side, 0.9 * side, 2)
        heading = rng.uniform(0, 2 * np.pi)
        top = rng.uniform(1500.0, 3000.0)
        v0, v1 = (rng.uniform(70.0, 100.0), rng.uniform(180.0, 250.0))
        z = 0.0 if departure else top
        for s in range(segments_per_flight):
            heading += rng.normal(0.0, 0.05)
            q = p + segment_m * np.array([np.cos(heading), np.sin(heading)])
            frac = (s + 1) / segments_per_flight
            z1 = top * min(frac * 2.0, 1.0) if departure else top * max(1.0 - frac * 2.0, 0.0)
            segs[k]["start"] = (p[0], p[1], z)
            segs[k]["end"] = (q[0], q[1], z1)
            power = (9.0 - 6.0 * frac) if departure else (2.0 + 1.0 * (1.0 - frac))
            segs[k]["power"] = np.clip(power + rng.normal(0, 0.2), 0.0, 9.0)
            segs[k]["speed_mps"] = v0 + (v1 - v0) * (frac if departure else 1.0 - frac)
            segs[k]["type"] = ty
            segs[k]["departure"] = departure
            segs[k]["flight"] = f
            p, z = q, z1
            k += 1
    grid = dict(origin_m=(spacing_m / 2, spacing_m / 2), spacing_m=spacing_m, nx=receivers, ny=receivers,
                receiver_height_m=4.0, reach_m=reach_m, duration_s=86400.0)
    return FlightScene(types=types, segments=segs, grid=grid, epnl_db=epnl, la_db=la,
                       info=dict(seed=seed, flights=n_flights, types=n_types))


# ---------------------------------------------------------------------------------------------
# Aircraft boxes: the flights of a square summed into boxes, and lattice points asking for them.

TAIL_ANCHOR_M = 16000.0
FINE_BOXES_WITHIN_M = 3000.0


def _row_energies(types):
    """Per type, operation and power row: SEL at the ten NPD distances, d_lambda there and the SEL
    at the tail anchor (the NPD curve beyond 25,000 ft falls by spherical spreading and the
    absorption fitted to its last three distances)."""
    d = NPD_DISTANCES_FT * 0.3048
    last = d[-1]
    sel = types["sel_db"].astype(np.float64)                      # [t][2][10][10]
    sml = sel - types["lamax_db"].astype(np.float64)
    v = types["v_ref_kt"].astype(np.float64) * 1852.0 / 3600.0
    d0 = (2.0 / np.pi * v)[:, None, None, None]
    scaled = d0 * 10.0 ** (sml / 10.0)
    y = sel[..., -3:] + 20.0 * np.log10(d[-3:] / last)
    x = d[-3:] - d[-3:].mean()
    slope = (x * (y - y.mean(axis=-1, keepdims=True))).sum(-1) / (x * x).sum()
    alpha = np.maximum(-slope, 0.0)
    tail = sel[..., -1] - 20.0 * np.log10(TAIL_ANCHOR_M / last) - alpha * (TAIL_ANCHOR_M - last)
    return sel, scaled, tail


def _cell_boxes(pieces, cell_m, slab_m, n_flights):
    """BoxSums of the pieces by their cells (physics/src/doc29/box_sums.rs:82-199 in numpy)."""
    mid = 0.5 * (pieces["start"] + pieces["end"])
    ix = np.floor(mid[:, 0] / cell_m).astype(np.int64)
    iy = np.floor(mid[:, 1] / cell_m).astype(np.int64)
    iz = np.floor(mid[:, 2] / slab_m).astype(np.int64)
    key = (ix + (1 << 20)) * (1 << 40) + (iy + (1 << 20)) * (1 << 20) + iz
    keys, inv = np.unique(key, return_inverse=True)
    nb = len(keys)
    add = lambda w: np.bincount(inv, weights=w, minlength=nb)
    pw = pieces["period_weights"]                                   # [n][3]
    E = pieces["energy"]                                            # [n][10]
    energy = np.stack([np.stack([add(pw[:, p] * E[:, k]) for k in range(10)], 1) for p in range(3)], 1)
    tail = np.stack([add(pw[:, p] * pieces["tail"]) for p in range(3)], 1)
    total = pw.sum(1)
    over = np.stack([add(total * E[:, k] / np.maximum(pieces["scaled"][:, k], 1.0)) for k in range(10)], 1)
    w = total * E[:, 3]
    delta = pieces["end"] - pieces["start"]
    length = np.hypot(delta[:, 0], delta[:, 1])
    weight = add(w)
    midpoint = np.stack([add(w * mid[:, a]) for a in range(3)], 1)
    period_weight = np.stack([add(pw[:, p] * E[:, 3]) for p in range(3)], 1)
    period_length = np.stack([add(pw[:, p] * E[:, 3] * length) for p in range(3)], 1)
    safe = np.maximum(length, 1e-300)
    c, s_, g = delta[:, 0] / safe, delta[:, 1] / safe, delta[:, 2] / safe
    on = length > 0.0
    dd = np.stack([add(np.where(on, w * (c * c - s_ * s_), 0.0)), add(np.where(on, w * 2.0 * s_ * c, 0.0))], 1)
    gd = np.stack([add(np.where(on, w * g * c, 0.0)), add(np.where(on, w * g * s_, 0.0))], 1)
    sq = w * g * g
    sg = np.stack([add(np.where(on, sq * c * c, 0.0)), add(np.where(on, sq * s_ * s_, 0.0)),
                   add(np.where(on, sq * s_ * c, 0.0))], 1)
    inst = np.zeros((nb, 3, 2, 3))
    for slot in range(3):
        mine = pieces["installation"] == slot
        for p in range(3):
            inst[:, p, 0, slot] = add(np.where(mine, pw[:, p] * E[:, 3], 0.0))
            inst[:, p, 1, slot] = add(np.where(mine, pw[:, p] * pieces["tail"], 0.0))
    out = np.zeros(nb, dtype=abi.FLIGHT_BOX_DTYPE)
    with np.errstate(divide="ignore"):
        out["levels_db"] = np.where(energy > 0.0, 10.0 * np.log10(np.maximum(energy, 1e-300)), -np.inf)
        out["tail_levels_db"] = np.where(tail > 0.0, 10.0 * np.log10(np.maximum(tail, 1e-300)), -np.inf)
    out["lg_scaled_distance"] = np.log10(energy.sum(1) / over)
    axis = np.mod(0.5 * np.arctan2(dd[:, 1], dd[:, 0]), np.pi)
    sa, ca = np.sin(axis), np.cos(axis)
    gradient = (gd[:, 0] * ca + gd[:, 1] * sa) / weight
    mean_square = (sg[:, 0] * ca * ca + sg[:, 1] * sa * sa + 2.0 * sg[:, 2] * sa * ca) / weight
    out["east_m"], out["north_m"], out["centroid_altitude_m"] = (midpoint / weight[:, None]).T
    out["axis_rad"], out["gradient"] = axis, gradient
    out["gradient_spread"] = np.sqrt(np.maximum(mean_square - gradient * gradient, 0.0))
    out["piece_length_m"] = np.where(period_weight > 0.0, period_length / np.maximum(period_weight, 1e-300), 0.0)
    tot = inst.sum(-1, keepdims=True)
    out["installation_shares"] = np.where(tot > 0.0, inst / np.maximum(tot, 1e-300), np.array([0.0, 0.0, 1.0]))
    # popup/src/aircraft/boxes.rs:225-266 box_passing: flights a day in the box over the period's seconds,
    # times the cell's mean chord along the box's axis over the pieces' mean speed.
    flight_key = inv.astype(np.int64) * n_flights + pieces["flight"]
    _, first = np.unique(flight_key, return_index=True)
    per_day = np.stack([np.bincount(inv[first], weights=pw[first, p], minlength=nb) for p in range(3)], 1)
    up = slab_m
    shadow = np.abs(ca) * cell_m * up + np.abs(sa) * cell_m * up
    spread = out["gradient_spread"]
    chord = 0.5 * sum(cell_m * cell_m * up / (shadow + np.abs(gradient + side * spread) * cell_m * cell_m)
                      for side in (-1.0, 1.0))
    seconds_per_metre = add(1.0 / pieces["speed_mps"]) / np.bincount(inv, minlength=nb)
    hours = np.array([12.0, 4.0, 8.0])
    out["passing"] = per_day / (hours * 3600.0) * (chord * seconds_per_metre)[:, None]
    return out


@dataclass
class FlightBoxScene:
    boxes: np.ndarray        # FLIGHT_BOX_DTYPE, grouped by aircraft tile and file (fine, far)
    tile_ranges: np.ndarray  # [tiles][2 files] (first, count) into boxes
    tile_m: float
    tiles_side: int
    side_m: float
    info: dict = field(default_factory=dict)


def flight_boxes_square(seed=3, n_flights=2000, segments_per_flight=50, receivers=1024, spacing_m=100.0,
                        tile_m=6400.0, fine_m=400.0, fine_slab_m=150.0, far_m=1600.0, far_slab_m=600.0,
                        helicopter_share=0.03):
    """The aircraft boxes of the flight workload's square (`flights_square`: its flights and NPD
    tables): each segment cut into pieces of at most half a cell, each piece's energies at the NPD
    distances and tail anchor, every piece summed into its fine cell (fine_m, fine_slab_m) and its far
    cell (far_m, far_slab_m) as the builder sums a box, flights flown by day, evening or night
    (70/15/15 %), the boxes grouped by aircraft tile (tile_m) and file. A share of the boxes is
    marked as helicopters'."""
    f = flights_square(seed=seed, n_flights=n_flights, segments_per_flight=segments_per_flight, receivers=receivers,
                       spacing_m=spacing_m)
    rng = np.random.default_rng(seed + 101)
    segs = f.segments
    sel, scaled, tail = _row_energies(f.types)
    t, op = segs["type"].astype(np.int64), segs["departure"].astype(np.int64)
    power = segs["power"].astype(np.float64)
    row = np.minimum(np.floor(power).astype(np.int64), 8)
    w = (power - row)[:, None]
    lerp = lambda a: a[t, op, row] + w * (a[t, op, row + 1] - a[t, op, row])
    v_ref = f.types["v_ref_kt"].astype(np.float64)[t]
    speed_kt = segs["speed_mps"].astype(np.float64) * 3600.0 / 1852.0
    dv = np.where(speed_kt > 10.0, 10.0 * np.log10(v_ref / np.maximum(speed_kt, 1e-9)), 0.0)
    seg_sel = lerp(sel) + dv[:, None]
    seg_scaled = lerp(scaled)
    seg_tail = (lerp(tail[..., None])[:, 0]) + dv
    period_of_flight = rng.choice(3, size=n_flights, p=[0.7, 0.15, 0.15])
    start, end = segs["start"].astype(np.float64), segs["end"].astype(np.float64)
    hlen = np.hypot(*(end - start)[:, :2].T)
    out = []
    for cell, slab in ((fine_m, fine_slab_m), (far_m, far_slab_m)):
        n_sub = np.maximum(1, np.ceil(hlen / (0.5 * cell))).astype(np.int64)
        owner = np.repeat(np.arange(len(segs)), n_sub)
        k = np.arange(len(owner)) - np.repeat(np.cumsum(n_sub) - n_sub, n_sub)
        a0, a1 = (k / n_sub[owner])[:, None], ((k + 1) / n_sub[owner])[:, None]
        d = end[owner] - start[owner]
        pieces = dict(start=start[owner] + a0 * d, end=start[owner] + a1 * d, energy=10.0 ** (seg_sel[owner] / 10.0),
                      tail=10.0 ** (seg_tail[owner] / 10.0), scaled=seg_scaled[owner],
                      installation=f.types["installation"].astype(np.int64)[t[owner]],
                      flight=segs["flight"].astype(np.int64)[owner], speed_mps=segs["speed_mps"].astype(np.float64)[owner])
        pw = np.zeros((len(owner), 3))
        pw[np.arange(len(owner)), period_of_flight[pieces["flight"]]] = 1.0
        pieces["period_weights"] = pw
        out.append(_cell_boxes(pieces, cell, slab, n_flights))
    side = receivers * spacing_m
    tiles_side = int(np.ceil(side / tile_m))
    groups, ranges = [], np.zeros((tiles_side * tiles_side, 2, 2), np.int64)
    for file, boxes in enumerate(out):
        tx = np.clip(np.floor(boxes["east_m"] / tile_m).astype(np.int64), 0, tiles_side - 1)
        ty = np.clip(np.floor(boxes["north_m"] / tile_m).astype(np.int64), 0, tiles_side - 1)
        boxes["helicopter"] = rng.random(len(boxes)) < helicopter_share
        groups.append((ty * tiles_side + tx, file, boxes))
    ordered, at = [], 0
    for tile in range(tiles_side * tiles_side):
        for tiles, file, boxes in groups:
            mine = boxes[tiles == tile]
            ranges[tile, file] = (at, len(mine))
            ordered.append(mine)
            at += len(mine)
    all_boxes = np.concatenate(ordered)
    return FlightBoxScene(boxes=all_boxes, tile_ranges=ranges, tile_m=tile_m, tiles_side=tiles_side, side_m=side,
                          info=dict(seed=seed, flights=n_flights, fine_boxes=len(out[0]), far_boxes=len(out[1])))


def synthetic_horizons(n, seed=5):
    """`n` points' horizons as the card keeps them (popup/src/aircraft/horizons.rs:50-64): gentle
    terrain (tangents -0.03..0.06 in 32 sectors x 6 bands of 30 m - 8 km, a fifth of the bands empty)
    and an urban building horizon (256 sectors x 6 bands of 16-512 m, tangents 0..0.6, half empty)."""
    rng = np.random.default_rng(seed)
    bands = abi.HORIZON_BANDS

    def one(sectors, limits, lo, hi, empty):
        edges = np.empty((n, sectors, bands, 2), np.float32)
        inner = np.concatenate([[limits[0] * 0.25], limits[:-1]])
        edges[..., 0] = rng.uniform(inner, limits, (n, sectors, bands))
        edges[..., 1] = rng.uniform(lo, hi, (n, sectors, bands))
        blank = rng.random((n, sectors, bands)) < empty
        edges[..., 0][blank] = np.nan
        tang = np.where(blank, -np.inf, edges[..., 1])
        steepest = tang.max(-1)
        out = np.empty((n, 1 + sectors * (1 + 2 * bands)), np.float32)
        out[:, 0] = steepest.max(-1)
        per = out[:, 1:].reshape(n, sectors, 1 + 2 * bands)
        per[:, :, 0] = steepest
        per[:, :, 1:] = edges.reshape(n, sectors, 2 * bands)
        return out

    terrain = one(abi.TERRAIN_SECTORS, np.array([500.0, 1000.0, 2000.0, 3500.0, 5500.0, 8000.0]), -0.03, 0.06, 0.2)
    buildings = one(abi.BUILDING_SECTORS, np.array([16.0, 32.0, 64.0, 128.0, 256.0, 512.0]), 0.0, 0.6, 0.5)
    return np.concatenate([terrain, buildings], 1).reshape(-1)


def flight_requests(world, points_xy, altitude_m=4.0, weights=(abi.FLIGHT_WEIGHT_ONE, None), within_m=16000.0,
                    coarse_m=0.0, impedance_gain=1.0, horizons=True, seed=5):
    """Lattice points asking for the square's boxes (paint/src/flights.rs:84-107 tiles_heard and
    paint-gpu/src/aircraft.rs:245-290): per point and band with a weight, a segment per aircraft tile
    within `within_m` of it, its fine boxes within 3 km and its far boxes beyond. Returns (points,
    horizons or None, segments, n_sums): sums 2 k + band for point k."""
    pts = np.asarray(points_xy, dtype=np.float64).reshape(-1, 2)
    n = len(pts)
    points = np.zeros(n, dtype=abi.FLIGHT_POINT_DTYPE)
    points["x"], points["y"] = pts[:, 0], pts[:, 1]
    points["altitude_m"] = altitude_m
    points["impedance_gain"] = impedance_gain
    points["horizons"] = np.arange(n, dtype=np.uint64) * abi.HORIZON_FLOATS
    hz = synthetic_horizons(n, seed) if horizons else None
    side, tm = world.tiles_side, world.tile_m
    tx, ty = np.meshgrid(np.arange(side), np.arange(side))
    lo_x, lo_y = (tx.ravel() * tm), (ty.ravel() * tm)
    segs = []
    for k in range(n):
        gx = np.maximum(np.maximum(lo_x - pts[k, 0], 0.0), pts[k, 0] - (lo_x + tm))
        gy = np.maximum(np.maximum(lo_y - pts[k, 1], 0.0), pts[k, 1] - (lo_y + tm))
        gap = np.hypot(gx, gy)
        for tile in np.nonzero(gap <= within_m)[0]:
            file = 0 if gap[tile] <= FINE_BOXES_WITHIN_M and world.tile_ranges[tile, 0, 1] else 1
            first, count = world.tile_ranges[tile, file]
            if count == 0:
                continue
            for band, weight in enumerate(weights):
                if weight is None:
                    continue
                segs.append((within_m, coarse_m, k, 2 * k + band, first, count, weight, 0))
    segments = np.array(segs, dtype=abi.BOX_SEGMENT_DTYPE) if segs else np.zeros(0, dtype=abi.BOX_SEGMENT_DTYPE)
    return points, hz, segments, 2 * n


# ---------------------------------------------------------------------------------------------
# Batches of uneven tiles.

def tiles_world():
    """The world tile batches are cut from: the config-1 road square (1 km, 400 roads as 1 m point
    sources, 300 buildings, flat G = 0.5, homogeneous)."""
    return road_square()[0]


def uneven_tiles(scene, n_tiles=4096, seed=5, side=(32, 512), sources=(10, 50000), spacing_steps=60):
    """`n_tiles` receiver tiles with sides (nx, ny) log-uniform in `side` receivers at
    `spacing_steps` lattice steps, each with a contiguous range of the scene's sources whose
    length is log-uniform in `sources`, at seeded positions inside the scene. Cells are numbered
    tile after tile."""
    rng = np.random.default_rng(seed)
    extent = scene.extent_steps[0]
    n_src = len(scene.sources)
    out, offset = [], 0
    for _ in range(n_tiles):
        nx, ny = (int(round(np.exp(rng.uniform(np.log(side[0]), np.log(side[1]))))) for _ in range(2))
        nx, ny = min(nx, (extent - 1) // spacing_steps), min(ny, (extent - 1) // spacing_steps)
        ox = int(rng.integers(0, extent - (nx - 1) * spacing_steps))
        oy = int(rng.integers(0, extent - (ny - 1) * spacing_steps))
        k = int(round(np.exp(rng.uniform(np.log(sources[0]), np.log(sources[1])))))
        k = max(1, min(k, n_src))
        b = int(rng.integers(0, n_src - k + 1))
        out.append(dict(origin=(ox, oy), spacing=spacing_steps, nx=nx, ny=ny, height_m=4.0, source_begin=b,
                        source_end=b + k, cell_offset=offset))
        offset += nx * ny
    return out


# ---------------------------------------------------------------------------------------------
# Packed pixels for Batch::loudness.

PACKED_LINE_FLOATS = 43


def loudness_pixels(n, seed=11, layers=6, profiles=12):
    """`n` seeded packed pixels in the reference's format (paint/src/sone.rs:32-51, 217-234): per
    layer its steady energy per period, its line count and its 43-float lines (energy per period,
    means per period and weather state, lambda per period, hourly profile or -1, duty per period or
    NaN, passes in progress per period or NaN), then each layer's curves and the place's (28
    third-octave levels at an A-weighted 0 dB per period, NaN: no shape). Lines mix roads at mean
    flow, profiled roads, events and streams of passes; energies span 20-70 dB. Returns (pixels as
    float32 arrays, hourly shares [profiles][24], the map's runs per period)."""
    rng = np.random.default_rng(seed)
    shares = rng.uniform(0.3, 9.0, (profiles, 24))
    out = []
    for _ in range(n):
        f = []
        for layer in range(layers):
            count = int(rng.integers(0, 5))
            f += list(10.0 ** rng.uniform(0.0, 6.0, 3)) + [float(count)]
            for _ in range(count):
                kind = int(rng.integers(0, 4))
                f += list(10.0 ** rng.uniform(2.0, 7.0, 3))
                f += list(10.0 ** rng.uniform(2.0, 7.0, 30))
                f += list(10.0 ** rng.uniform(-3.0, 3.0, 3))
                f.append(-1.0 if kind == 0 else float(rng.integers(0, profiles)))
                f += list(rng.uniform(0.0, 0.3, 3)) if kind == 1 else [np.nan] * 3
                f += list(rng.uniform(0.0, 5.0, 3)) if kind == 2 else [np.nan] * 3
        for _ in range(layers + 1):
            for _ in range(3):
                f += [np.nan] * 28 if rng.random() < 0.2 else list(rng.uniform(-60.0, 5.0, 28))
        out.append(np.array(f, dtype=np.float32))
    return out, shares, [4, 1, 3]


# ---------------------------------------------------------------------------------------------
# Uneven tiles, each with its own buildings and roads.

TILE_SPACING_M = 7.8125  # the receivers' spacing of the road square


def uneven_tile_specs(n_tiles=4096, seed=5, side=(32, 512), segments=(10, 50000), buildings=(0, 20000)):
    """Per tile of a batch: receivers nx x ny (each side log-uniform in `side`), its count of road
    segments (log-uniform in `segments`) and of buildings (log-uniform over 1 .. buildings[1] + 1,
    less one, so 0 occurs), and its own seed. Cheap: a tile's geometry is drawn only when a batch
    holding it is built (`uneven_tile_world`)."""
    rng = np.random.default_rng(seed)
    lu = lambda lo, hi: float(np.exp(rng.uniform(np.log(lo), np.log(hi))))
    out = []
    for _ in range(n_tiles):
        nx, ny = int(round(lu(*side))), int(round(lu(*side)))
        n_seg = int(round(lu(*segments)))
        n_b = int(round(lu(buildings[0] + 1, buildings[1] + 1))) - 1
        out.append(dict(nx=nx, ny=ny, segments=n_seg, buildings=n_b, seed=int(rng.integers(0, 2**31))))
    return out


def _tile_region_m(spec):
    """A tile's square region: its receivers with 100 m around them, widened so that its buildings
    (config-1 rectangles, 8-40 m sides) cover about a quarter of it."""
    rec = (max(spec["nx"], spec["ny"]) - 1) * TILE_SPACING_M + 200.0
    return max(rec, float(np.sqrt(spec["buildings"])) * 48.0)


def uneven_tile_world(specs, max_paths_per_tile=1 << 28, step_m=1.0 / 32.0, cell_steps=1024):
    """One scene holding each tile of `specs` in a square region of its own (on a grid of regions
    the size of the largest, 200 m apart), drawn from the tile's seed as the road square is drawn:
    its buildings (rotated rectangles, sides 8-40 m, heights 3-30 m, apart by rejection) and its
    roads (ends uniform in the region, length clipped to 20-200 m, 1 m points at 0.05 m, base
    level 70-100 dB plus the road tilt and N(0, 2 dB) a band); flat G = 0.5, homogeneous air. A
    tile's receivers stand at 7.8125 m in the middle of its region and hear only its own sources
    (a contiguous range). A tile whose cells x points would pass `max_paths_per_tile` keeps its
    first roads up to that bound (independent draws, so a prefix is a sample of them). Returns
    (scene, tiles as dicts for BatchPlan, each with `kept_segments`)."""
    regions = [_tile_region_m(sp) for sp in specs]
    # Regions start on whole lattice steps, so a tile's geometry on the lattice is the same wherever
    # its region lies.
    cellm = float(np.ceil((max(regions) + 200.0) / step_m)) * step_m
    cols = int(np.ceil(np.sqrt(len(specs))))
    rows = (len(specs) + cols - 1) // cols
    spacing = int(round(TILE_SPACING_M / step_m))

    def rect(rng):
        sides = rng.uniform(8.0, 40.0, 2)
        return _rectangle(rng, np.zeros(2), sides, rng.uniform(0, np.pi)), float(np.hypot(*sides) / 2)
    verts, outls, srcs, tiles = [], [], [], []
    n_vert = n_src = cell_offset = 0
    first_id = 1
    for k, sp in enumerate(specs):
        rng = np.random.default_rng(sp["seed"])
        side = regions[k]
        ox, oy = 100.0 + (k % cols) * cellm, 100.0 + (k // cols) * cellm
        polys = _place_buildings(rng, sp["buildings"], side, rect, 1.0, 1.0)
        heights = rng.uniform(3.0, 30.0, len(polys))
        v, o = _rings_to_arrays([p + np.array([ox, oy]) for p in polys], heights, step_m, first_id=first_id)
        first_id += len(polys)
        o["first_vertex"] += n_vert
        n_vert += len(v)
        verts.append(v)
        outls.append(o)
        cells = sp["nx"] * sp["ny"]
        kept = []
        src = _segments_to_points(rng, sp["segments"], side, step_m, lambda i: 0, lambda kind: rng.uniform(70.0, 100.0),
                                  origin_m=(ox, oy), max_points=max(1, max_paths_per_tile // cells), kept=kept)
        srcs.append(src)
        rx0 = ox + side / 2 - (sp["nx"] - 1) * TILE_SPACING_M / 2
        ry0 = oy + side / 2 - (sp["ny"] - 1) * TILE_SPACING_M / 2
        tiles.append(dict(origin=(int(round(rx0 / step_m)), int(round(ry0 / step_m))), spacing=spacing, nx=sp["nx"],
                          ny=sp["ny"], height_m=4.0, source_begin=n_src, source_end=n_src + len(src),
                          cell_offset=cell_offset, kept_segments=len(kept), buildings=len(polys)))
        n_src += len(src)
        cell_offset += cells
    extent = int(round((max(cols, rows) * cellm + 200.0) / step_m))
    vertices = np.concatenate(verts) if verts else np.zeros((0, 2), np.int32)
    scene = Scene(step_m=step_m, cell_steps=cell_steps, extent_steps=(extent, extent), vertices=vertices,
                  outlines=np.concatenate(outls), sources=np.concatenate(srcs), favourable=np.zeros((3, 16)),
                  alpha_db_per_km=alpha_bands(15.0, 70.0), flat_altitude_m=0.0, flat_ground_factor=0.5,
                  name="uneven_tile_world", info=dict(tiles=len(specs)))
    return scene, tiles
