"""Small hand-built scenes for edge-case tests (buildings and walls in metres)."""

import numpy as np

from quietmap_b200 import abi
from quietmap_b200.physics import alpha_bands
from quietmap_b200.scenes import Scene


class Stock:
    """Buildings and walls placed in metres on a lattice of `step_m`, inside a square of
    `side_m` whose origin is shifted by `offset_m` so negative test coordinates fit."""

    def __init__(self, step_m=1.0 / 32.0, side_m=12000.0, offset_m=6000.0, cell_steps=256):
        self.step_m, self.side_m, self.offset_m, self.cell_steps = step_m, side_m, offset_m, cell_steps
        self.verts, self.records = [], []

    def steps(self, xy):
        return np.round((np.asarray(xy, dtype=np.float64) + self.offset_m) / self.step_m).astype(np.int64)

    def snapped(self, xy):
        return self.steps(xy)

    def _add(self, points, fp, height, building, close):
        pts = [tuple(self.steps(p)) for p in points]
        if close:
            pts = pts + [pts[0]]
        first = sum(len(v) for v in self.verts)
        self.verts.append(pts)
        self.records.append((first, len(pts), fp, height, 1 if building else 0))

    def building(self, fp, height, rings):
        for ring in rings:
            self._add(ring, fp, height, True, True)

    def wall(self, fp, height, points):
        self._add(points, fp, height, False, False)

    def scene(self, sources=None, favourable=0.0, flat_ground_factor=0.5):
        vertices = np.array([p for v in self.verts for p in v], dtype=np.int32).reshape(-1, 2)
        outlines = np.zeros(len(self.records), dtype=abi.OUTLINE_DTYPE)
        for k, r in enumerate(self.records):
            outlines[k] = r
        if sources is None:
            sources = np.zeros(0, dtype=abi.SOURCE_DTYPE)
        extent = int(round(self.side_m / self.step_m))
        return Scene(step_m=self.step_m, cell_steps=self.cell_steps, extent_steps=(extent, extent),
                     vertices=vertices, outlines=outlines, sources=sources,
                     favourable=np.full((3, 16), favourable), alpha_db_per_km=alpha_bands(15.0, 70.0),
                     flat_altitude_m=0.0, flat_ground_factor=flat_ground_factor, name="stock")


def square(cx, cy, half):
    return [(cx - half, cy - half), (cx + half, cy - half), (cx + half, cy + half), (cx - half, cy + half)]


def point_sources(stock, points_m, level_db=90.0, height_m=0.05):
    """Point sources at `points_m` (metres), every band and period at `level_db`."""
    src = np.zeros(len(points_m), dtype=abi.SOURCE_DTYPE)
    for k, p in enumerate(points_m):
        x, y = stock.steps(p)
        src[k]["x"], src[k]["y"] = x, y
        src[k]["height_m"] = height_m
        src[k]["ground_factor"] = -1.0
        src[k]["energy"][:] = 10.0 ** (level_db / 10.0)
    return src
