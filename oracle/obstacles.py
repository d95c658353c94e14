"""The reference's `obstacles` tile writer (qmobs2), restated in Python — TEST INFRASTRUCTURE ONLY.

It makes the tiles the library's reader is tested on: `edge_cells` follows the supercover cell
walk of tiles/src/obstacles/cells.rs:13-47 and `encode` the byte layout of
tiles/src/obstacles.rs:151-276 (header, occupied-cell bitmap and counts, first runs, footprint
squares, runs, outline records, vertices); `tiles_crossed` names the tiles that store an outline
(cells.rs:49-75). Only tests import this module.
"""

import math
import struct

MAGIC = b"qmobs2\n\0"
CELL_STEPS = 256
CELLS_PER_SIDE = 128
CELLS = CELLS_PER_SIDE * CELLS_PER_SIDE
HALF_TILE_CELLS = CELLS_PER_SIDE // 2
HEADER_BYTES = 32
CELL_WORDS = CELLS // 64
CELL_INDEX_BYTES = CELL_WORDS * (8 + 2)
RUN_BYTES, OUTLINE_BYTES, VERTEX_BYTES = 8, 12, 4
EXTERIOR, HOLE, WALL = 0, 1, 2
OUTDOOR, RESIDENTIAL, COMMERCIAL, INDUSTRIAL, HISTORIC, DEFAULT = range(6)


def edge_cells(start, end):
    """The 256-step cells the edge start -> end passes through, 4-connected in walking order; a
    tie steps the row, and the walk never leaves the box of its end cells (cells.rs:13-47)."""
    cell = [start[0] // CELL_STEPS, start[1] // CELL_STEPS]
    last = [end[0] // CELL_STEPS, end[1] // CELL_STEPS]
    delta = [float(end[0] - start[0]), float(end[1] - start[1])]
    step = [1 if d >= 0.0 else -1 for d in delta]
    t_delta = [abs(CELL_STEPS / d) if d != 0.0 else math.inf for d in delta]
    t_max = []
    for axis in (0, 1):
        if delta[axis] == 0.0:
            t_max.append(math.inf)
            continue
        boundary = (cell[axis] + (1 if delta[axis] >= 0.0 else 0)) * CELL_STEPS
        t_max.append(abs((boundary - start[axis]) / delta[axis]))
    visited = []
    while True:
        visited.append((cell[0], cell[1]))
        if cell == last:
            return visited
        if cell[0] == last[0]:
            axis = 1
        elif cell[1] == last[1] or t_max[0] < t_max[1]:
            axis = 0
        else:
            axis = 1
        t_max[axis] += t_delta[axis]
        cell[axis] += step[axis]


def _height_code(height_m):
    """Decimetres rounded half away from zero (obstacles.rs:139-146)."""
    x = height_m * 10.0
    f = math.floor(x)
    code = f + 1 if x - f >= 0.5 else f
    assert 1 <= code <= 0xFFFF, height_m
    return int(code)


def encode(outlines):
    """The bytes of a tile holding `outlines` (dicts: footprint_id, kind, envelope, height_m,
    vertices [(x, y) int16, ...]), stored in the given order, which is sorted by footprint id."""
    cells = [[] for _ in range(CELLS)]
    for index, outline in enumerate(outlines):
        vertices = [tuple(v) for v in outline["vertices"]]
        if outline["kind"] == WALL:
            assert len(vertices) >= 2
        else:
            assert len(vertices) >= 4 and vertices[0] == vertices[-1]
        assert index == 0 or outlines[index - 1]["footprint_id"] <= outline["footprint_id"]
        for edge in range(len(vertices) - 1):
            for column, row in edge_cells(vertices[edge], vertices[edge + 1]):
                column, row = column + HALF_TILE_CELLS, row + HALF_TILE_CELLS
                if not (0 <= column < CELLS_PER_SIDE and 0 <= row < CELLS_PER_SIDE):
                    continue
                runs = cells[row * CELLS_PER_SIDE + column]
                if runs and runs[-1][0] == index and runs[-1][1] + runs[-1][2] == edge:
                    runs[-1][2] += 1
                else:
                    runs.append([index, edge, 1])
    vertex_count = sum(len(o["vertices"]) for o in outlines)
    run_count = sum(len(runs) for runs in cells)
    occupied = sum(1 for runs in cells if runs)
    squares = []
    for outline in outlines:
        high = outline["footprint_id"] >> 32
        if not squares or squares[-1] != high:
            squares.append(high)
    assert len(squares) <= 256
    out = bytearray(MAGIC)
    for count in (len(outlines), vertex_count, run_count, occupied, len(squares), 0):
        out += struct.pack("<I", count)
    words = []
    for w in range(CELL_WORDS):
        bits = 0
        for bit in range(64):
            if cells[64 * w + bit]:
                bits |= 1 << bit
        words.append(bits)
    for word in words:
        out += struct.pack("<Q", word)
    before = 0
    for word in words:
        out += struct.pack("<H", before)
        before += bin(word).count("1")
    first_run = 0
    for runs in cells:
        if runs:
            out += struct.pack("<I", first_run)
            first_run += len(runs)
    out += struct.pack("<I", first_run)
    for square in squares:
        out += struct.pack("<I", square)
    for runs in cells:
        for outline, first_edge, edge_count in runs:
            out += struct.pack("<IHH", outline, first_edge, edge_count)
    first_vertex = 0
    for outline in outlines:
        row = squares.index(outline["footprint_id"] >> 32)
        out += struct.pack("<IIHBB", first_vertex, outline["footprint_id"] & 0xFFFFFFFF,
                           _height_code(outline["height_m"]), row, outline["kind"] | outline["envelope"] << 2)
        first_vertex += len(outline["vertices"])
    for outline in outlines:
        for x, y in outline["vertices"]:
            out += struct.pack("<hh", x, y)
    return bytes(out)


def cell_runs(outlines):
    """Every cell's runs as `encode` lists them: {cell: [(outline, first edge, edge count)]}."""
    cells = {}
    for index, outline in enumerate(outlines):
        vertices = [tuple(v) for v in outline["vertices"]]
        for edge in range(len(vertices) - 1):
            for column, row in edge_cells(vertices[edge], vertices[edge + 1]):
                column, row = column + HALF_TILE_CELLS, row + HALF_TILE_CELLS
                if not (0 <= column < CELLS_PER_SIDE and 0 <= row < CELLS_PER_SIDE):
                    continue
                runs = cells.setdefault(row * CELLS_PER_SIDE + column, [])
                if runs and runs[-1][0] == index and runs[-1][1] + runs[-1][2] == edge:
                    runs[-1][2] += 1
                else:
                    runs.append([index, edge, 1])
    return {cell: [tuple(r) for r in runs] for cell, runs in cells.items()}


TILES_PER_AXIS = 1 << 12
STEPS_PER_TILE = CELLS_PER_SIDE * CELL_STEPS  # 32,768


def tile_centre(tile):
    """A z12 tile's centre in global steps (tiles/src/geo.rs:133-138)."""
    return (tile[0] * STEPS_PER_TILE + STEPS_PER_TILE // 2, tile[1] * STEPS_PER_TILE + STEPS_PER_TILE // 2)


def tiles_crossed(vertices):
    """The tiles (x, y) whose cells an outline's edges (global steps) pass through, sorted: every
    tile that stores it (tiles/src/obstacles/cells.rs:49-75; rows beyond the poles have no tiles,
    columns wrap at the antimeridian)."""
    tiles = set()
    for a, b in zip(vertices[:-1], vertices[1:]):
        for column, row in edge_cells(a, b):
            y = row // CELLS_PER_SIDE
            if not 0 <= y < TILES_PER_AXIS:
                continue
            tiles.add(((column // CELLS_PER_SIDE) % TILES_PER_AXIS, y))
    return sorted(tiles)


def _wrap_to_pi(angle):
    """physics/src/line.rs:39-48 (Rust's % on floats is C's fmod)."""
    a = math.fmod(angle, 2.0 * math.pi)
    if a > math.pi:
        return a - 2.0 * math.pi
    if a <= -math.pi:
        return a + 2.0 * math.pi
    return a


def _origin_to_segment_distance(a, b):
    """popup/src/obstacles/skyline.rs:9-20."""
    ex, ey = b[0] - a[0], b[1] - a[1]
    length2 = ex * ex + ey * ey
    t = min(max(-(a[0] * ex + a[1] * ey) / length2, 0.0), 1.0) if length2 > 0.0 else 0.0
    x, y = a[0] + t * ex, a[1] + t * ey
    return math.sqrt(x * x + y * y)


class Skyline:
    """The receiver skyline of the line quadrature (popup/src/obstacles/skyline.rs:22-110) over
    outlines on the global step lattice (y growing south): each edge's supercover cells give the
    cells' runs and their tallest outline, as a tile's index holds them (tiles/src/obstacles.rs,
    popup/src/obstacles/tile.rs:93-104)."""

    def __init__(self, outlines, metres_per_step):
        self.outlines = outlines
        self.east_m, self.north_m = metres_per_step
        self.runs = {}
        for index, outline in enumerate(outlines):
            vertices = [tuple(v) for v in outline["vertices"]]
            for edge in range(len(vertices) - 1):
                for cell in edge_cells(vertices[edge], vertices[edge + 1]):
                    runs = self.runs.setdefault(cell, [])
                    if runs and runs[-1][0] == index and runs[-1][1] + runs[-1][2] == edge:
                        runs[-1][2] += 1
                    else:
                        runs.append([index, edge, 1])
        self.max_height = {cell: max(outlines[r[0]]["height_m"] for r in runs) for cell, runs in self.runs.items()}

    def arcs(self, origin_steps, lo_rad, hi_rad, radius_m, los_floor_m):
        """Every (lo, hi, nearest) arc an edge near the receiver at `origin_steps` hands over for the
        wedge [lo_rad, hi_rad], once per cell it is listed in."""
        ox, oy = origin_steps
        east_m, north_m = self.east_m, self.north_m
        cs = float(CELL_STEPS)
        span = lambda centre, half: range(math.floor((centre - half) / cs), math.floor((centre + half) / cs) + 1)
        low, high = (math.cos(lo_rad), math.sin(lo_rad)), (math.cos(hi_rad), math.sin(hi_rad))
        relative = lambda v: ((v[0] - ox) * east_m, (oy - v[1]) * north_m)
        out = []
        for row in span(oy, radius_m / north_m):
            south = (oy - (row + 1) * cs) * north_m
            north = (oy - row * cs) * north_m
            dy = max(south, -north, 0.0)
            for column in span(ox, radius_m / east_m):
                west = (column * cs - ox) * east_m
                east = ((column + 1) * cs - ox) * east_m
                dx = max(west, -east, 0.0)
                if dx * dx + dy * dy > radius_m * radius_m:
                    continue
                corners = [(west, south), (east, south), (west, north), (east, north)]
                below = all(low[0] * c[1] - low[1] * c[0] < 0.0 for c in corners)
                above = all(c[0] * high[1] - c[1] * high[0] < 0.0 for c in corners)
                if below or above:
                    continue
                runs = self.runs.get((column, row))
                if not runs or self.max_height[(column, row)] <= los_floor_m:
                    continue
                for index, first_edge, edge_count in runs:
                    outline = self.outlines[index]
                    if outline["kind"] == WALL and outline["height_m"] <= los_floor_m:
                        continue
                    vertices = outline["vertices"]
                    a = relative(vertices[first_edge])
                    azimuth_a = math.atan2(a[1], a[0])
                    for nxt in range(first_edge + 1, first_edge + edge_count + 1):
                        b = relative(vertices[nxt])
                        azimuth_b = math.atan2(b[1], b[0])
                        nearest = _origin_to_segment_distance(a, b)
                        if 1e-6 <= nearest <= radius_m:
                            unwrapped_b = azimuth_a + _wrap_to_pi(azimuth_b - azimuth_a)
                            out.append((min(azimuth_a, unwrapped_b), max(azimuth_a, unwrapped_b), nearest))
                        a, azimuth_a = b, azimuth_b
        return out
