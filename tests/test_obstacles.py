"""`obstacles` tiles (qmobs2): the library's reader against tiles the oracle writes, pinned to the
reference's own tests (tiles/src/obstacles/tests.rs: round trip, cell runs, the supercover walk,
corrupt files, footprint squares). The reader runs on the host; no device is needed."""

import struct

import numpy as np
import pytest

from oracle import obstacles as ob
from quietmap_b200 import native

HEADER, WORDS = ob.HEADER_BYTES, ob.CELL_WORDS


def courtyard_block_and_wall():
    """A 600-step block with a 200-step courtyard, and a wall whose last edge leaves the tile."""
    def ring(kind, half):
        return dict(footprint_id=0x0114_00AD_0000_0007, kind=kind, envelope=ob.RESIDENTIAL, height_m=29.0,
                    vertices=[(-half, -half), (half, -half), (half, half), (-half, half), (-half, -half)])
    return [ring(ob.EXTERIOR, 300), ring(ob.HOLE, 100),
            dict(footprint_id=0x0114_00AD_0000_0009, kind=ob.WALL, envelope=ob.OUTDOOR, height_m=3.6,
                 vertices=[(16_000, 10), (16_300, 20), (16_600, 30), (32_767, -32_768)])]


def test_the_supercover_walk_steps_the_row_on_a_tie_and_stays_in_its_box():
    assert ob.edge_cells((0, 0), (512, 512)) == [(0, 0), (0, 1), (1, 1), (1, 2), (2, 2)]
    assert ob.edge_cells((5, 5), (5, 5)) == [(0, 0)]
    assert ob.edge_cells((-1, -1), (-300, -1)) == [(-1, -1), (-2, -1)]
    assert ob.edge_cells((0, 511), (256, 256)) == [(0, 1), (1, 1)]


def test_round_trip_outlines_and_cell_runs():
    outlines = courtyard_block_and_wall()
    data = ob.encode(outlines)
    counts = native.obstacles_check(data)
    assert (counts["outlines"], counts["vertices"], counts["footprint_squares"]) == (3, 14, 1)
    recs, vertices, envelope = native.obstacles_outlines(data, offset=(1000, -2000), first_vertex_base=7)
    for rec, env, outline in zip(recs, envelope, outlines):
        v = vertices[rec["first_vertex"] - 7:rec["first_vertex"] - 7 + rec["vertex_count"]]
        assert [tuple(p) for p in (v - [1000, -2000])] == outline["vertices"]
        assert rec["footprint_id"] == outline["footprint_id"]
        assert rec["height_m"] == np.float32(outline["height_m"])
        assert rec["building"] == (outline["kind"] != ob.WALL)
        assert env == outline["envelope"]
    # The block's west edge runs down column 62; corner cells also hold the edge before it.
    assert native.obstacles_cell_runs(data, 62, 65) == [(0, 2, 2)]
    assert native.obstacles_cell_runs(data, 62, 64) == [(0, 3, 1)]
    assert native.obstacles_cell_runs(data, 62, 62) == [(0, 0, 1), (0, 3, 1)]
    assert native.obstacles_cell_runs(data, 63, 63) == [(1, 0, 1), (1, 3, 1)]
    # The wall is stored whole but listed only where it crosses the tile's cells.
    assert native.obstacles_cell_runs(data, 126, 64) == [(2, 0, 1)]
    assert native.obstacles_cell_runs(data, 127, 64) == [(2, 0, 2)]
    listed = sum(1 for c in range(ob.CELLS) for r in native.obstacles_cell_runs(data, c % 128, c // 128) if r[0] == 2)
    assert listed == 2
    assert native.obstacles_check(ob.encode([]))["runs"] == 0


def test_corrupt_files_are_rejected():
    data = ob.encode(courtyard_block_and_wall())
    native.obstacles_check(data)
    header = lambda at: struct.unpack_from("<I", data, at)[0]
    occupied, squares = header(20), header(24)
    runs_total = header(16)
    before = HEADER + 8 * WORDS
    first_runs = HEADER + ob.CELL_INDEX_BYTES
    runs = first_runs + 4 * (occupied + 1) + 4 * squares
    outlines = runs + ob.RUN_BYTES * runs_total

    def rejected(changes):
        copy = bytearray(data)
        for at, value in changes:
            copy[at] = value
        try:
            native.obstacles_check(bytes(copy))
        except native.QmError:
            return True
        return False

    for short in (data[:-1], data + b"\0"):
        with pytest.raises(native.QmError, match="length does not match"):
            native.obstacles_check(short)
    assert rejected([(0, ord("x"))]), "magic"
    assert rejected([(8, 4)]), "outline count against the length"
    assert rejected([(28, 1)]), "reserved header word"
    assert rejected([(HEADER, 0x01)]), "an occupied bit more"
    assert rejected([(before + 2 * (WORDS - 1), 0)]), "occupied cells miscounted"
    assert rejected([(first_runs + 4, 0)]), "a cell's runs out of order"
    assert rejected([(runs, 7)]), "a run naming a missing outline"
    assert rejected([(runs + 6, 5)]), "a run past its outline's last edge"
    assert not rejected([(runs + 6, 4)]), "a run up to the last edge is fine"
    assert rejected([(outlines + 11, 3)]), "outline kind"
    assert rejected([(outlines + 11, 6 << 2)]), "envelope class"
    assert rejected([(outlines + 8, 0), (outlines + 9, 0)]), "zero height"
    assert rejected([(outlines + 10, 1)]), "a missing square"
    assert rejected([(outlines + ob.OUTLINE_BYTES, 1)]), "a ring that no longer closes"
    assert rejected([(outlines + ob.OUTLINE_BYTES + 4, 0)]), "footprint ids out of order"


def test_footprints_of_two_squares_keep_their_ids():
    outlines = courtyard_block_and_wall()
    outlines[2]["footprint_id"] = 0x0115_00AD_8000_0001
    data = ob.encode(outlines)
    recs, _, _ = native.obstacles_outlines(data)
    assert [int(r) for r in recs["footprint_id"]] == [o["footprint_id"] for o in outlines]
    assert native.obstacles_check(data)["footprint_squares"] == 2


def test_a_crowded_tile_reads_back_whole():
    rng = np.random.default_rng(8)
    outlines = []
    for k in range(300):
        cx, cy = (int(v) for v in rng.integers(-16_000, 16_000, 2))
        w, h = (int(v) for v in rng.integers(20, 900, 2))
        ring = [(cx, cy), (cx + w, cy), (cx + w, cy + h), (cx, cy + h), (cx, cy)]
        ring = [(max(-32_768, min(32_767, x)), max(-32_768, min(32_767, y))) for x, y in ring]
        outlines.append(dict(footprint_id=(0x0200 + k // 120) << 32 | k, kind=ob.EXTERIOR, envelope=k % 6,
                             height_m=float(rng.integers(10, 600)) / 10.0, vertices=ring))
    for k in range(40):
        pts = [tuple(int(v) for v in rng.integers(-20_000, 20_000, 2)) for _ in range(int(rng.integers(2, 6)))]
        pts = [(max(-32_768, min(32_767, x)), max(-32_768, min(32_767, y))) for x, y in pts]
        outlines.append(dict(footprint_id=(0x0203 << 32) | k, kind=ob.WALL, envelope=ob.OUTDOOR,
                             height_m=2.5, vertices=pts))
    data = ob.encode(outlines)
    recs, vertices, envelope = native.obstacles_outlines(data)
    assert len(recs) == len(outlines)
    for rec, env, outline in zip(recs, envelope, outlines):
        v = vertices[rec["first_vertex"]:rec["first_vertex"] + rec["vertex_count"]]
        assert [tuple(p) for p in v] == outline["vertices"]
        assert env == outline["envelope"] and rec["footprint_id"] == outline["footprint_id"]
    expected = ob.cell_runs(outlines)
    for cell in range(0, ob.CELLS, 7):
        got = native.obstacles_cell_runs(data, cell % 128, cell // 128, cap=512)
        assert got == expected.get(cell, []), cell


def test_an_outline_is_listed_in_every_tile_whose_cells_it_crosses():
    """tiles/src/obstacles/tests.rs:103-134."""
    centre = ob.tile_centre((2212, 1387))
    east_edge = (centre[0] + 16_383, centre[1])
    assert ob.tiles_crossed([east_edge, (east_edge[0] + 2, east_edge[1])]) == [(2212, 1387), (2213, 1387)]
    assert ob.tiles_crossed([(-10, 5_000), (10, 5_000)]) == [(0, 0), (ob.TILES_PER_AXIS - 1, 0)]
    assert ob.tiles_crossed([(0, -600), (0, -300)]) == []


def test_tiles_merge_into_one_scene_keeping_each_outline_once():
    rng = np.random.default_rng(12)
    block = [(10, 10), (11, 10), (10, 11), (11, 11)]
    corner = ob.tile_centre((11, 11))
    corner = (corner[0] - ob.STEPS_PER_TILE // 2, corner[1] - ob.STEPS_PER_TILE // 2)  # shared by the four
    world = []
    for k in range(120):
        cx, cy = (int(v) for v in corner + rng.integers(-9_000, 9_000, 2))
        w, h = (int(v) for v in rng.integers(100, 3_000, 2))
        kind = ob.WALL if k % 9 == 0 else ob.EXTERIOR
        verts = ([(cx, cy), (cx + w, cy + h)] if kind == ob.WALL else
                 [(cx, cy), (cx + w, cy), (cx + w, cy + h), (cx, cy + h), (cx, cy)])
        world.append(dict(footprint_id=(0x0300 << 32) | k, kind=kind, envelope=ob.OUTDOOR if kind == ob.WALL else
                          ob.COMMERCIAL, height_m=12.5, vertices=verts))
    files, offsets, stored = [], [], 0
    origin = ob.tile_centre(block[0])
    origin = (origin[0] - ob.STEPS_PER_TILE // 2, origin[1] - ob.STEPS_PER_TILE // 2)  # the scene's (0, 0)
    for tile in block:
        cx, cy = ob.tile_centre(tile)
        mine = [dict(o, vertices=[(x - cx, y - cy) for x, y in o["vertices"]])
                for o in world if tile in ob.tiles_crossed(o["vertices"])]
        stored += len(mine)
        files.append(ob.encode(mine))
        offsets.append((cx - origin[0], cy - origin[1]))
    assert stored > len(world)  # some outlines are stored in several tiles
    outlines, vertices, envelope = native.obstacles_merge(files, offsets)
    got = {int(o["footprint_id"]): [tuple(p) for p in vertices[o["first_vertex"]:o["first_vertex"] + o["vertex_count"]]]
           for o in outlines}
    assert len(outlines) == len(world) == len(got)
    for o in world:
        assert got[o["footprint_id"]] == [(x - origin[0], y - origin[1]) for x, y in o["vertices"]]
    assert set(int(e) for e in envelope) == {ob.OUTDOOR, ob.COMMERCIAL}
    with pytest.raises(native.QmError, match="tile 1: obstacles: bad magic"):
        native.obstacles_merge([files[0], b"x" * 40], offsets[:2])
