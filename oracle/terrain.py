"""The reference's `terrain` tile writer (qmterr2), restated in Python — TEST INFRASTRUCTURE ONLY.

`encode` follows tiles/src/terrain.rs:183-214: the 24-byte header (magic, north and west node,
rows, columns), then one zstd frame of five planes: the height code's residual after the planar
prediction from the west, north and north-west nodes (u16 ring, terrain.rs:145-153), zigzag-coded
into a low and a high byte plane, then imperviousness, forest cover and canopy height. The frame
is made by the system's libzstd (the reference's level, 19). Only tests import this module.
"""

import ctypes as C
import struct

import numpy as np

MAGIC = b"qmterr2\n"
HEIGHT_MISSING = 65535
LEVEL = 19

_zstd = None


def _lib():
    global _zstd
    if _zstd is None:
        _zstd = C.CDLL("libzstd.so.1")
        _zstd.ZSTD_compressBound.argtypes = [C.c_size_t]
        _zstd.ZSTD_compressBound.restype = C.c_size_t
        _zstd.ZSTD_compress.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_int]
        _zstd.ZSTD_compress.restype = C.c_size_t
        _zstd.ZSTD_isError.argtypes = [C.c_size_t]
        _zstd.ZSTD_isError.restype = C.c_uint
    return _zstd


def compress(data):
    z = _lib()
    src = bytes(data)
    cap = z.ZSTD_compressBound(len(src))
    dst = C.create_string_buffer(cap)
    n = z.ZSTD_compress(dst, cap, src, len(src), LEVEL)
    assert not z.ZSTD_isError(n)
    return dst.raw[:n]


def predicted(heights, r, c):
    """terrain.rs:145-153, in the u16 ring."""
    west = int(heights[r, c - 1]) if c > 0 else 0
    north = int(heights[r - 1, c]) if r > 0 else 0
    north_west = int(heights[r - 1, c - 1]) if r > 0 and c > 0 else 0
    return (west + north - north_west) & 0xFFFF


def planes(heights, impervious, forest, canopy):
    """The five planes before compression."""
    rows, columns = heights.shape
    low = np.zeros(heights.shape, np.uint8)
    high = np.zeros(heights.shape, np.uint8)
    for r in range(rows):
        for c in range(columns):
            residual = (int(heights[r, c]) - predicted(heights, r, c)) & 0xFFFF
            signed = residual - 0x10000 if residual >= 0x8000 else residual
            zigzag = ((signed << 1) ^ (signed >> 15)) & 0xFFFF
            low[r, c], high[r, c] = zigzag & 0xFF, zigzag >> 8
    return b"".join(np.ascontiguousarray(p, dtype=np.uint8).tobytes()
                    for p in (low, high, impervious, forest, canopy))


def encode(north_node, west_node, heights, impervious, forest, canopy):
    """The bytes of a terrain tile of a window whose row 0 is `north_node` and column 0 `west_node`."""
    rows, columns = heights.shape
    header = MAGIC + struct.pack("<iiII", north_node, west_node, rows, columns)
    return header + compress(planes(heights, impervious, forest, canopy))


FINE_MAGIC = b"qmtfin2\n"
BLOCK_CELLS = 128


def _block_span(block, nodes):
    """tiles/src/terrain_fine.rs:52-56."""
    first = block * BLOCK_CELLS
    return first, min(first + BLOCK_CELLS, nodes - 1)


def _blocks_along(nodes):
    """tiles/src/terrain_fine.rs:47-50."""
    return max(-(-(nodes - 1) // BLOCK_CELLS), 1)


def encode_fine(north_node, west_node, details):
    """A fine terrain tile (tiles/src/terrain_fine.rs:58-110): header, the directory of each
    block's frame end, then per block (row-major) one frame of its planar residual's two planes."""
    rows, columns = details.shape
    codes = details.astype(np.int16).view(np.uint16)
    frames, ends = b"", []
    for br in range(_blocks_along(rows)):
        r0, r1 = _block_span(br, rows)
        for bc in range(_blocks_along(columns)):
            c0, c1 = _block_span(bc, columns)
            block = codes[r0:r1 + 1, c0:c1 + 1]
            zero = np.zeros(block.shape, np.uint8)
            frames += compress(planes(block, zero, zero, zero)[:2 * block.size])
            ends.append(len(frames))
    header = FINE_MAGIC + struct.pack("<iiII", north_node, west_node, rows, columns)
    return header + b"".join(struct.pack("<I", e) for e in ends) + frames
