"""CPU-side checks of the C ABI: the library loads, exports every entry point the header
declares, and the ctypes mirror matches the header's struct layout."""

import ctypes as C
import os
import re
import subprocess

import pytest

from quietmap_b200 import abi, native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for header in os.listdir(os.path.join(ROOT, "include")):
        if header.endswith(".h"):
            text = open(os.path.join(ROOT, "include", header)).read()
            names |= set(re.findall(r"^\s*(?:qm_status|void|int|const char \*)\s*\*?\s*(qm_\w+)\s*\(", text, re.M))
    return names


def test_library_exports_every_declared_entry_point():
    if not os.path.exists(native.LIB_PATH):
        from quietmap_b200 import build
        build.build()
    lib = C.CDLL(native.LIB_PATH)
    declared = declared_functions()
    assert {"qm_open", "qm_paint_grid", "qm_evaluate_pairs", "qm_zwicker"} <= declared
    missing = [name for name in sorted(declared) if not hasattr(lib, name)]
    assert not missing, missing
    assert lib.qm_abi_version() == abi.ABI_VERSION


def test_struct_layouts_match_the_header():
    # Compile a tiny C program against the header and compare sizes and offsets.
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "qm_batch.h"
#include "qm_surrogate.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu\n", sizeof(qm_outline), sizeof(qm_source), sizeof(qm_scene_desc),
         sizeof(qm_grid_desc), sizeof(qm_paint_stats));
  printf("%zu %zu %zu %zu\n", offsetof(qm_source, energy), offsetof(qm_scene_desc, favourable),
         offsetof(qm_scene_desc, alpha_db_per_km), offsetof(qm_grid_desc, n_bins));
  printf("%zu %zu\n", sizeof(qm_train_config), offsetof(qm_train_config, exact_within_m));
  return 0;
}
'''
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "layout.c")
        open(path, "w").write(src)
        exe = os.path.join(d, "layout")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), path, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()
    sizes = list(map(int, out[:5]))
    offsets = list(map(int, out[5:9]))
    assert list(map(int, out[9:])) == [C.sizeof(abi.TrainConfig), abi.TrainConfig.exact_within_m.offset]
    assert sizes == [C.sizeof(abi.Outline), C.sizeof(abi.Source), C.sizeof(abi.SceneDesc), C.sizeof(abi.GridDesc),
                     C.sizeof(abi.PaintStats)]
    assert offsets == [abi.Source.energy.offset, abi.SceneDesc.favourable.offset,
                       abi.SceneDesc.alpha_db_per_km.offset, abi.GridDesc.n_bins.offset]


def test_flight_records_match_the_header():
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "qm_flights.h"
int main(void) {
  printf("%zu %zu %zu %zu\n", sizeof(qm_flight_box), sizeof(qm_flight_point), sizeof(qm_box_segment),
         sizeof(qm_flight_sums_stats));
  printf("%zu %zu %zu %zu %zu\n", offsetof(qm_flight_box, levels_db), offsetof(qm_flight_box, installation_shares),
         offsetof(qm_flight_box, helicopter), offsetof(qm_flight_point, impedance_gain), offsetof(qm_box_segment, weight));
  printf("%d %d %d\n", QM_FLIGHT_SUMS, QM_TERRAIN_HORIZON_FLOATS, QM_HORIZON_FLOATS);
  return 0;
}
'''
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "flights.c")
        open(path, "w").write(src)
        exe = os.path.join(d, "flights")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), path, "-o", exe], check=True)
        out = list(map(int, subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()))
    assert out[:4] == [abi.FLIGHT_BOX_DTYPE.itemsize, abi.FLIGHT_POINT_DTYPE.itemsize, abi.BOX_SEGMENT_DTYPE.itemsize,
                       C.sizeof(abi.FlightSumsStats)]
    assert out[4:9] == [abi.FLIGHT_BOX_DTYPE.fields[k][1] for k in ("levels_db", "installation_shares", "helicopter")] + [
        abi.FLIGHT_POINT_DTYPE.fields["impedance_gain"][1], abi.BOX_SEGMENT_DTYPE.fields["weight"][1]]
    assert out[9:] == [abi.FLIGHT_SUMS, abi.TERRAIN_HORIZON_FLOATS, abi.HORIZON_FLOATS]


def test_open_without_a_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(native.QmError):
        native.Context(0)
