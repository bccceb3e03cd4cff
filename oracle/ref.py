"""ctypes binding of oracle/_ref/libcmgref.so: the reference's own host-compilable
functions, built from the reference tree by oracle/build_ref.py (test infrastructure).

Used only by tests/ to pin the oracle and the product to the reference.  available()
is False when the library is neither built nor buildable (no reference tree and no
prebuilt .so), and the pin tests skip with that reason.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libcmgref.so")
REF_ROOT = "/root/reference"

# tests/TestGridsStr.h order
TEST_GRIDS = ["uniform8", "uniform32", "uniform128", "uniform256", "uniform512", "staircase12", "staircase21",
              "staircase34", "staircase43", "twosources67", "twosources_deform", "centersource"]

_lib = None
_why = None


def lib():
    global _lib, _why
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH) or (os.path.isdir(REF_ROOT) and _stale()):
        if not os.path.isdir(REF_ROOT):
            _why = "oracle/_ref/libcmgref.so is not built and the reference tree is absent"
            return None
        from oracle import build_ref

        build_ref.build(REF_ROOT)
    L = ctypes.CDLL(LIB_PATH)
    P, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
    sig = {
        "cr_layout": (I, [P, I]),
        "cr_hagr_layout": (I, [P, I]),
        "cr_frac_inside": (F, [F, F]),
        "cr_face_fluid_ratio": (None, [P, I, P]),
        "cr_cell_corner_inside_count": (None, [P, I, F, P]),
        "cr_case_target": (I, [I, F, I, I, I, I, I, I]),
        "cr_case_types": (I, [I, F, I, I, I, I, P]),
        "cr_solvertests_level_target": (I, [I, F, I, I, I, I]),
        "cr_child_tile": (None, [P, P, I, I, I, P, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return _lib


def _stale():
    """The library is older than its recipe (rebuild in a container that has the reference)."""
    t = os.path.getmtime(LIB_PATH)
    return any(os.path.getmtime(os.path.join(HERE, f)) > t for f in ("ref_harness.cu", "build_ref.py"))


def available():
    return lib() is not None


def why_unavailable():
    lib()
    return _why


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def layout():
    out = np.zeros(16, np.int64)
    m = lib().cr_layout(_p(out), 16)
    keys = ["tile_bytes", "off_data", "off_neighbors", "off_cell_types", "off_interest", "off_locked", "off_status",
            "off_serial", "channel_stride", "channels", "info_bytes", "info_off_tile_ptr", "info_off_type"]
    return dict(zip(keys, out[:m].tolist()))


def hagr_layout():
    out = np.zeros(16, np.int64)
    m = lib().cr_hagr_layout(_p(out), 16)
    keys = ["header_bytes", "off_magic", "off_version", "off_num_levels", "off_max_level", "off_tile_size",
            "off_coord_size", "off_h0", "off_tile_count", "coord_bytes", "tile_bytes"]
    return dict(zip(keys, out[:m].tolist()))


def frac_inside(a, b):
    return lib().cr_frac_inside(a, b)


def face_fluid_ratio(phi4):
    phi4 = np.ascontiguousarray(phi4, np.float32).reshape(-1, 4)
    out = np.zeros(len(phi4), np.float32)
    lib().cr_face_fluid_ratio(_p(phi4), len(phi4), _p(out))
    return out


def cell_corner_inside_count(nodes729, iso, chan=5):
    nodes = np.ascontiguousarray(nodes729, np.float32).reshape(729)
    out = np.zeros(512, np.int32)
    lib().cr_cell_corner_inside_count(_p(nodes), chan, iso, _p(out))
    return out


def case_target(case_id, h0, level, ijk, min_level, max_level):
    return lib().cr_case_target(case_id, h0, level, int(ijk[0]), int(ijk[1]), int(ijk[2]), min_level, max_level)


def case_types(case_id, h0, level, ijk):
    out = np.zeros(512, np.uint8)
    rc = lib().cr_case_types(case_id, h0, level, int(ijk[0]), int(ijk[1]), int(ijk[2]), _p(out))
    assert rc == 0
    return out


def solvertests_level_target(name, h0, level, ijk):
    return lib().cr_solvertests_level_target(TEST_GRIDS.index(name), h0, level, int(ijk[0]), int(ijk[1]), int(ijk[2]))


def child_tile(parent_channels, parent_types, offset):
    pc = np.ascontiguousarray(parent_channels, np.float32).reshape(15, 512)
    pt = np.ascontiguousarray(parent_types, np.uint8).reshape(512)
    cc = np.zeros((15, 512), np.float32)
    ct = np.zeros(512, np.uint8)
    lib().cr_child_tile(_p(pc), _p(pt), int(offset[0]), int(offset[1]), int(offset[2]), _p(cc), _p(ct))
    return cc, ct
