"""CPU checks of the native library: it loads, exports every entry point the
header declares, builds the octree topology on the host identically to the
oracle, and rejects bad arguments with status codes.  No device call is made."""
import ctypes
import os
import re

import numpy as np
import pytest

import cmg
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "cmg.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cmg_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(cmg.LIB_PATH)
    names = header_functions()
    assert len(names) >= 38
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert sorted(cmg.EXPORTS) == names


@pytest.mark.parametrize("case_id,prm", [
    (cmg.CASE_UNIFORM, [3, 3]),
    (cmg.CASE_CENTER_POINT, [2, 6]),
    (cmg.CASE_SPHERE_EMPTY, [2, 5]),
    (cmg.CASE_SPHERE_SOLID, [2, 5]),
    (cmg.CASE_STAR_EMPTY, [3, 6]),
    (cmg.CASE_STAR_SOLID, [2, 5]),
    (cmg.CASE_SHELL, [4, 6, 5, 0.5, 0.5, 0.5, 0.1, 0.05, 0.15]),
    (cmg.CASE_MULTI_SPHERE, [3, 5, 0.05, 2, 0.3, 0.3, 0.4, 0.08, 0.7, 0.6, 0.5, 0.12]),
])
def test_host_topology_matches_oracle(case_id, prm):
    G = cmg.HADeviceGrid(0.125, 10, 16)
    G.set_tile_host(0, (0, 0, 0), cmg.LEAF)
    G.rebuild()
    G.refine_case(case_id, prm)
    g = O.Grid(0.125, 10)
    g.set_tile(0, 0, 0, 0, O.LEAF)
    g.rebuild()
    g.refine_case(case_id, prm)
    for a, b in zip(G.tiles(), g.tiles()):
        assert np.array_equal(a, b)
    nb, ch = G.tables()
    onb, opar, och = g.tables()
    assert np.array_equal(nb[:, :6], onb)
    assert np.array_equal(nb[:, 6], opar)
    assert np.all(nb[:, 7] == -1)
    assert np.array_equal(ch, och)


def test_callback_refinement_equals_builtin_case():
    """iterativeRefine with a host callback reproduces the built-in uniform case."""
    G = cmg.HADeviceGrid(0.125, 10, 16)
    G.set_tile_host(0, (0, 0, 0), cmg.LEAF)
    G.rebuild()
    G.iterative_refine(lambda l, i, j, k: 3)
    H = cmg.HADeviceGrid(0.125, 10, 16)
    H.set_tile_host(0, (0, 0, 0), cmg.LEAF)
    H.rebuild()
    H.refine_case(cmg.CASE_UNIFORM, [3, 3])
    for a, b in zip(G.tiles(), H.tiles()):
        assert np.array_equal(a, b)


def test_refinement_respects_level_capacity():
    G = cmg.HADeviceGrid(0.125, 3, 16)  # levels 0..2 only
    G.set_tile_host(0, (0, 0, 0), cmg.LEAF)
    G.rebuild()
    G.refine_case(cmg.CASE_UNIFORM, [5, 5])
    assert G.max_level == 2


def test_bad_arguments_return_status_codes():
    L = cmg.lib()
    h = ctypes.c_void_p()
    assert L.cmg_grid_create(-1.0, 10, 16, ctypes.byref(h)) == 1
    assert L.cmg_grid_create(0.125, 0, 16, ctypes.byref(h)) == 1
    G = cmg.HADeviceGrid(0.125, 10, 16)
    assert L.cmg_grid_set_tile(G.h, 0, 0, 0, 0, 3) == 1          # not a tile type
    assert L.cmg_grid_set_tile(G.h, 12, 0, 0, 0, 1) == 1         # level beyond capacity
    p = ctypes.c_void_p()
    assert L.cmg_grid_channel_ptr(G.h, 0, ctypes.byref(p)) == 3  # not built yet
    prm = np.array([3.0, 3.0])
    assert L.cmg_grid_refine_case(G.h, 99, prm.ctypes.data_as(ctypes.c_void_p), 2, None) == 1
    assert b"not built" in L.cmg_last_error() or b"bad argument" in L.cmg_last_error()


def test_learned_entry_points_reject_bad_arguments():
    """The learned smoother's entry points validate their arguments before touching the GPU."""
    L = cmg.lib()
    out = ctypes.c_void_p()
    assert L.cmg_learned_create(12, 0, ctypes.byref(out)) == 1  # hidden must be 8, 16 or 32
    assert L.cmg_learned_create(8, 0, None) == 1
    assert L.cmg_learned_set_inference(2) == 1
    assert L.cmg_learned_set_loss(None, 0) == 1
    n = ctypes.c_int(0)
    assert L.cmg_learned_num_params(None, ctypes.byref(n)) == 1
    assert L.cmg_learned_forward(None, 0, 1, None) == 1
    assert L.cmg_learned_gradient(None, 0, 1, None, None) == 1
    assert L.cmg_learned_train(None, 1, 1, ctypes.c_float(1e-3), 0, None) == 1
    assert L.cmg_amg_solver_set_learned(None, None) == 1
    assert L.cmg_amg_solver_learned_status(None, None, None, None) == 1
    assert L.cmg_learned_destroy(None) == 0
    assert L.cmg_learned_create(12, 0, ctypes.byref(out)) == 1
    assert b"hidden" in L.cmg_last_error()


def test_learned_oracle_parameter_layout_matches_header():
    """The parameter layout of the FP64 restatement: W1[H][27][8], b1[H], W2[H][27][H], b2[H], W3[27][H]."""
    from oracle import learned_oracle as LO

    for H in (8, 16):
        L = LO.layout(H)
        assert L["B1"] == H * 216 and L["W2"] == L["B1"] + H
        assert L["B2"] == L["W2"] + 27 * H * H and L["W3"] == L["B2"] + H and L["n"] == L["W3"] + 27 * H


def test_autotune_rejects_bad_arguments():
    """cmg_amg_solver_autotune checks its arguments before touching the GPU (a solver needs a
    GPU to exist, so only the null-object and empty-candidate cases run here)."""
    L = cmg.lib()
    arr = (cmg.TuneCandidate * 1)(cmg.TuneCandidate(1.0, 1, 2, 5, -1))
    ms = np.zeros(1, np.float32)
    its = np.zeros(1, np.int32)
    best = ctypes.c_int(7)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    for n, tol in [(1, 1e-6), (0, 1e-6), (1, 0.0)]:
        assert L.cmg_amg_solver_autotune(None, None, n, ctypes.cast(arr, ctypes.c_void_p), 10, ctypes.c_double(tol), 1, P(ms),
                                         P(its), ctypes.byref(best)) == 1
    assert b"autotune" in L.cmg_last_error()
    assert L.cmg_amg_solver_set_finest_iters(None, 2) == 1
    assert ctypes.sizeof(cmg.TuneCandidate) == 24


def test_default_tune_candidates_are_valid_and_symmetric():
    """The autotuner's default search: distinct settings, the reference setting among them, and
    a finest-level sweep count below the level count only (never asymmetric pre/post)."""
    cands = cmg.default_tune_candidates()
    assert len(cands) == len(set(cands)) == 156
    assert (1.5, 2, 2, 10, -1) in cands
    for om, mu, li, ci, fi in cands:
        assert om > 0 and mu in (1, 2) and li >= 1 and ci >= 1
        assert fi == -1 or 1 <= fi < li


def test_moving_sphere_positions_stay_inside_the_domain():
    """The moving-sphere sequence: centre on a circle of radius 0.25 in z = 0.5, 400 steps per
    turn, sphere (r = 0.1) and its 0.15 refinement band inside [0, 1]^3."""
    import bench

    for k in (0, 50, 100, 199, 399):
        sp = bench.moving_sphere_spec(k)
        cx, cy, cz, r = sp["spheres"][0]
        assert abs(np.hypot(cx - 0.5, cy - 0.5) - 0.25) < 1e-12 and cz == 0.5 and r == 0.1
        assert min(cx, cy, cz) - r - 0.15 >= 0.0 - 1e-12 and max(cx, cy, cz) + r + 0.15 <= 1.0 + 1e-12
        assert sp["params"][3:6] == [cx, cy, cz]
    c0, c400 = bench.moving_sphere_spec(0)["spheres"][0], bench.moving_sphere_spec(400)["spheres"][0]
    assert np.allclose(c0, c400)
