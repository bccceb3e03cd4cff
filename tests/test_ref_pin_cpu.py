"""The oracle (and the product's host side) pinned to the reference's own code.

oracle/_ref/libcmgref.so is built by oracle/build_ref.py from the reference tree:
its headers as they lie, and the host-callable function definitions of
cirrus_cutcell/MeshCutCell.cu and tests/SolverTests.cu cut out verbatim.  These
tests run that code on the CPU and compare it bit for bit with the oracle's
restatement and with the layout constants the product uses:

  - PoissonTile<float,15> / HATileInfo / 'HAGR' header layout (src/PoissonTile.h:34-39,
    src/HATileInfo.h:61-95, src/HAGrid.h:699-735);
  - FracInside, FaceFluidRatio, CellCornerSDFInsideCount (MeshCutCell.cu:239-412) over
    random and adversarial inputs;
  - the refinement targets and leaf cell types of the test grids (tests/TestGrids.cuh);
  - the solver tests' named grids (tests/SolverTests.cu:17-121) refined by the oracle and
    by the product's host topology through the reference's own level-target function;
  - PoissonTile::childTile (src/PoissonTile.h:151-172), the data refinement hands down.

Plus two findings about the reference's coarsening, shown on the oracle:
  - with NONLEAF cell types set from the leaves (CalcCellTypesFromLeafs, which the
    reference's callers run first: cirrus_cutcell/FluidEuler.cu:940,
    tests/SolverTests.cu:1018), the cell-type mask of CoarsenOffDiagCoefficientsOneStepKernel
    (src/AMGSolver.cu:40-42) is open, so the oracle's open mask is the reference's result;
  - with NONLEAF types left unset (zero or arbitrary bytes), the coarse operator of the
    adaptive sphere octree changes but every INTERIOR diagonal stays positive.
"""
import numpy as np
import pytest

import cmg
from oracle import oracle as O
from oracle import ref as R
from workloads import COEFF, shell_params

pytestmark = pytest.mark.skipif(not R.available(), reason=str(R.why_unavailable()))


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def test_tile_and_blob_layout_match_reference():
    t = R.layout()
    h = R.hagr_layout()
    p = cmg.ref_record_layout()
    assert t["tile_bytes"] == p["tile_bytes"] == h["tile_bytes"] == 44880
    assert t["off_data"] == 0
    assert t["channel_stride"] == p["channel_stride"] == 736
    assert t["channels"] == p["channels"] == 15
    assert t["off_cell_types"] == p["types_offset"]
    assert t["off_neighbors"] == 15 * 736 * 4 and t["off_cell_types"] - t["off_neighbors"] == 6 * t["info_bytes"]
    assert t["info_bytes"] == 32
    for k in ["header_bytes", "off_magic", "off_version", "off_num_levels", "off_max_level", "off_tile_size",
              "off_coord_size", "off_h0", "off_tile_count", "coord_bytes"]:
        assert h[k] == p[k], k


def adversarial_values(rng):
    tiny = np.float32(np.finfo(np.float32).tiny)
    base = np.array([0.0, -0.0, 1.0, -1.0, 0.5, -0.5, 1e-30, -1e-30, tiny, -tiny, tiny / 2, -tiny / 2,
                     1e30, -1e30, 3.0, -3.0, 1e-7, -1e-7, 0.1, -0.1, 2.0 ** -24, -(2.0 ** -24)], np.float32)
    return np.concatenate([base, rng.standard_normal(40).astype(np.float32),
                           (rng.standard_normal(40) * 1e-3).astype(np.float32)])


def test_frac_inside_bitwise():
    rng = np.random.default_rng(0)
    v = adversarial_values(rng)
    a, b = np.meshgrid(v, v, indexing="ij")
    pairs = np.stack([a.ravel(), b.ravel()], 1)
    pairs = pairs[~((pairs[:, 0] == 0) & (pairs[:, 1] == 0))]  # 0/0 is NaN on both sides
    got = np.array([O.frac_inside(float(x), float(y)) for x, y in pairs], np.float32)
    want = np.array([R.frac_inside(float(x), float(y)) for x, y in pairs], np.float32)
    assert np.array_equal(bits(got), bits(want))


def test_face_fluid_ratio_bitwise():
    rng = np.random.default_rng(1)
    quads = [rng.standard_normal((200000, 4)).astype(np.float32),
             (rng.standard_normal((50000, 4)) * 1e-4).astype(np.float32)]
    # every sign pattern with magnitudes from the adversarial set, zeros of both signs included
    v = adversarial_values(rng)
    idx = rng.integers(0, len(v), (100000, 4))
    quads.append(v[idx])
    # corners exactly on the surface, and ratios just around the 0.1 clamp
    z = rng.standard_normal((20000, 4)).astype(np.float32)
    z[rng.random((20000, 4)) < 0.4] = 0.0
    quads.append(z)
    e = np.float32(0.2)
    quads.append(np.array([[s0 * e, s1 * 1.0, s2 * 1.0, s3 * 1.0] for s0 in (-1, 1) for s1 in (-1, 1)
                           for s2 in (-1, 1) for s3 in (-1, 1)], np.float32))
    q = np.concatenate(quads)
    got = O.face_fluid_ratio(q)
    want = R.face_fluid_ratio(q)
    assert np.array_equal(bits(got), bits(want))
    assert 0.0 < want[(want > 0)].min() <= 0.1 + 1e-7


def test_cell_corner_inside_count_matches_reference():
    rng = np.random.default_rng(2)
    for iso in (0.0, 1e-3 / 64, 0.05):
        for scale in (1.0, 1e-3):
            nodes = (rng.standard_normal(729) * scale).astype(np.float32)
            nodes[rng.random(729) < 0.2] = np.float32(iso)
            assert np.array_equal(O.cell_corner_inside_count(nodes, iso), R.cell_corner_inside_count(nodes, iso))


CASES = [(O.CASE_UNIFORM, [3, 3]), (O.CASE_CENTER_POINT, [2, 6]), (O.CASE_SPHERE_EMPTY, [2, 5]),
         (O.CASE_SPHERE_SOLID, [2, 5]), (O.CASE_STAR_EMPTY, [3, 6]), (O.CASE_STAR_SOLID, [2, 5])]


@pytest.mark.parametrize("case_id,prm", CASES)
def test_test_grid_targets_and_types_match_reference(case_id, prm):
    """Every tile of levels 0-4, and every tile of the refined octree, gets the reference's
    target; every LEAF tile of the refined octree gets the reference's cell types."""
    h0 = 0.125
    coords = []
    for L in range(5):
        n = 1 << L
        g = np.stack(np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij"), -1).reshape(-1, 3)
        coords += [(L, c) for c in g]
    g = O.Grid(h0, 10)
    g.set_tile(0, 0, 0, 0, O.LEAF)
    g.rebuild()
    g.refine_case(case_id, prm)
    lv, ijk, ty = g.tiles()
    coords += [(int(l), c) for l, c in zip(lv, ijk) if l >= 5]
    for L, c in coords:
        assert O.case_target_at(h0, case_id, prm, L, c) == R.case_target(case_id, h0, L, c, prm[0], prm[1]), (L, c)
    for l, c, t in zip(lv, ijk, ty):
        if t == O.LEAF:
            assert np.array_equal(O.case_types_at(h0, case_id, int(l), c), R.case_types(case_id, h0, int(l), c)), (l, c)


@pytest.mark.parametrize("name", ["uniform32", "staircase12", "staircase21", "staircase34", "staircase43",
                                  "centersource", "twosources_deform"])
def test_named_solver_test_grids_refine_identically(name):
    """tests/SolverTests.cu's named grids, refined through the reference's own
    SolverTestsLevelTarget by the oracle and by the product's host topology."""
    h0 = 0.125

    def target(level, i, j, k):
        return R.solvertests_level_target(name, h0, level, (i, j, k))

    g = O.Grid(h0, 10)
    g.set_tile(0, 0, 0, 0, O.LEAF)
    g.rebuild()
    g.iterative_refine(target)
    G = cmg.HADeviceGrid(h0, 10, 16)
    G.set_tile_host(0, (0, 0, 0), cmg.LEAF)
    G.rebuild()
    G.iterative_refine(target)
    for a, b in zip(G.tiles(), g.tiles()):
        assert np.array_equal(a, b)
    lv, ijk, ty = g.tiles()
    # every LEAF tile reached the reference's target (a 2:1 graded tree may refine further)
    for l, c, t in zip(lv, ijk, ty):
        if t == O.LEAF:
            assert target(int(l), *map(int, c)) <= l


def child_tile_restated(pc, pt, off):
    """PoissonTile::childTile: child cell (i, j, k) takes the parent cell ((8*o + i) >> 1, ...)."""
    i, j, k = np.meshgrid(np.arange(8), np.arange(8), np.arange(8), indexing="ij")
    pi, pj, pk = (8 * off[0] + i) >> 1, (8 * off[1] + j) >> 1, (8 * off[2] + k) >> 1
    src = (pi * 64 + pj * 8 + pk).ravel()
    return pc[:, src], pt[src]


def test_child_tile_hand_down_matches_reference():
    rng = np.random.default_rng(3)
    pc = rng.standard_normal((15, 512)).astype(np.float32)
    pt = rng.integers(0, 8, 512).astype(np.uint8)
    for o in range(8):
        off = (o & 1, (o >> 1) & 1, (o >> 2) & 1)
        cc, ct = R.child_tile(pc, pt, off)
        wc, wt = child_tile_restated(pc, pt, off)
        assert np.array_equal(bits(cc), bits(wc)) and np.array_equal(ct, wt)


def sphere_system(nonleaf_types=None, mask=False, from_leafs=False, prm=None):
    g = O.Grid(0.125, 10)
    g.set_tile(0, 0, 0, 0, O.LEAF)
    g.rebuild()
    g.refine_case(O.CASE_SHELL, prm or shell_params(4, 5, 6))
    g.alloc(16)
    g.set_leaf_cell_types_case(O.CASE_UNIFORM)
    lv, ijk, ty = g.tiles()
    if from_leafs:
        g.calc_cell_types_from_leafs()
    if nonleaf_types is not None:
        ct = g.cell_types()
        ct[ty == O.NONLEAF] = nonleaf_types(int((ty == O.NONLEAF).sum()))
    g.set_reference_mask(mask)
    g.cutcell_sphere_coeffs(COEFF, [(0.5, 0.5, 0.5, 0.1)], 0.5)
    return g, lv, ijk, ty


def test_reference_mask_is_open_once_nonleaf_types_come_from_the_leaves():
    prm = shell_params(3, 4, 5)
    a, *_ = sphere_system(prm=prm)
    b, *_ = sphere_system(mask=True, from_leafs=True, prm=prm)
    for c in range(4):
        assert np.array_equal(bits(a.channel(COEFF + c)), bits(b.channel(COEFF + c)))
    assert np.array_equal(a.cell_types(), b.cell_types())


def test_unset_nonleaf_types_change_the_coarse_operator_but_keep_diagonals_positive():
    """The reference reads NONLEAF cell types in its coarsening before writing them
    (src/AMGSolver.cu:40-42 before :237).  On the 4/5/6-level sphere octree, zero or
    arbitrary bytes there drop coarse off-diagonals, yet no INTERIOR cell of any level gets
    a zero or negative diagonal -- so such types alone do not explain a non-finite
    Gauss-Seidel update at level 2."""
    open_g, lv, ijk, ty = sphere_system()
    d_open = open_g.channel(COEFF + 3)
    for f in (lambda n: np.zeros((n, 512), np.uint8),
              lambda n: np.random.default_rng(5).integers(0, 256, (n, 512)).astype(np.uint8)):
        g, *_ = sphere_system(nonleaf_types=f, mask=True)
        d, ct = g.channel(COEFF + 3), g.cell_types()
        interior = (ct == O.INTERIOR) & (ty != O.GHOST)[:, None]
        assert np.all(np.isfinite(d[interior])) and d[interior].min() > 0
        coarse = (lv <= 3)[:, None] & interior
        assert not np.array_equal(d[coarse], d_open[coarse])
