"""Refinement keeps and hands down channel data and cell types as the reference does
(refineStep, src/HAGrid.h:1140-1160, with PoissonTile::childTile, src/PoissonTile.h:151-172):
a tile that survives keeps its data, a tile made by refinement takes every cell's value and
type from the cell of its nearest surviving ancestor that contains it, and a new GHOST
tile starts at zero."""
import numpy as np
import pytest

import cmg

pytestmark = pytest.mark.gpu


def _expected(old, lv, ijk, ty, data0, types0, ty0):
    n = len(lv)
    exp = np.zeros((n, 512), np.float32)
    expt = np.zeros((n, 512), np.uint8)
    l = np.arange(512)
    li, lj, lk = l >> 6, (l >> 3) & 7, l & 7
    for t in range(n):
        key = (int(lv[t]), tuple(int(v) for v in ijk[t]))
        o = old.get(key)
        if o is not None and (ty0[o] != cmg.GHOST or ty[t] == cmg.GHOST):
            exp[t], expt[t] = data0[o], types0[o]
            continue
        if ty[t] == cmg.GHOST:
            continue
        for s in range(1, int(lv[t]) + 1):
            c = ijk[t] >> s
            oa = old.get((int(lv[t]) - s, tuple(int(v) for v in c)))
            if oa is not None and ty0[oa] != cmg.GHOST:
                gi = ((ijk[t][0] * 8 + li) >> s) - c[0] * 8
                gj = ((ijk[t][1] * 8 + lj) >> s) - c[1] * 8
                gk = ((ijk[t][2] * 8 + lk) >> s) - c[2] * 8
                src = gi * 64 + gj * 8 + gk
                exp[t], expt[t] = data0[oa][src], types0[oa][src]
                break
    return exp, expt


@pytest.mark.parametrize("fine", [3, 5])
def test_refinement_hands_down_parent_data(fine):
    G = cmg.HADeviceGrid(0.125, 10, 16)
    G.set_tile_host(0, (0, 0, 0), cmg.LEAF)
    G.rebuild()
    G.refine_case(cmg.CASE_UNIFORM, [2, 2])
    rng = np.random.default_rng(7)
    n0 = G.num_tiles
    data0 = rng.standard_normal((n0, 512)).astype(np.float32)
    types0 = rng.choice(np.array([cmg.DIRICHLET, cmg.INTERIOR, cmg.NEUMANN], np.uint8), size=(n0, 512))
    G.upload(5, data0)
    G.upload_cell_types(types0)
    lv0, ijk0, ty0 = G.tiles()
    old = {(int(l), tuple(int(v) for v in c)): i for i, (l, c) in enumerate(zip(lv0, ijk0))}
    G.refine_case(cmg.CASE_MULTI_SPHERE, [2, fine, 0.05, 1, 0.5, 0.5, 0.5, 0.2])
    lv, ijk, ty = G.tiles()
    assert len(lv) > n0 and int(lv.max()) == fine
    exp, expt = _expected(old, lv, ijk, ty, data0, types0, ty0)
    assert np.array_equal(G.download(5), exp)
    assert np.array_equal(G.download_cell_types(), expt)
