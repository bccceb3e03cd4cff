"""The CUDA product against the golden fixtures of tests/golden (written from the oracle by
tests/golden/make_golden.py): the 32^3 solve and the learned smoother's network."""
import os
import sys

import numpy as np
import pytest

import cmg

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_uniform32_solve_matches_golden():
    d = np.load(os.path.join(GOLDEN, "uniform32.npz"))
    G = cmg.HADeviceGrid(0.125, 10, 16)
    G.set_tile_host(0, (0, 0, 0), cmg.LEAF)
    G.rebuild()
    G.refine_case(cmg.CASE_UNIFORM, [2, 2])
    G.set_leaf_cell_types_case(cmg.CASE_UNIFORM)
    solver = cmg.AMGSolver(6, 0.5, 1.0, 1.0)
    solver.prepareTypesAndCoeffs(G)
    _, _, ty = G.tiles()
    sys.path.insert(0, GOLDEN)
    import make_golden as M

    G.upload(1, M.uniform32_rhs(ty))
    it, rel = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
    x = G.download(0)[ty == cmg.LEAF]
    assert rel < 1e-6 and abs(it - int(d["oracle_iters"])) <= 1
    assert np.linalg.norm(x - d["x64"]) <= 1e-5 * np.linalg.norm(d["x64"])


def test_learned_net_matches_golden():
    d = np.load(os.path.join(GOLDEN, "learned_h8.npz"))
    net = cmg.LearnedNet(8, seed=0)
    net.set_params(d["params"])
    net.set_loss("energy")
    net.set_samples(d["rho"], d["diag"], d["types"], d["target"])
    out = net.forward()
    for s in range(out.shape[0]):
        m = np.abs(d["forward"][s]).max()
        assert np.abs(out[s] - d["forward"][s]).max() <= 1e-2 * m + 1e-30
    loss, g = net.gradient()
    assert abs(loss - float(d["loss"])) <= 1e-3 * float(d["loss"])
    assert np.linalg.norm(g - d["grad"]) <= 2e-2 * np.linalg.norm(d["grad"])
