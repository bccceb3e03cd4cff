"""Batched solves (cmg_amg_solve_batch): many independent octrees solved together, each
on its own stream, must give exactly what solving them one by one gives."""
import numpy as np
import pytest

import cmg
from workloads import setup_shell, setup_uniform, shell_params

pytestmark = pytest.mark.gpu


def _instances():
    out = []
    G, _, S, _ = setup_uniform(2, with_oracle=False)
    out.append((G, S))
    G, _, S = setup_shell(shell_params(coarse=3, mid=4, fine=5), with_oracle=False)
    out.append((G, S))
    G, _, S = setup_shell(shell_params(coarse=3, mid=4, fine=5, center=(0.45, 0.5, 0.55), r=0.15), seed=2,
                          spheres=((0.45, 0.5, 0.55, 0.15),), with_oracle=False)
    out.append((G, S))
    return out


def test_batched_solves_match_one_by_one():
    import torch

    inst = _instances()
    bs = [G.download(1) for G, _ in inst]
    ref = []
    for (G, S), b in zip(inst, bs):
        G.upload(1, b)
        it, rel = S.solve(G, False, 100, 1e-6, 2, 10, 1, False)
        ref.append((it, rel, G.download(0)))
    streams = [torch.cuda.Stream() for _ in inst]
    for (G, _), st in zip(inst, streams):
        G.set_stream(st.cuda_stream)
    # device buffers: b restored in channel 1, x read from channel 0
    for (G, _), b in zip(inst, bs):
        G.upload(1, b)
        G.synchronize()
    its, rels, ms = cmg.solve_batch([S for _, S in inst], [G for G, _ in inst], 100, 1e-6, 2, 10, 1, False)
    for (G, _), r, it, rel, t in zip(inst, ref, its, rels, ms):
        assert (it, rel) == r[:2]
        assert np.array_equal(G.download(0), r[2])
        assert t > 0.0
    # host buffers: b copied in and x copied out inside the call
    b_host = [torch.from_numpy(b.ravel().copy()).pin_memory() for b in bs]
    x_host = [torch.zeros_like(b).pin_memory() for b in b_host]
    its, rels, _ = cmg.solve_batch([S for _, S in inst], [G for G, _ in inst], 100, 1e-6, 2, 10, 1, False,
                                   b_host=[b.data_ptr() for b in b_host], x_host=[x.data_ptr() for x in x_host])
    for r, it, rel, x in zip(ref, its, rels, x_host):
        assert (it, rel) == r[:2]
        assert np.array_equal(x.numpy().reshape(r[2].shape), r[2])
    for G, _ in inst:
        G.set_stream(0)


def test_batch_rejects_a_repeated_solver():
    inst = _instances()[:2]
    S = inst[0][1]
    with pytest.raises(cmg.CmgError):
        cmg.solve_batch([S, S], [G for G, _ in inst], 100, 1e-6, 2, 10, 1, False)


def test_solver_reused_across_destroyed_and_recreated_grids():
    """One solver, grids destroyed and created in turn (a new grid may take a destroyed one's
    address): every solve equals a solve by a fresh solver on the same grid."""
    import gc

    from workloads import COEFF

    solver = cmg.AMGSolver(COEFF, 0.5, 1.0, 1.0)
    for c in [(0.5, 0.5, 0.5), (0.55, 0.5, 0.5), (0.5, 0.5, 0.5)]:
        G, _, _ = setup_shell(shell_params(3, 4, 5, c, 0.1), spheres=[c + (0.1,)], with_oracle=False)
        b = G.download(1)
        it, rel = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
        x = G.download(0)
        G.upload(1, b)
        fresh = cmg.AMGSolver(COEFF, 0.5, 1.0, 1.0)
        it2, rel2 = fresh.solve(G, False, 100, 1e-6, 2, 10, 1, False)
        assert it == it2 and rel == rel2 and np.array_equal(x, G.download(0))
        del G, fresh
        gc.collect()
