"""Many octrees in ONE persistent launch (cmg_batch_*): every octree's result must equal
its one-by-one solve bit for bit, whatever the schedule (blocks per group), with the
solvers' own settings, host buffers, the pure-Neumann recentring and fixed-count solves."""
import numpy as np
import pytest

import cmg
from workloads import COEFF, setup_shell, setup_uniform, shell_params

pytestmark = pytest.mark.gpu


def _instances():
    out = []
    G, _, S, _ = setup_uniform(2, with_oracle=False)
    out.append((G, S))
    G, _, S = setup_shell(shell_params(coarse=3, mid=4, fine=5), with_oracle=False)
    out.append((G, S))
    G, _, S = setup_shell(shell_params(coarse=3, mid=4, fine=5, center=(0.45, 0.5, 0.55), r=0.15), seed=2,
                          spheres=((0.45, 0.5, 0.55, 0.15),), with_oracle=False)
    # a solver with other settings: the instance must be solved with them
    S.omega, S.mu_cycle_repeat_times = 1.3, 1
    out.append((G, S))
    G, _, S, _ = setup_uniform(3, seed=4, with_oracle=False)
    S.finest_iters = 3
    out.append((G, S))
    return out


def _one_by_one(inst, bs, args):
    ref = []
    for (G, S), b in zip(inst, bs):
        G.upload(1, b)
        it, rel = S.solve(G, False, *args)
        ref.append((it, rel, G.download(0)))
    return ref


ARGS = [(100, 1e-6, 2, 10, 1, False), (6, 1e-6, 2, 10, 0, False), (100, 1e-6, 1, 4, 2, True)]


@pytest.mark.parametrize("args", ARGS, ids=["converge", "fixed6", "neumann_stride2"])
def test_persistent_batch_equals_one_by_one(args):
    inst = _instances()
    bs = [G.download(1) for G, _ in inst]
    ref = _one_by_one(inst, bs, args)
    batch = cmg.PersistentBatch([S for _, S in inst], [G for G, _ in inst])
    # uniform groups of 0 (automatic), 1, 2, 3, 8 blocks; groups of their own for the larger
    # octrees (split 0.5 and 1 of the per-block budget); blocks of 4, 6 and 8 slots
    for gb, split, ns in ((0, 0.0, 4), (1, 0.0, 4), (2, 0.0, 6), (3, 0.0, 8), (8, 0.0, 4), (1, 0.5, 8), (2, 1.0, 6)):
        batch.set_schedule(gb, split, ns)
        slots, G_, groups, dedicated, resident = batch.schedule()
        assert slots == ns and resident > 0 and groups >= 1 and G_ * (groups - dedicated) <= resident
        for (G, _), b in zip(inst, bs):
            G.upload(1, b)
        its, rels, ims, bms = batch.solve(*args)
        for (G, _), r, it, rel, t in zip(inst, ref, its, rels, ims):
            assert (it, rel) == r[:2], (gb, split, ns, it, rel, r[:2])
            assert np.array_equal(G.download(0), r[2]), (gb, split, ns)
            assert t > 0.0
        assert bms > 0.0


def test_persistent_batch_host_buffers():
    import torch

    inst = _instances()
    bs = [G.download(1) for G, _ in inst]
    args = ARGS[0]
    ref = _one_by_one(inst, bs, args)
    b_host = [torch.from_numpy(b.ravel().copy()).pin_memory() for b in bs]
    x_host = [torch.zeros_like(b).pin_memory() for b in b_host]
    batch = cmg.PersistentBatch([S for _, S in inst], [G for G, _ in inst])
    its, rels, _, _ = batch.solve(*args, b_host=[b.data_ptr() for b in b_host], x_host=[x.data_ptr() for x in x_host])
    for r, it, rel, x in zip(ref, its, rels, x_host):
        assert (it, rel) == r[:2]
        assert np.array_equal(x.numpy().reshape(r[2].shape), r[2])


def test_persistent_batch_one_solver_for_many_grids_and_autotune():
    inst = _instances()[:3]
    S = cmg.AMGSolver(COEFF, 0.5, 1.0, 1.0)
    bs = [G.download(1) for G, _ in inst]
    ref = []
    for (G, _), b in zip(inst, bs):
        G.upload(1, b)
        ref.append(S.solve(G, False, 100, 1e-6, 2, 10, 1, False) + (G.download(0),))
        G.upload(1, b)
    batch = cmg.PersistentBatch([S] * len(inst), [G for G, _ in inst])
    cands = [1, 2, (1, 0.5), (2, 1.0, 8), (1, 0.0, 6)]
    best, ms = batch.autotune(cands, 100, 1e-6, 2, 10, repeats=1)
    assert best in cands and all(m > 0 for m in ms)
    want = (best,) if isinstance(best, int) else best
    sched = batch.schedule()
    assert sched[1] == want[0] and sched[0] == (want[2] if len(want) > 2 else 4)
    # the right-hand sides are back in place after tuning
    for (G, _), b in zip(inst, bs):
        assert np.array_equal(G.download(1), b)
    its, rels, _, _ = batch.solve(100, 1e-6, 2, 10, 1, False)
    for (G, _), r, it, rel in zip(inst, ref, its, rels):
        assert (it, rel) == r[:2] and np.array_equal(G.download(0), r[2])


def test_persistent_batch_rejects_unsupported_settings():
    inst = _instances()[:2]
    S = inst[0][1]
    batch = cmg.PersistentBatch([S for _, S in inst], [G for G, _ in inst])
    S.set_storage("bf16")
    with pytest.raises(cmg.CmgError):
        batch.solve(100, 1e-6, 2, 10, 1, False)
    S.set_storage("fp32")
    G = inst[0][0]
    with pytest.raises(cmg.CmgError):
        cmg.PersistentBatch([S, S], [G, G])
