"""The octree built on the device (cmg_grid_refine_case_device: refinement flags, new tiles,
ghost layer, canonical order and tables in device memory) against the host builder that
the CPU tests pin to the oracle: the same tiles in the same order with the same tables, for
every built-in case, for a second refinement of an already refined tree, and through a
whole solve."""
import numpy as np
import pytest

import cmg
from workloads import COEFF, shell_params

pytestmark = pytest.mark.gpu

CASES = [
    (cmg.CASE_UNIFORM, [3, 3]),
    (cmg.CASE_CENTER_POINT, [2, 6]),
    (cmg.CASE_SPHERE_EMPTY, [2, 5]),
    (cmg.CASE_SPHERE_SOLID, [2, 5]),
    (cmg.CASE_STAR_EMPTY, [3, 5]),  # refined on the host by the device entry point
    (cmg.CASE_SHELL, shell_params(4, 5, 6)),
    (cmg.CASE_SHELL, shell_params(3, 4, 5, center=(0.73, 0.41, 0.5))),
    (cmg.CASE_MULTI_SPHERE, [3, 5, 0.05, 3, 0.3, 0.3, 0.4, 0.08, 0.7, 0.6, 0.5, 0.12, 0.5, 0.75, 0.3, 0.06]),
]


def _grid(case_id, prm, on_device, first=None):
    G = cmg.HADeviceGrid(0.125, 10, 16)
    G.set_tile_host(0, (0, 0, 0), cmg.LEAF)
    G.rebuild()
    if first is not None:
        G.refine_case(first[0], first[1], on_device=on_device)
    G.refine_case(case_id, prm, on_device=on_device)
    return G


def _same_topology(A, B):
    for a, b in zip(A.tiles(), B.tiles()):
        assert np.array_equal(a, b)
    for a, b in zip(A.tables(), B.tables()):
        assert np.array_equal(a, b)
    assert A.info() == B.info()


@pytest.mark.parametrize("case_id,prm", CASES)
def test_device_octree_equals_host_octree(case_id, prm):
    _same_topology(_grid(case_id, prm, True), _grid(case_id, prm, False))


def test_device_refinement_of_a_refined_tree():
    first = (cmg.CASE_UNIFORM, [2, 2])
    prm = shell_params(3, 4, 5, center=(0.6, 0.45, 0.52))
    _same_topology(_grid(cmg.CASE_SHELL, prm, True, first), _grid(cmg.CASE_SHELL, prm, False, first))


def test_device_built_octree_solves_identically():
    prm = shell_params(3, 4, 5)
    out = []
    for on_device in (False, True):
        G = _grid(cmg.CASE_SHELL, prm, on_device)
        G.set_leaf_cell_types_case(cmg.CASE_UNIFORM)
        G.cutcell_sphere_coeffs(COEFF, [(0.5, 0.5, 0.5, 0.1)], 0.5)
        rng = np.random.default_rng(4)
        b = rng.standard_normal((G.num_tiles, 512)).astype(np.float32)
        b[G.tiles()[2] != cmg.LEAF] = 0
        b[G.download_cell_types() != cmg.INTERIOR] = 0
        G.upload(1, b)
        S = cmg.AMGSolver(COEFF, 0.5, 1.0, 1.0)
        it, rel = S.solve(G, False, 100, 1e-6, 2, 10, 1, False)
        out.append((it, rel, G.download(0)))
    assert out[0][:2] == out[1][:2] and np.array_equal(out[0][2], out[1][2])


def test_rebuilt_octrees_reuse_pool_memory():
    """Octrees rebuilt one after another around a moving sphere (each one built while the
    previous one still exists, then the previous one destroyed) take back the pool blocks
    that earlier ones freed: the tile counts differ, but the planes are allocated in size
    classes.  Device memory grows by less than one octree's planes after the first octrees,
    and not at all when the sphere moves back over positions already seen."""
    import torch

    free, counts, G = [], [], None
    ks = list(range(10)) + list(range(9, -1, -1))
    for k in ks:
        c = (0.42 + 0.02 * k, 0.5, 0.5)
        Gn = _grid(cmg.CASE_SHELL, shell_params(3, 4, 5, center=c), True)
        Gn.set_leaf_cell_types_case(cmg.CASE_UNIFORM)
        Gn.synchronize()
        G = Gn
        del Gn
        counts.append(G.num_tiles)
        free.append(torch.cuda.mem_get_info()[0])
    assert len(set(counts)) > 1, counts
    planes = 16 * 512 * 4 * min(counts)
    grown = [free[3] - f for f in free]
    assert max(grown[3:10]) < planes, (grown, planes)
    assert free[-1] == free[9], grown
