"""Seeded workloads shared by the tests: the same octree and right-hand side
built by the CUDA product (through the C ABI) and by the CPU oracle.

Workloads (synthetic, seeded; the reference publishes no dataset):
  uniform(L)   uniform (8*2^L)^3 grid, all INTERIOR, Dirichlet walls, rhs N(0,1)
               from numpy default_rng(seed), mean removed (64^3 is L = 3).
  shell(...)   octree refined to `fine` within `bf` of a solid sphere surface,
               to `mid` within `bm`, else `coarse`; the sphere is a Neumann
               cut-cell boundary; rhs = divergence of 16 random Fourier modes.
"""
import numpy as np

import cmg
from oracle import oracle as O

COEFF = 6  # coefficient channels 6..9 (the reference tests use 6, SolverTests.cu:1857)
U = 10     # face-velocity channels 10..12


def same_bits(a, b):
    """Bitwise equality of float arrays (np.array_equal treats -0.0 and 0.0 as equal)."""
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


def fourier_modes(seed, n=16):
    rng = np.random.default_rng(seed)
    k = rng.integers(1, 9, size=(n, 3)).astype(np.float64)
    amp = rng.standard_normal((n, 3))
    ph = rng.uniform(0.0, 2.0 * np.pi, n)
    return k, amp, ph


def shell_params(coarse=4, mid=5, fine=6, center=(0.5, 0.5, 0.5), r=0.1, bf=0.05, bm=0.15):
    return [coarse, fine, mid, center[0], center[1], center[2], r, bf, bm]


def build_product(case_id, params, h0=0.125, nlev=10, nch=16):
    G = cmg.HADeviceGrid(h0, nlev, nch)
    G.set_tile_host(0, (0, 0, 0), cmg.LEAF)
    G.rebuild()
    G.refine_case(case_id, params)
    return G


def build_oracle(case_id, params, h0=0.125, nlev=10, nch=16):
    g = O.Grid(h0, nlev)
    g.set_tile(0, 0, 0, 0, O.LEAF)
    g.rebuild()
    g.refine_case(case_id, params)
    g.alloc(nch)
    return g


def uniform_rhs(leaf_mask, seed=0):
    rng = np.random.default_rng(seed)
    n = int(leaf_mask.sum())
    v = rng.standard_normal(n * 512).astype(np.float32)
    v -= v.mean(dtype=np.float64).astype(np.float32)
    b = np.zeros((leaf_mask.size, 512), np.float32)
    b[leaf_mask] = v.reshape(n, 512)
    return b


def setup_uniform(L=3, seed=0, with_oracle=True):
    """64^3 for L = 3: both sides prepared, rhs uploaded into channel 1."""
    prm = [L, L]
    G = build_product(cmg.CASE_UNIFORM, prm)
    lv, ijk, ty = G.tiles()
    G.set_leaf_cell_types_case(cmg.CASE_UNIFORM)
    solver = cmg.AMGSolver(COEFF, 0.5, 1.0, 1.0)
    solver.prepareTypesAndCoeffs(G)
    b = uniform_rhs(ty == cmg.LEAF, seed)
    G.upload(1, b)
    g = None
    if with_oracle:
        g = build_oracle(cmg.CASE_UNIFORM, prm)
        g.set_leaf_cell_types_case(O.CASE_UNIFORM)
        g.coarsen_types_and_coeffs(COEFF, 0.5)
        g.channel(1)[:] = b
    return G, g, solver, b


def setup_shell(params, seed=1, spheres=((0.5, 0.5, 0.5, 0.1),), with_oracle=True):
    G = build_product(cmg.CASE_SHELL, params)
    G.set_leaf_cell_types_case(cmg.CASE_UNIFORM)
    G.cutcell_sphere_coeffs(COEFF, spheres, 0.5)
    k, amp, ph = fourier_modes(seed)
    G.face_velocity_fourier(U, k, amp, ph)
    G.divergence(U, COEFF, 1)
    solver = cmg.AMGSolver(COEFF, 0.5, 1.0, 1.0)
    g = None
    if with_oracle:
        g = build_oracle(cmg.CASE_SHELL, params)
        g.set_leaf_cell_types_case(O.CASE_UNIFORM)
        g.cutcell_sphere_coeffs(COEFF, spheres, 0.5)
        g.face_velocity_fourier(U, k, amp, ph)
        g.divergence(U, COEFF, 1)
    return G, g, solver


def boundary_rule_types(lv, ijk, ty, nb):
    """Cell types of the reference's recovery and flux tests (tests/SolverTests.cu:283-303, 387-411):
    a LEAF cell with an empty same-level neighbour on the -x side is NEUMANN, on any other
    side DIRICHLET, otherwise INTERIOR.  nb: [n][>=6] face neighbours (-x,-y,-z,+x,+y,+z)."""
    v = np.arange(512)
    l = np.stack([v >> 6, (v >> 3) & 7, v & 7], axis=1)
    n = len(lv)
    neu = np.zeros((n, 512), bool)
    dir_ = np.zeros((n, 512), bool)
    for axis in range(3):
        lo = (l[:, axis] == 0)[None, :] & (nb[:, axis] < 0)[:, None]
        hi = (l[:, axis] == 7)[None, :] & (nb[:, 3 + axis] < 0)[:, None]
        if axis == 0:
            neu |= lo
        else:
            dir_ |= lo
        dir_ |= hi
    ct = np.full((n, 512), 2, np.uint8)
    ct[dir_] = 1
    ct[neu] = 4
    return ct


def cell_centres(lv, ijk, h0=0.125):
    v = np.arange(512)
    l = np.stack([v >> 6, (v >> 3) & 7, v & 7], axis=1)
    h = (h0 / (2.0 ** lv)).astype(np.float32)
    gc = ijk[:, None, :] * 8 + l[None, :, :]
    return ((gc + 0.5) * h[:, None, None]).astype(np.float32)


def recovery_fields(lv, ijk, ty, ct):
    """x_true = exp(x) sin(y) on INTERIOR cells of LEAF tiles (tests/SolverTests.cu:412-415)."""
    xc = cell_centres(lv, ijk)
    f = (np.exp(xc[..., 0]) * np.sin(xc[..., 1])).astype(np.float32)
    f[(ty != 1)] = 0
    f[ct != 2] = 0
    return f


def flux_fields(lv, ijk, ty, ct):
    """x = sin(-2.5 x + y + 7 z) on INTERIOR cells (tests/SolverTests.cu:292-295)."""
    xc = cell_centres(lv, ijk)
    f = np.sin(-2.5 * xc[..., 0] + xc[..., 1] + 7 * xc[..., 2]).astype(np.float32)
    f[(ty != 1)] = 0
    f[ct != 2] = 0
    return f


def away_from_walls(lv, ijk):
    """Cells whose 6 neighbours lie inside the domain.  The divergence treats the outer
    wall as closed (empty neighbour: u = 0, src/AMGSolver.cu:813-816) while the Laplacian
    treats it as a Dirichlet wall, so the projection is exact only away from it."""
    v = np.arange(512)
    l = np.stack([v >> 6, (v >> 3) & 7, v & 7], axis=1)
    gc = ijk[:, None, :] * 8 + l[None]
    nmax = (8 << lv.astype(np.int64))[:, None, None] - 1
    return ~((gc == 0) | (gc == nmax)).any(-1)


def projected_divergence(download, lv, ijk, ty, ct, b0, div_ch):
    """|div u_projected|_2 / |div u|_2 over INTERIOR leaf cells away from the outer walls."""
    m = (ty[:, None] == 1) & (ct == 2) & away_from_walls(lv, ijk)
    d0 = np.linalg.norm(b0[m].astype(np.float64))
    d1 = np.linalg.norm(download(div_ch)[m].astype(np.float64))
    return d1 / d0


def pure_neumann_setup(lv, ijk, ty, seed=4):
    """LEAF cell types with the outer layer of the domain NEUMANN (no Dirichlet cell anywhere:
    the operator is singular) and a zero-mean rhs on the INTERIOR cells."""
    ct = np.where(~away_from_walls(lv, ijk), 4, 2).astype(np.uint8)
    ct[ty != 1] = 0
    m = (ty[:, None] == 1) & (ct == 2)
    rng = np.random.default_rng(seed)
    b = np.zeros((len(lv), 512), np.float32)
    b[m] = rng.standard_normal(int(m.sum())).astype(np.float32)
    b[m] -= b[m].mean(dtype=np.float64).astype(np.float32)
    return ct, b
