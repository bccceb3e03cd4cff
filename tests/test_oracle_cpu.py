"""CPU checks of the oracle against the reference's own known-answer tests.

The reference stores no golden vectors for this path; its tests are analytic
(tests/SolverTests.cu).  These restate them on the oracle:
  * operator structure on a uniform grid (7-point, -h off-diagonal, 6h diagonal
    with Dirichlet walls folded in, symmetric);
  * discrete-Laplacian truncation error against an analytic -lap f * h^3
    (TestDiscretizedLaplacian, tests/SolverTests.cu:1282-1361): second order;
  * refinement rules: 2:1 face balance, GHOST parents are LEAF
    (src/HAGrid.h:856-889, 1088-1170);
  * the oracle's FAS mu-cycle PCG converges to 1e-6 and agrees with the FP64
    CSR solution of the same operator (a 1e-5 relative bar).
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

COEFF = 6


def uniform_grid(L):
    g = O.Grid(0.125, 10)
    g.set_tile(0, 0, 0, 0, O.LEAF)
    g.rebuild()
    g.refine_case(O.CASE_UNIFORM, [L, L])
    g.alloc(16)
    g.set_leaf_cell_types_case(O.CASE_UNIFORM)
    g.coarsen_types_and_coeffs(COEFF, 0.5)
    return g


def cell_centres(g):
    lv, ijk, ty = g.tiles()
    v = np.arange(512)
    l = np.stack([v >> 6, (v >> 3) & 7, v & 7], axis=1)
    h = 0.125 / (2.0 ** lv)
    gc = ijk[:, None, :] * 8 + l[None, :, :]
    return (gc + 0.5) * h[:, None, None], h


def test_uniform_tile_counts():
    g = uniform_grid(3)
    lv, ijk, ty = g.tiles()
    assert g.n == 585
    for L, (nleaf, nnon) in enumerate([(0, 1), (0, 8), (0, 64), (512, 0)]):
        assert int(((lv == L) & (ty == O.LEAF)).sum()) == nleaf
        assert int(((lv == L) & (ty == O.NONLEAF)).sum()) == nnon
    assert not np.any(ty == O.GHOST)


def test_uniform_operator_values_and_symmetry():
    g = uniform_grid(3)
    lv, ijk, ty = g.tiles()
    leaf = ty == O.LEAF
    h = 0.125 / 8
    assert np.all(g.channel(COEFF + 3)[leaf] == np.float32(6 * h))
    for a in range(3):
        assert set(np.unique(g.channel(COEFF + a)[leaf]).tolist()) == {np.float32(-h)}
    # NONLEAF levels: scaled Galerkin coarsening keeps the 7-point form at 2h
    lev2 = lv == 2
    assert np.all(g.channel(COEFF + 3)[lev2] == np.float32(6 * 2 * h))
    rp, ci, va, rt, rc = g.assemble(COEFF)
    import scipy.sparse as sp

    n = len(rp) - 1
    A = sp.csr_matrix((va, ci, rp), shape=(n, n))
    assert n == 64 ** 3
    assert abs(A - A.T).max() == 0.0
    # row sums: 0 inside, k*h for a cell touching k Dirichlet walls
    rs = np.asarray(A.sum(axis=1)).ravel()
    assert np.allclose(np.unique(np.round(rs / h, 6)), [0, 1, 2, 3])


@pytest.mark.parametrize("L", [2])
def test_truncation_error_second_order(L):
    """A f versus -lap f * h^3 for f = sin(pi x) sin(pi y) sin(pi z) (zero on the walls).
    Levels 2 -> 3: finer than that the float32 operator apply (the stencil cancels
    ~6/(3 pi^2 h^2) = O(1e3)) reaches round-off."""
    errs = []
    for lev in (L, L + 1):
        g = uniform_grid(lev)
        xc, h = cell_centres(g)
        f = np.sin(np.pi * xc[..., 0]) * np.sin(np.pi * xc[..., 1]) * np.sin(np.pi * xc[..., 2])
        g.channel(2)[:] = f.astype(np.float32)
        g.full_neg_lap_leafs(2, COEFF, 3)
        lv, ijk, ty = g.tiles()
        leaf = ty == O.LEAF
        exact = 3 * np.pi ** 2 * f * (h[:, None] ** 3)
        # the Dirichlet wall sits at the empty neighbour's cell centre (AMGSolver.cu:489-493),
        # a first-order boundary treatment; the second-order rate holds away from the walls
        far = np.all((xc > 2 * h[:, None, None]) & (xc < 1 - 2 * h[:, None, None]), axis=-1)
        sel = leaf[:, None] & far
        e = np.abs(g.channel(3)[sel] - exact[sel]).mean() / np.abs(exact[sel]).mean()
        errs.append(e)
    assert errs[1] < errs[0] / 3.0, errs  # halving h cuts the error ~4x


@pytest.mark.parametrize("case_id,prm", [(O.CASE_SPHERE_EMPTY, [2, 5]), (O.CASE_STAR_SOLID, [2, 5]), (O.CASE_SHELL, [3, 5, 4, 0.5, 0.5, 0.5, 0.1, 0.05, 0.15])])
def test_refinement_rules(case_id, prm):
    g = O.Grid(0.125, 10)
    g.set_tile(0, 0, 0, 0, O.LEAF)
    g.rebuild()
    g.refine_case(case_id, prm)
    lv, ijk, ty = g.tiles()
    nbr, par, ch = g.tables()
    for t in range(g.n):
        if ty[t] == O.GHOST:
            assert par[t] >= 0 and ty[par[t]] == O.LEAF
        if ty[t] == O.LEAF:
            for a in range(6):
                q = nbr[t, a]
                if q >= 0 and ty[q] == O.NONLEAF:
                    axis, plus = a % 3, a // 3
                    for ci in range(8):
                        bit = (ci >> (2 - axis)) & 1
                        if bit == (0 if plus else 1):
                            assert ty[ch[q, ci]] == O.LEAF
    # every LEAF tile's face neighbours are within one level (2:1 balance across faces)
    key = {(int(lv[t]), *map(int, ijk[t])): t for t in range(g.n)}
    for t in np.nonzero(ty == O.LEAF)[0]:
        L = int(lv[t])
        for a in range(6):
            c = list(map(int, ijk[t]))
            c[a % 3] += 1 if a >= 3 else -1
            if (L, *c) in key:
                continue
            # neighbour region not at this level: must be covered by a LEAF one level up
            pc = [x >> 1 for x in c]
            assert (L - 1, *pc) in key or min(c) < 0 or max(c) >= 2 ** L


def test_oracle_solve_matches_fp64():
    g = uniform_grid(2)
    lv, ijk, ty = g.tiles()
    leaf = ty == O.LEAF
    rng = np.random.default_rng(0)
    b = np.zeros((g.n, 512), np.float32)
    b[leaf] = rng.standard_normal((int(leaf.sum()), 512)).astype(np.float32)
    g.channel(1)[:] = b
    it, rel = g.amg_solve(COEFF, omega=1.5, mu=2, max_iters=100, tol=1e-6, level_iters=2, coarsest_iters=10)
    assert rel < 1e-6 and 3 <= it <= 12
    rp, ci, va, rt, rc = g.assemble(COEFF)
    xs, its, rr = O.csr_solve(rp, ci, va, b[rt, rc].astype(np.float64), 1e-12, 5000, 0)
    x = g.channel(0)[rt, rc]
    assert np.linalg.norm(x - xs) / np.linalg.norm(xs) < 1e-5


def test_cutcell_face_fraction_rules():
    """Face fluid fractions: 0 inside the solid, 1 in open fluid, clamped to >= 0.1 when cut (MeshCutCell.cu:405)."""
    g = O.Grid(0.125, 10)
    g.set_tile(0, 0, 0, 0, O.LEAF)
    g.rebuild()
    g.refine_case(O.CASE_SHELL, [3, 4, 3, 0.5, 0.5, 0.5, 0.2, 0.05, 0.05])
    g.alloc(16)
    g.set_leaf_cell_types_case(O.CASE_UNIFORM)
    g.cutcell_sphere_coeffs(COEFF, [[0.5, 0.5, 0.5, 0.2]], 0.5)
    lv, ijk, ty = g.tiles()
    ct = g.cell_types()
    leaf = ty == O.LEAF
    h = (0.125 / 2.0 ** lv)[:, None]
    for a in range(3):
        c = g.channel(COEFF + a)
        ratio = (-c / h)[leaf]
        assert np.all(ratio >= 0) and np.all(ratio <= 1.0 + 1e-6)
        cut = (ratio > 0) & (ratio < 1)
        assert np.all(ratio[cut] >= 0.1 - 1e-7)
    assert np.any(ct[leaf] == O.NEUMANN)
    assert np.all(g.channel(COEFF + 3)[leaf][ct[leaf] == O.NEUMANN] == 0)


def _kat_grid(case_id, prm):
    from workloads import boundary_rule_types

    g = O.Grid(0.125, 10)
    g.set_tile(0, 0, 0, 0, O.LEAF)
    g.rebuild()
    g.refine_case(case_id, prm)
    g.alloc(16)
    lv, ijk, ty = g.tiles()
    nbr, par, ch = g.tables()
    ct = boundary_rule_types(lv, ijk, ty, nbr)
    types = g.cell_types()
    types[ty == O.LEAF] = ct[ty == O.LEAF]
    g.coarsen_types_and_coeffs(COEFF, 0.5)
    return g


@pytest.mark.parametrize("case_id,prm", [(O.CASE_UNIFORM, [2, 2]), (O.CASE_CENTER_POINT, [2, 4])])
def test_kat_neumann_dirichlet_recovery(case_id, prm):
    """TestNeumannDirichletRecovery (tests/SolverTests.cu:363-512): b = A x_true, solve, |x - x_true|_inf < 1e-4."""
    from workloads import recovery_fields

    g = _kat_grid(case_id, prm)
    lv, ijk, ty = g.tiles()
    ct = g.cell_types()
    xt = recovery_fields(lv, ijk, ty, ct)
    g.channel(5)[:] = xt
    g.full_neg_lap_leafs(5, COEFF, 1)
    it, rel = g.amg_solve(COEFF, max_iters=1000, tol=1e-6, level_iters=2, coarsest_iters=10)
    m = (ty[:, None] == O.LEAF) & (ct == O.INTERIOR)
    err = np.abs(g.channel(0)[m] - xt[m]).max()
    assert rel < 1e-6 and err < 1e-4, (it, rel, err)


def test_kat_laplacian_flux_consistency():
    """TestAMGLaplacianAndFluxConsistency (tests/SolverTests.cu:242-361): -lap x + div(grad x) = 0, L_inf < 1e-5."""
    from workloads import flux_fields

    g = _kat_grid(O.CASE_UNIFORM, [2, 2])
    lv, ijk, ty = g.tiles()
    ct = g.cell_types()
    g.channel(0)[:] = flux_fields(lv, ijk, ty, ct)
    for a in range(3):
        g.channel(10 + a)[:] = 0
    g.full_neg_lap_leafs(0, COEFF, 1)
    g.add_gradient_to_face(0, COEFF, 10)
    g.divergence(10, COEFF, 2)
    m = (ty[:, None] == O.LEAF) & (ct == O.INTERIOR)
    diff = np.abs(g.channel(2)[m] + g.channel(1)[m]).max()
    assert diff < 1e-5, diff


def test_kat_projection_divergence_free():
    """Projection on the cut-cell sphere octree (tests/SolverTests.cu:1846-2158): solve
    -lap p = div u, u += grad p, then div u vanishes to the solve tolerance."""
    from workloads import U, fourier_modes, projected_divergence, shell_params

    g = O.Grid(0.125, 10)
    g.set_tile(0, 0, 0, 0, O.LEAF)
    g.rebuild()
    g.refine_case(O.CASE_SHELL, shell_params(2, 3, 4))
    g.alloc(16)
    g.set_leaf_cell_types_case(O.CASE_UNIFORM)
    g.cutcell_sphere_coeffs(COEFF, [(0.5, 0.5, 0.5, 0.1)], 0.5)
    k, amp, ph = fourier_modes(1)
    g.face_velocity_fourier(U, k, amp, ph)
    g.divergence(U, COEFF, 1)
    b0 = g.channel(1).copy()
    it, rel = g.amg_solve(COEFF, max_iters=200, tol=1e-6)
    g.add_gradient_to_face(0, COEFF, U)
    g.divergence(U, COEFF, 13)
    lv, ijk, ty = g.tiles()
    ratio = projected_divergence(g.channel, lv, ijk, ty, g.cell_types(), b0, 13)
    assert rel < 1e-6 and ratio < 1e-5, (it, rel, ratio)


def _geo_grid(case_id, prm, seed=0):
    from workloads import uniform_rhs

    g = O.Grid(0.125, 10)
    g.set_tile(0, 0, 0, 0, O.LEAF)
    g.rebuild()
    g.refine_case(case_id, prm)
    g.alloc(16)
    g.set_leaf_cell_types_case(O.CASE_UNIFORM)
    g.calc_cell_types_from_leafs()
    lv, ijk, ty = g.tiles()
    g.channel(1)[:] = uniform_rhs(ty == O.LEAF, seed)
    return g


@pytest.mark.parametrize("kind", [O.GMG, O.CMG])
@pytest.mark.parametrize("case_id,prm", [(O.CASE_UNIFORM, [2, 2]), (O.CASE_CENTER_POINT, [2, 4])])
def test_geometric_solvers_converge(kind, case_id, prm):
    """GMGSolver / CMGSolver::solve (src/GMGSolver.cu:472, src/CMGSolver.cu:466) with the
    reference test harness's settings (1, 1) (tests/SolverTests.cu:1055,1077)."""
    g = _geo_grid(case_id, prm)
    it, rel = g.geo_solve(kind, 1.0, 1.0, max_iters=100, tol=1e-6, level_iters=2, coarsest_iters=10)
    assert rel < 1e-6 and it < 30, (it, rel)


def test_cmg_operator_equals_amg_finest_operator_on_uniform_grid():
    """On a single-level grid both are h * (6 x - sum of neighbours): equal solutions."""
    g = _geo_grid(O.CASE_UNIFORM, [2, 2])
    b = g.channel(1).copy()
    g.geo_solve(O.CMG, max_iters=100, tol=1e-7)
    xc = g.channel(0).copy()
    g.channel(1)[:] = b
    g.coarsen_types_and_coeffs(COEFF, 0.5)
    g.amg_solve(COEFF, max_iters=100, tol=1e-7)
    lv, ijk, ty = g.tiles()
    m = ty == O.LEAF
    assert np.linalg.norm(xc[m] - g.channel(0)[m]) <= 1e-5 * np.linalg.norm(xc[m])


@pytest.mark.parametrize("kind", [O.GMG, O.CMG])
def test_kat_recovery_geometric(kind):
    """TestNeumannDirichletRecovery (tests/SolverTests.cu:363-512) with the geometric solvers."""
    from workloads import boundary_rule_types, recovery_fields

    g = O.Grid(0.125, 10)
    g.set_tile(0, 0, 0, 0, O.LEAF)
    g.rebuild()
    g.refine_case(O.CASE_UNIFORM, [2, 2])
    g.alloc(16)
    lv, ijk, ty = g.tiles()
    nbr, par, ch = g.tables()
    types = g.cell_types()
    types[ty == O.LEAF] = boundary_rule_types(lv, ijk, ty, nbr)[ty == O.LEAF]
    g.calc_cell_types_from_leafs()
    ct = g.cell_types()
    xt = recovery_fields(lv, ijk, ty, ct)
    g.channel(5)[:] = xt
    g.geo_full_neg_lap(kind, 5, 1)
    it, rel = g.geo_solve(kind, max_iters=1000, tol=1e-6, level_iters=2, coarsest_iters=10)
    m = (ty[:, None] == O.LEAF) & (ct == O.INTERIOR)
    err = np.abs(g.channel(0)[m] - xt[m]).max()
    assert rel < 1e-6 and err < 1e-4, (it, rel, err)


def test_pure_neumann_solve_converges():
    """is_pure_neumann: r recentred to zero mean before every preconditioning (src/AMGSolver.cu:1425,1505)."""
    from workloads import pure_neumann_setup

    g = O.Grid(0.125, 10)
    g.set_tile(0, 0, 0, 0, O.LEAF)
    g.rebuild()
    g.refine_case(O.CASE_CENTER_POINT, [2, 4])
    g.alloc(16)
    lv, ijk, ty = g.tiles()
    ct, b = pure_neumann_setup(lv, ijk, ty)
    g.cell_types()[:] = ct
    g.coarsen_types_and_coeffs(COEFF, 0.5)
    g.channel(1)[:] = b
    it, rel = g.amg_solve(COEFF, max_iters=100, tol=1e-6, pure_neumann=True)
    assert rel < 1e-6 and it < 30


def test_divergence_without_coeff_equals_coefficient_form_on_uniform_faces():
    """AMGVolumeWeightedDivergenceWithoutCoeffOnLeafs (AMGSolver.cu:750-788) weights every face
    by h*h; where every face coefficient is -h (a uniform grid, no cut cells, Dirichlet walls)
    it must equal AMGVolumeWeightedDivergenceOnLeafs (AMGSolver.cu:790-835) bit for bit."""
    from workloads import build_oracle

    g = build_oracle(O.CASE_UNIFORM, [2, 2])
    g.set_leaf_cell_types_case(O.CASE_UNIFORM)
    g.coarsen_types_and_coeffs(COEFF, 0.5)
    rng = np.random.default_rng(3)
    u = [rng.standard_normal(g.channel(10).shape).astype(np.float32) for _ in range(3)]
    for a in range(3):
        g.channel(10 + a)[:] = u[a]
    g.divergence(10, COEFF, 1)
    for a in range(3):
        g.channel(10 + a)[:] = u[a]
    g.divergence_without_coeff(10, 2)
    lv, ijk, ty = g.tiles()
    m = ty == O.LEAF
    assert np.array_equal(g.channel(1)[m], g.channel(2)[m])


@pytest.mark.parametrize("kind", [0, 1])
def test_learned_oracle_gradient_matches_finite_differences(kind):
    """The FP64 restatement of the learned smoother's network: its backward pass against
    central differences of its own loss (no BF16 rounding), on two tiles, for the squared
    error and the energy loss."""
    from oracle import learned_oracle as LO

    H = 8
    rng = np.random.default_rng(0)
    n = 2
    types = np.full((n, 512), LO.INTERIOR, np.uint8)
    types[:, rng.uniform(size=512) < 0.1] = LO.DIRICHLET
    rho = rng.standard_normal((n, 512)).astype(np.float32)
    diag = rng.uniform(0.5, 6.0, (n, 512)).astype(np.float32)
    target = rng.standard_normal((n, 512)).astype(np.float32)
    L = LO.layout(H)
    p = rng.standard_normal(L["n"]) * 0.2
    p[L["B1"]:L["W2"]] = 0.3
    p[L["B2"]:L["W3"]] = 0.3
    _, g = LO.loss_and_grad(p, H, rho, diag, types, target, emulate_bf16=False, kind=kind)
    picks = list(rng.choice(L["n"], 24, replace=False)) + [L["B1"], L["B2"] + 1, L["W3"] + 5]
    eps = 1e-6
    for i in picks:
        if L["W1"] <= i < L["B1"] and (i - L["W1"]) % 8 >= 4:
            continue  # padded input channels: zero input, zero gradient
        q = p.copy()
        q[i] += eps
        lp, _ = LO.loss_and_grad(q, H, rho, diag, types, target, emulate_bf16=False, kind=kind)
        q[i] -= 2 * eps
        lm, _ = LO.loss_and_grad(q, H, rho, diag, types, target, emulate_bf16=False, kind=kind)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(g[i])) + 1e-7, (i, fd, g[i])


def test_learned_oracle_bf16_rounding():
    from oracle import learned_oracle as LO

    v = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -2.5, 0.0, 3.0e38])
    r = LO.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == 1.0 + 2.0 ** -6  # tie to even (upwards)
    assert r[3] == -2.5 and r[4] == 0.0


def _golden(name):
    return np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", name))


def test_oracle_reproduces_golden_uniform32():
    """tests/golden/uniform32.npz (make_golden.py): the oracle's FP32 mu-cycle PCG takes the
    recorded iterations and lands within 1e-5 of the recorded FP64 solution."""
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import make_golden as M

    d = _golden("uniform32.npz")
    g = M.build_uniform32()
    _, _, ty = g.tiles()
    g.channel(1)[:] = M.uniform32_rhs(ty)
    it, rel = g.amg_solve(M.COEFF, max_iters=100, tol=1e-6)
    x = g.channel(0)[ty == O.LEAF]
    assert it == int(d["oracle_iters"]) and rel < 1e-6
    assert np.linalg.norm(x - d["x64"]) <= 1e-5 * np.linalg.norm(d["x64"])


def test_learned_oracle_reproduces_golden():
    """tests/golden/learned_h8.npz: the FP64 restatement of the learned smoother's network
    gives the recorded forward output, energy loss and gradient."""
    from oracle import learned_oracle as LO

    d = _golden("learned_h8.npz")
    fwd = LO.forward(d["params"], 8, d["rho"], d["diag"], d["types"])
    loss, grad = LO.loss_and_grad(d["params"], 8, d["rho"], d["diag"], d["types"], d["target"], kind=1)
    assert np.allclose(fwd, d["forward"], rtol=1e-5, atol=1e-6 * np.abs(d["forward"]).max())
    assert abs(loss - float(d["loss"])) <= 1e-9 * abs(float(d["loss"]))
    assert np.allclose(grad, d["grad"], rtol=1e-5, atol=1e-6 * np.abs(d["grad"]).max())


def test_oracle_bf16_cycle_storage_converges_like_fp32():
    """The mixed-precision cycle of the oracle (x and rhs of levels >= 3 rounded to BF16 at
    every write) on uniform 64^3: the iterations of the FP32 cycle within one, the FP32
    solution within 1e-5."""
    from workloads import build_oracle, uniform_rhs

    g = build_oracle(O.CASE_UNIFORM, [3, 3])
    g.set_leaf_cell_types_case(O.CASE_UNIFORM)
    g.coarsen_types_and_coeffs(COEFF, 0.5)
    b = uniform_rhs(g.tiles()[2] == O.LEAF, 0)
    g.channel(1)[:] = b
    it0, rel0 = g.amg_solve(COEFF, max_iters=100, tol=1e-6)
    x0 = g.channel(0).copy()
    g.channel(1)[:] = b
    g.set_x_bf16(True)
    it1, rel1 = g.amg_solve(COEFF, max_iters=100, tol=1e-6)
    assert rel1 <= 1e-6 and abs(it1 - it0) <= 1
    assert np.linalg.norm((g.channel(0) - x0).astype(np.float64)) <= 1e-5 * np.linalg.norm(x0.astype(np.float64))


@pytest.mark.parametrize("cycle", ["vcycle", "mu1", "mu2", "fcycle"])
@pytest.mark.parametrize("case", ["uniform3", "shell345"])
def test_oracle_cycle_variants_reduce_the_residual(cycle, case):
    """AMGSolver::VCycle, muCycle and FASFCycle (src/AMGSolver.cu:1060-1174, 1358-1387) as the
    oracle restates them: one cycle from x = 0 leaves a residual well below |f| on the LEAF
    tiles' INTERIOR cells, and f itself is left unchanged."""
    from workloads import build_oracle, shell_params, uniform_rhs

    if case == "uniform3":
        g = build_oracle(O.CASE_UNIFORM, [3, 3])
    else:
        g = build_oracle(O.CASE_SHELL, shell_params(3, 4, 5))
    g.set_leaf_cell_types_case(O.CASE_UNIFORM)
    g.coarsen_types_and_coeffs(COEFF, 0.5)
    lv, ijk, ty = g.tiles()
    f = uniform_rhs(ty == O.LEAF, 0)
    g.channel(11)[:] = f
    g.channel(1)[:] = f
    if cycle == "vcycle":
        g.vcycle(0, 11, 1, COEFF, 2, 10, 1.5, 1.0, 1.0)
    elif cycle.startswith("mu"):
        g.mu_cycle(int(cycle[2]), 0, 11, 1, COEFF, 2, 10, 1.5, 1.0, 1.0)
    else:
        g.fas_f_cycle(2, 0, 1, 3, COEFF, 2, 10, 1.5, 1.0, 1.0)
    x = g.channel(0)
    assert np.all(np.isfinite(x))
    g.full_neg_lap_leafs(0, COEFF, 12)
    m = (g.cell_types() == O.INTERIOR) & (ty == O.LEAF)[:, None]
    r = f - g.channel(12)
    assert np.linalg.norm(r[m]) < 0.2 * np.linalg.norm(f[m])
    if cycle != "fcycle":
        assert np.array_equal(g.channel(11), f)


def test_deep_oracle_gradient_matches_finite_differences():
    """The residual net's FP64 restatement (hidden = 32): its analytic gradient against central
    differences of its loss, on parameters of every layer (both loss kinds)."""
    import numpy as np

    from oracle import learned_oracle as LO

    L = LO.layout_deep()
    assert L["n"] == 229248
    rng = np.random.default_rng(0)
    p = rng.normal(size=L["n"]) * 0.05
    rho = rng.normal(size=(2, 512)).astype(np.float32)
    diag = (6 + rng.random((2, 512))).astype(np.float32)
    types = np.full((2, 512), 2, np.uint8)
    types[0, :10] = 1
    tg = rng.normal(size=(2, 512)).astype(np.float32)
    for kind in (0, 1):
        _, g = LO.loss_and_grad_deep(p, rho, diag, types, tg, emulate_bf16=False, kind=kind)
        for idx in (L["W0"] + 9, L["B0"] + 3, L["Wa0"] + 100, L["Ba1"] + 5, L["Wb2"] + 7, L["Bb3"] + 2, L["WO"] + 40):
            e = 1e-6
            pp, pm = p.copy(), p.copy()
            pp[idx] += e
            pm[idx] -= e
            lp, _ = LO.loss_and_grad_deep(pp, rho, diag, types, tg, emulate_bf16=False, kind=kind)
            lm, _ = LO.loss_and_grad_deep(pm, rho, diag, types, tg, emulate_bf16=False, kind=kind)
            fd = (lp - lm) / (2 * e)
            assert abs(fd - g[idx]) <= 1e-6 + 1e-5 * abs(fd), (kind, idx, fd, g[idx])
