"""Parity of the CUDA product (through the C ABI) with the CPU oracle.

Tolerances: the operator set-up is integer/elementwise float work and must be
bit-identical; single stencil passes follow the same float operation order
and are compared at 1e-6 relative to the field's magnitude; whole
multigrid cycles and solves are FP32 iterations and are compared at 1e-5
relative L2, with PCG iteration counts within +-1 (the reference's
tolerance for this path), against both the oracle's float run and the FP64
CSR solution of the same operator.
"""
import numpy as np
import pytest

import cmg
from oracle import oracle as O
from oracle import ref as R
from workloads import COEFF, U, setup_uniform, setup_shell, shell_params, build_product, build_oracle, same_bits

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def leaf_mask(G):
    return G.tiles()[2] == cmg.LEAF


def fp64_solution(g, b_leaf_tiles, method):
    rp, ci, va, rt, rc = g.assemble(COEFF)
    bb = b_leaf_tiles[rt, rc].astype(np.float64)
    x, its, rel = O.csr_solve(rp, ci, va, bb, 1e-12, 50000, method)
    assert rel < 1e-10
    return x, rt, rc


def test_uniform_coefficients_bitwise():
    G, g, solver, b = setup_uniform(3)
    assert np.array_equal(G.download_cell_types(), g.cell_types())
    for a in range(4):
        assert same_bits(G.download(COEFF + a), g.channel(COEFF + a)), f"coefficient channel {a}"


def test_uniform_laplacian_matches_oracle():
    G, g, solver, b = setup_uniform(3)
    rng = np.random.default_rng(5)
    x = rng.standard_normal((G.num_tiles, 512)).astype(np.float32)
    G.upload(2, x)
    g.channel(2)[:] = x
    G.full_neg_lap(2, COEFF, 3)
    g.full_neg_lap_leafs(2, COEFF, 3)
    m = leaf_mask(G)
    ax, axo = G.download(3)[m], g.channel(3)[m]
    assert np.max(np.abs(ax - axo)) <= 1e-6 * np.max(np.abs(axo))


@pytest.mark.parametrize("level", [3, 2, 1, 0])
def test_uniform_gauss_seidel_matches_oracle(level):
    G, g, solver, b = setup_uniform(3)
    rng = np.random.default_rng(7 + level)
    x = rng.standard_normal((G.num_tiles, 512)).astype(np.float32)
    r = rng.standard_normal((G.num_tiles, 512)).astype(np.float32)
    for ch, v in ((4, x), (1, r)):
        G.upload(ch, v)
        g.channel(ch)[:] = v
    solver.gauss_seidel(G, 2, 0, level, 4, 1)
    g.gauss_seidel(2, 0, level, 4, COEFF, 1, 1.5)
    lv = G.tiles()[0]
    sel = lv == level
    xd, xo = G.download(4)[sel], g.channel(4)[sel]
    assert np.max(np.abs(xd - xo)) <= 1e-6 * np.max(np.abs(xo))


def test_uniform_mu_cycle_matches_oracle():
    G, g, solver, b = setup_uniform(3)
    solver.fas_mu_cycle(G, 4, 1, 3, 2, 10)
    g.fas_mu_cycle(2, 4, 1, 3, COEFF, 2, 10, 1.5, 1.0, 1.0)
    m = leaf_mask(G)
    assert rel_l2(G.download(4)[m], g.channel(4)[m]) <= 1e-5


@pytest.mark.parametrize("cycle", ["vcycle", "mu1", "mu2", "fcycle"])
@pytest.mark.parametrize("shell", [False, True])
def test_cycle_variants_match_oracle(cycle, shell):
    """AMGSolver::VCycle, muCycle (repeat 1 and 2) and FASFCycle (src/AMGSolver.cu:1060-1174,
    1358-1387), which nothing in the reference's solve calls: x and the working rhs on every
    tile against the oracle.  The sphere octree has LEAF tiles next to NONLEAF tiles on a
    coarser level (muCycleStep's flux deduction) and GHOST tiles."""
    if shell:
        G, g, solver = setup_shell(shell_params(coarse=3, mid=4, fine=5))
        f = G.download(1)
    else:
        G, g, solver, f = setup_uniform(3)
    for ch, v in ((11, f), (1, f)):
        G.upload(ch, v)
        g.channel(ch)[:] = v
    if cycle == "vcycle":
        solver.VCycle(G, 0, 11, 1, 2, 10)
        g.vcycle(0, 11, 1, COEFF, 2, 10, 1.5, 1.0, 1.0)
    elif cycle.startswith("mu"):
        solver.muCycle(int(cycle[2]), G, 0, 11, 1, 2, 10)
        g.mu_cycle(int(cycle[2]), 0, 11, 1, COEFF, 2, 10, 1.5, 1.0, 1.0)
    else:
        solver.FASFCycle(G, 0, 1, 3, 2, 10)
        g.fas_f_cycle(2, 0, 1, 3, COEFF, 2, 10, 1.5, 1.0, 1.0)
    x, xo = G.download(0), g.channel(0)
    assert np.all(np.isfinite(x))
    assert rel_l2(x, xo) <= 1e-6
    assert rel_l2(G.download(1), g.channel(1)) <= 1e-6
    if cycle != "fcycle":
        assert np.array_equal(G.download(11), f)  # f is read only


@pytest.mark.parametrize("graph", [True, False])
def test_dependent_launch_gives_the_same_bits(graph):
    """The pipelined passes launched as programmatic dependents (the default) or as ordinary
    launches: the same iterations, residual and x, in graph and in stream launch mode."""
    G, _, solver = setup_shell(shell_params(coarse=3, mid=4, fine=5), with_oracle=False)
    b = G.download(1)
    out = []
    try:
        for on in (True, False):
            cmg.set_dependent_launch(on)
            s = cmg.AMGSolver(COEFF, 0.5, 1.0, 1.0)
            s.set_launch_mode(use_graph=graph)
            G.upload(1, b)
            it, rel = s.solve(G, False, 100, 1e-6, 2, 10, 1, False)
            out.append((it, rel, G.download(0)))
    finally:
        cmg.set_dependent_launch(True)
    assert out[0][:2] == out[1][:2]
    assert np.array_equal(out[0][2], out[1][2])


@pytest.mark.parametrize("mu", [2, 1])
def test_uniform_solve_matches_oracle_and_fp64(mu):
    G, g, solver, b = setup_uniform(3)
    solver.mu_cycle_repeat_times = mu
    it, rel = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
    ito, relo = g.amg_solve(COEFF, omega=1.5, mu=mu, max_iters=100, tol=1e-6, level_iters=2, coarsest_iters=10)
    assert rel <= 1e-6 and relo <= 1e-6
    assert abs(it - ito) <= 1
    m = leaf_mask(G)
    x = G.download(0)
    assert rel_l2(x[m], g.channel(0)[m]) <= 1e-5
    xs, rt, rc = fp64_solution(g, b, 0)
    assert rel_l2(x[rt, rc], xs) <= 1e-5


def test_solve_zero_rhs_returns_zero():
    G, g, solver, b = setup_uniform(3, with_oracle=False)
    G.fill(1, 0.0)
    it, rel = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
    assert (it, rel) == (0, 0.0)
    assert not np.any(G.download(0)[leaf_mask(G)])


def test_sync_stride_semantics():
    G, g, solver, b = setup_uniform(3)
    it, rel = solver.solve(G, False, 5, 1e-6, 2, 10, -1, False)
    assert (it, rel) == (5, -1.0)
    G.upload(1, b)
    it3, rel3 = solver.solve(G, False, 100, 1e-6, 2, 10, 3, False)
    ito, relo = g.amg_solve(COEFF, max_iters=100, tol=1e-6, sync_stride=3)
    assert it3 % 3 == 0 and it3 == ito and rel3 <= 1e-6


def test_shell_setup_matches_oracle():
    prm = shell_params(coarse=3, mid=4, fine=5)
    G, g, solver = setup_shell(prm)
    assert np.array_equal(G.download_cell_types(), g.cell_types())
    for a in range(4):
        d, o = G.download(COEFF + a), g.channel(COEFF + a)
        assert same_bits(d, o), f"coefficient channel {a}: max diff {np.max(np.abs(d - o))}"
    bd, bo = G.download(1), g.channel(1)
    assert np.max(np.abs(bd - bo)) <= 1e-5 * np.max(np.abs(bo))


def test_sphere_octree_config2_solve_matches_oracle_and_fp64():
    """The headline octree itself: levels 4/5/6 (128^3/256^3/512^3), cut-cell sphere r = 0.1,
    rhs = divergence of 16 Fourier modes from seed 1, the reference's solver setting."""
    G, g, solver = setup_shell(shell_params(4, 5, 6))
    assert np.array_equal(G.download_cell_types(), g.cell_types())
    for a in range(4):
        assert same_bits(G.download(COEFF + a), g.channel(COEFF + a)), f"coefficient channel {a}"
    b = G.download(1)
    g.channel(1)[:] = b
    it, rel = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
    ito, relo = g.amg_solve(COEFF, max_iters=100, tol=1e-6)
    assert rel <= 1e-6 and relo <= 1e-6 and abs(it - ito) <= 1, (it, ito, rel, relo)
    m = leaf_mask(G)
    x = G.download(0)
    assert rel_l2(x[m], g.channel(0)[m]) <= 1e-5
    xs, rt, rc = fp64_solution(g, b, 1)
    assert rel_l2(x[rt, rc], xs) <= 1e-5


def test_shell_solve_matches_oracle_and_fp64():
    prm = shell_params(coarse=3, mid=4, fine=5)
    G, g, solver = setup_shell(prm)
    b = G.download(1)
    g.channel(1)[:] = b  # identical rhs on both sides
    it, rel = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
    ito, relo = g.amg_solve(COEFF, max_iters=100, tol=1e-6)
    assert rel <= 1e-6 and abs(it - ito) <= 1
    m = leaf_mask(G)
    x = G.download(0)
    assert rel_l2(x[m], g.channel(0)[m]) <= 1e-5
    xs, rt, rc = fp64_solution(g, b, 1)
    assert rel_l2(x[rt, rc], xs) <= 1e-5


@pytest.mark.parametrize("seed", [3, 11])
def test_random_multi_sphere_octree_solve_matches_oracle_and_fp64(seed):
    """A random octree of the batched workload's kind: two or three spheres at random
    centres and radii, refined around each to level 5 from level 3, cut-cell faces of every
    sphere, rhs the divergence of Fourier modes; the same set-up on the GPU and in the
    oracle (bitwise), then the solve against the oracle and the FP64 solution."""
    from workloads import fourier_modes

    rng = np.random.default_rng(seed)
    ns = int(rng.integers(2, 4))
    sph = [tuple(float(v) for v in rng.uniform(0.25, 0.75, 3)) + (float(rng.uniform(0.06, 0.14)),) for _ in range(ns)]
    prm = [3, 5, 0.05, ns] + [v for s_ in sph for v in s_]
    k, amp, ph = fourier_modes(100 + seed)
    G = build_product(cmg.CASE_MULTI_SPHERE, prm)
    G.set_leaf_cell_types_case(cmg.CASE_UNIFORM)
    G.cutcell_sphere_coeffs(COEFF, sph, 0.5)
    G.face_velocity_fourier(U, k, amp, ph)
    G.divergence(U, COEFF, 1)
    g = build_oracle(cmg.CASE_MULTI_SPHERE, prm)
    g.set_leaf_cell_types_case(O.CASE_UNIFORM)
    g.cutcell_sphere_coeffs(COEFF, sph, 0.5)
    g.face_velocity_fourier(U, k, amp, ph)
    g.divergence(U, COEFF, 1)
    assert np.array_equal(G.download_cell_types(), g.cell_types())
    for a in range(4):
        assert same_bits(G.download(COEFF + a), g.channel(COEFF + a)), f"coefficient channel {a}"
    b = G.download(1)
    assert np.abs(b).max() > 0
    g.channel(1)[:] = b
    solver = cmg.AMGSolver(COEFF, 0.5, 1.0, 1.0)
    it, rel = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
    ito, relo = g.amg_solve(COEFF, max_iters=100, tol=1e-6)
    assert rel <= 1e-6 and relo <= 1e-6 and abs(it - ito) <= 1, (it, ito, rel, relo)
    m = leaf_mask(G)
    x = G.download(0)
    assert rel_l2(x[m], g.channel(0)[m]) <= 1e-5
    xs, rt, rc = fp64_solution(g, b, 1)
    assert rel_l2(x[rt, rc], xs) <= 1e-5


@pytest.mark.parametrize("case_id,prm", [(cmg.CASE_SPHERE_SOLID, [2, 4]), (cmg.CASE_STAR_EMPTY, [2, 4]), (cmg.CASE_CENTER_POINT, [2, 5])])
def test_reference_test_grids_solve(case_id, prm):
    """Octrees of tests/TestGrids.cuh solved by both sides (Dirichlet walls, random rhs on INTERIOR cells)."""
    G = build_product(case_id, prm)
    G.set_leaf_cell_types_case(case_id)
    solver = cmg.AMGSolver(COEFF, 0.5, 1.0, 1.0)
    solver.prepareTypesAndCoeffs(G)
    g = build_oracle(case_id, prm)
    g.set_leaf_cell_types_case(case_id)
    g.coarsen_types_and_coeffs(COEFF, 0.5)
    assert np.array_equal(G.download_cell_types(), g.cell_types())
    for a in range(4):
        assert same_bits(G.download(COEFF + a), g.channel(COEFF + a))
    ct = g.cell_types()
    rng = np.random.default_rng(11)
    b = rng.standard_normal(ct.shape).astype(np.float32)
    b[(G.tiles()[2] != cmg.LEAF)] = 0
    b[ct != cmg.INTERIOR] = 0
    G.upload(1, b)
    g.channel(1)[:] = b
    it, rel = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
    ito, relo = g.amg_solve(COEFF, max_iters=100, tol=1e-6)
    assert rel <= 1e-6 and abs(it - ito) <= 1
    m = leaf_mask(G)
    assert rel_l2(G.download(0)[m], g.channel(0)[m]) <= 1e-5


@pytest.mark.skipif(not R.available(), reason=str(R.why_unavailable()))
@pytest.mark.parametrize("name", ["staircase12", "staircase21", "staircase34", "staircase43", "centersource",
                                  "twosources67"])
def test_reference_named_grids_solve(name):
    """tests/SolverTests.cu's named octrees, refined on both sides through the reference's own
    SolverTestsLevelTarget (oracle/_ref), all INTERIOR with Dirichlet walls, random rhs."""
    def target(level, i, j, k):
        return R.solvertests_level_target(name, 0.125, level, (i, j, k))

    G = cmg.HADeviceGrid(0.125, 10, 16)
    G.set_tile_host(0, (0, 0, 0), cmg.LEAF)
    G.rebuild()
    G.iterative_refine(target)
    G.set_leaf_cell_types_case(cmg.CASE_UNIFORM)
    solver = cmg.AMGSolver(COEFF, 0.5, 1.0, 1.0)
    solver.prepareTypesAndCoeffs(G)
    g = O.Grid(0.125, 10)
    g.set_tile(0, 0, 0, 0, O.LEAF)
    g.rebuild()
    g.iterative_refine(target)
    g.alloc(16)
    g.set_leaf_cell_types_case(O.CASE_UNIFORM)
    g.coarsen_types_and_coeffs(COEFF, 0.5)
    for a, b in zip(G.tiles(), g.tiles()):
        assert np.array_equal(a, b)
    assert np.array_equal(G.download_cell_types(), g.cell_types())
    for a in range(4):
        assert same_bits(G.download(COEFF + a), g.channel(COEFF + a))
    rng = np.random.default_rng(12)
    b = rng.standard_normal(g.cell_types().shape).astype(np.float32)
    b[G.tiles()[2] != cmg.LEAF] = 0
    G.upload(1, b)
    g.channel(1)[:] = b
    it, rel = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
    ito, relo = g.amg_solve(COEFF, max_iters=100, tol=1e-6)
    assert rel <= 1e-6 and abs(it - ito) <= 1, (it, ito)
    m = leaf_mask(G)
    assert rel_l2(G.download(0)[m], g.channel(0)[m]) <= 1e-5


@pytest.mark.parametrize("L", [0, 1, 2])
def test_shallow_trees_match_oracle(L):
    """Trees of 1, 9 and 73 tiles: the coarse-level kernel runs the whole cycle (levels 0 and 1)."""
    G, g, solver, b = setup_uniform(L)
    it, rel = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
    ito, relo = g.amg_solve(COEFF, max_iters=100, tol=1e-6)
    assert abs(it - ito) <= 1 and rel <= 1e-6
    m = leaf_mask(G)
    assert rel_l2(G.download(0)[m], g.channel(0)[m]) <= 1e-5


def test_graph_and_stream_launch_modes_agree():
    G, g, solver, b = setup_uniform(3, with_oracle=False)
    it1, rel1 = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
    x1 = G.download(0)
    G.upload(1, b)
    solver.set_launch_mode(False)
    it2, rel2 = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
    x2 = G.download(0)
    assert it1 == it2 and rel1 == rel2
    assert np.array_equal(x1, x2)


@pytest.mark.parametrize("shell", [False, True])
def test_persistent_levels_match_per_phase_launches(shell):
    """Levels 2-3 in one cooperative kernel give bit-identical results to one launch per phase."""
    if shell:
        G, g, solver = setup_shell(shell_params(coarse=3, mid=4, fine=5), with_oracle=False)
        b = G.download(1)
    else:
        G, g, solver, b = setup_uniform(3, with_oracle=False)
    solver.set_launch_mode(use_graph=True, persistent=False, cluster=False)
    it1, rel1 = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
    x1 = G.download(0)
    G.upload(1, b)
    solver.set_launch_mode(use_graph=True, persistent=True, cluster=False)
    it2, rel2 = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
    x2 = G.download(0)
    assert (it1, rel1) == (it2, rel2)
    assert np.array_equal(x1, x2)


def _kat_product_and_oracle(case_id, prm):
    from workloads import boundary_rule_types

    G = build_product(case_id, prm)
    g = build_oracle(case_id, prm)
    lv, ijk, ty = G.tiles()
    nb, ch = G.tables()
    ct = np.zeros((G.num_tiles, 512), np.uint8)
    leaf = ty == cmg.LEAF
    ct[leaf] = boundary_rule_types(lv, ijk, ty, nb)[leaf]
    G.upload_cell_types(ct)
    g.cell_types()[:] = ct
    solver = cmg.AMGSolver(COEFF, 0.5, 1.0, 1.0)
    solver.prepareTypesAndCoeffs(G)
    g.coarsen_types_and_coeffs(COEFF, 0.5)
    assert np.array_equal(G.download_cell_types(), g.cell_types())
    return G, g, solver


@pytest.mark.parametrize("case_id,prm", [(cmg.CASE_UNIFORM, [2, 2]), (cmg.CASE_CENTER_POINT, [2, 4])])
def test_kat_recovery_on_gpu(case_id, prm):
    """TestNeumannDirichletRecovery (tests/SolverTests.cu:363-512) through the C ABI."""
    from workloads import recovery_fields

    G, g, solver = _kat_product_and_oracle(case_id, prm)
    lv, ijk, ty = G.tiles()
    ct = G.download_cell_types()
    xt = recovery_fields(lv, ijk, ty, ct)
    G.upload(5, xt)
    G.full_neg_lap(5, COEFF, 1)
    it, rel = solver.solve(G, False, 1000, 1e-6, 2, 10, 1, False)
    m = (ty[:, None] == cmg.LEAF) & (ct == cmg.INTERIOR)
    err = np.abs(G.download(0)[m] - xt[m]).max()
    assert rel < 1e-6 and err < 1e-4, (it, rel, err)


def test_divergence_without_coeff_matches_oracle():
    """The coefficient-free divergence the reference's projection calls (FluidEuler.cu:698)
    on the cut-cell shell octree (GHOST and T-junction faces included), bit for bit."""
    G, g, _ = setup_shell(shell_params(coarse=3, mid=4, fine=5))
    rng = np.random.default_rng(9)
    for a in range(3):
        u = rng.standard_normal((G.num_tiles, 512)).astype(np.float32)
        G.upload(U + a, u)
        g.channel(U + a)[:] = u
    G.divergence_without_coeff(U, 13)
    g.divergence_without_coeff(U, 13)
    m = leaf_mask(G)
    assert np.array_equal(G.download(13)[m], g.channel(13)[m])


def test_kat_flux_consistency_on_gpu():
    """TestAMGLaplacianAndFluxConsistency (tests/SolverTests.cu:242-361) through the C ABI, and equal to the oracle."""
    from workloads import flux_fields

    G, g, solver = _kat_product_and_oracle(cmg.CASE_UNIFORM, [2, 2])
    lv, ijk, ty = G.tiles()
    ct = G.download_cell_types()
    x = flux_fields(lv, ijk, ty, ct)
    G.upload(0, x)
    for a in range(3):
        G.fill(10 + a, 0.0)
    G.full_neg_lap(0, COEFF, 1)
    G.add_gradient_to_face(0, COEFF, 10)
    G.divergence(10, COEFF, 2)
    m = (ty[:, None] == cmg.LEAF) & (ct == cmg.INTERIOR)
    assert np.abs(G.download(2)[m] + G.download(1)[m]).max() < 1e-5
    g.channel(0)[:] = x
    g.add_gradient_to_face(0, COEFF, 10)
    for a in range(3):
        ud, uo = G.download(10 + a), g.channel(10 + a)
        assert np.max(np.abs(ud[ty == cmg.LEAF] - uo[ty == cmg.LEAF])) <= 1e-6 * max(1.0, np.max(np.abs(uo)))


@pytest.mark.parametrize("prm", [shell_params(3, 4, 5), shell_params(4, 5, 6)])
def test_kat_projection_on_gpu(prm):
    """Projection (tests/SolverTests.cu:1846-2158) on the cut-cell sphere octree: after
    u += grad p the divergence vanishes to the solve tolerance."""
    from workloads import projected_divergence

    G, _, solver = setup_shell(prm, with_oracle=False)
    lv, ijk, ty = G.tiles()
    b0 = G.download(1)
    it, rel = solver.solve(G, False, 200, 1e-6, 2, 10, 1, False)
    G.add_gradient_to_face(0, COEFF, U)
    G.divergence(U, COEFF, 13)
    ratio = projected_divergence(G.download, lv, ijk, ty, G.download_cell_types(), b0, 13)
    assert rel < 1e-6 and ratio < 1e-5, (it, rel, ratio)


def _mu_cycle_planes(G, solver, cluster, seed, mu, omega, pipeline=True):
    rng = np.random.default_rng(seed)
    n = G.num_tiles
    solver.mu_cycle_repeat_times = mu
    solver.omega = omega
    G.upload(1, rng.standard_normal((n, 512)).astype(np.float32))
    G.upload(3, rng.standard_normal((n, 512)).astype(np.float32))
    G.upload(4, rng.standard_normal((n, 512)).astype(np.float32))
    solver.set_launch_mode(use_graph=False, cluster=cluster, pipeline=pipeline)
    solver.fas_mu_cycle(G, 4, 1, 3, 2, 10)
    return G.download(4), G.download(1), G.download(3)


@pytest.mark.parametrize("grid", ["uniform32", "uniform64", "shell345"])
@pytest.mark.parametrize("mu,omega", [(2, 1.5), (1, 1.5), (2, 1.3)])
def test_cluster_mu_step_matches_per_level_launches(grid, mu, omega):
    """Levels 0-2 in one 8-CTA cluster launch give the same x, rhs and saved x on
    every tile as the per-level launches (levels 2 and 1-0 separately)."""
    if grid == "shell345":
        G, _, solver = setup_shell(shell_params(coarse=3, mid=4, fine=5), with_oracle=False)
    else:
        G, _, solver, _ = setup_uniform(2 if grid == "uniform32" else 3, with_oracle=False)
    a = _mu_cycle_planes(G, solver, True, 11, mu, omega)
    b = _mu_cycle_planes(G, solver, False, 11, mu, omega)
    for pa, pb in zip(a, b):
        assert np.array_equal(pa, pb)


def test_cluster_solve_matches_per_level_launches():
    G, g, solver = setup_shell(shell_params(coarse=3, mid=4, fine=5), with_oracle=False)
    b = G.download(1)
    solver.set_launch_mode(use_graph=True, cluster=False)
    it1, rel1 = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
    n1 = solver.last_solve_launches()
    x1 = G.download(0)
    G.upload(1, b)
    solver.set_launch_mode(use_graph=True, cluster=True)
    it2, rel2 = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
    n2 = solver.last_solve_launches()
    assert n2 < n1  # the cluster path ran
    assert (it1, rel1) == (it2, rel2)
    assert np.array_equal(x1, G.download(0))


@pytest.mark.parametrize("seed", [1, 2])
def test_division_by_reciprocal_is_ieee_exact(seed):
    """The coarse-level Gauss-Seidel divides by multiplying with a double reciprocal;
    on 2^26 adversarial pairs it must equal the IEEE division bit for bit."""
    m, first = cmg.check_division(1 << 26, seed)
    assert m == 0, (m, [hex(v) for v in first])


@pytest.mark.parametrize("grid", ["uniform64", "shell345", "shell456"])
def test_pipelined_smoother_matches_per_tile_launches(grid):
    """The persistent, prefetching smoothing kernel gives the same x, rhs and saved x on
    every tile as one block per tile, through a whole mu-cycle and a whole solve."""
    if grid == "uniform64":
        G, _, solver, _ = setup_uniform(3, with_oracle=False)
    else:
        prm = shell_params(coarse=3, mid=4, fine=5) if grid == "shell345" else shell_params(coarse=4, mid=5, fine=6)
        G, _, solver = setup_shell(prm, with_oracle=False)
    b = G.download(1)
    a = _mu_cycle_planes(G, solver, True, 17, 2, 1.5, pipeline=True)
    c = _mu_cycle_planes(G, solver, True, 17, 2, 1.5, pipeline=False)
    for pa, pc in zip(a, c):
        assert np.array_equal(pa, pc)
    res = []
    for pipeline in (False, True):
        G.upload(1, b)
        solver.set_launch_mode(use_graph=True, pipeline=pipeline)
        it, rel = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
        res.append((it, rel, G.download(0)))
    assert res[0][:2] == res[1][:2]
    assert np.array_equal(res[0][2], res[1][2])


def test_masked_gauss_seidel_entry_matches_plain_sweeps():
    """cmg_amg_gauss_seidel_masked (the cycle's pipelined kernel) gives the same x as
    cmg_amg_gauss_seidel on every level when x is 0 on the cells that are not INTERIOR."""
    G, _, solver = setup_shell(shell_params(coarse=3, mid=4, fine=5), with_oracle=False)
    rng = np.random.default_rng(23)
    n = G.num_tiles
    interior = G.download_cell_types() == cmg.INTERIOR
    x = np.where(interior, rng.standard_normal((n, 512)), 0.0).astype(np.float32)
    G.upload(3, rng.standard_normal((n, 512)).astype(np.float32))
    for level in range(G.max_level + 1):
        for order in (0, 1):
            out = []
            for masked in (False, True):
                G.upload(4, x)
                (solver.gauss_seidel_masked if masked else solver.gauss_seidel)(G, 2, order, level, 4, 3)
                out.append(G.download(4))
            assert np.array_equal(out[0], out[1]), (level, order)


def _geo_pair(case_id, prm, kind, seed=3):
    from workloads import uniform_rhs

    G = build_product(case_id, prm)
    g = build_oracle(case_id, prm)
    G.set_leaf_cell_types_case(cmg.CASE_UNIFORM)
    g.set_leaf_cell_types_case(O.CASE_UNIFORM)
    G.calc_cell_types_from_leafs()
    g.calc_cell_types_from_leafs()
    assert np.array_equal(G.download_cell_types(), g.cell_types())
    lv, ijk, ty = G.tiles()
    b = uniform_rhs(ty == cmg.LEAF, seed)
    G.upload(1, b)
    g.channel(1)[:] = b
    solver = (cmg.GMGSolver if kind == O.GMG else cmg.CMGSolver)(1.0, 1.0)
    return G, g, solver, b


GEO_GRIDS = [(cmg.CASE_UNIFORM, [2, 2]), (cmg.CASE_CENTER_POINT, [2, 4]), (cmg.CASE_SHELL, shell_params(coarse=3, mid=4, fine=5))]


@pytest.mark.parametrize("kind", [O.GMG, O.CMG])
@pytest.mark.parametrize("case_id,prm", GEO_GRIDS)
def test_geometric_operator_smoother_and_vcycle_match_oracle(kind, case_id, prm):
    G, g, solver, b = _geo_pair(case_id, prm, kind)
    rng = np.random.default_rng(9)
    x = rng.standard_normal((G.num_tiles, 512)).astype(np.float32)
    G.upload(5, x)
    g.channel(5)[:] = x
    solver.full_neg_lap(G, 5, 6)
    g.geo_full_neg_lap(kind, 5, 6)
    lv, ijk, ty = G.tiles()
    leaf = ty == cmg.LEAF
    assert np.array_equal(G.download(6)[leaf], g.channel(6)[leaf])
    # one smoothing call per level, then a V-cycle
    for level in range(G.info()[1] + 1):
        G.upload(7, x)
        g.channel(7)[:] = x
        solver.gauss_seidel(G, 1, 0, level, 7, 1)
        g.geo_gauss_seidel(kind, 1, 0, level, 7, 1)
        assert np.array_equal(G.download(7), g.channel(7))
    solver.VCycle(G, 4, 1, 3, 2, 10)
    g.geo_vcycle(kind, 4, 1, 3, 2, 10)
    assert np.array_equal(G.download(4), g.channel(4))


@pytest.mark.parametrize("kind", [O.GMG, O.CMG])
@pytest.mark.parametrize("case_id,prm", GEO_GRIDS)
def test_geometric_solve_matches_oracle(kind, case_id, prm):
    G, g, solver, b = _geo_pair(case_id, prm, kind)
    it, rel = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
    ito, relo = g.geo_solve(kind, 1.0, 1.0, max_iters=100, tol=1e-6, level_iters=2, coarsest_iters=10)
    assert rel <= 1e-6 and relo <= 1e-6
    assert abs(it - ito) <= 1
    lv, ijk, ty = G.tiles()
    m = ty == cmg.LEAF
    x = G.download(0)[m]
    assert np.linalg.norm(x - g.channel(0)[m]) <= 1e-5 * np.linalg.norm(g.channel(0)[m])


@pytest.mark.parametrize("case_id,prm", [(cmg.CASE_UNIFORM, [2, 2]), (cmg.CASE_CENTER_POINT, [2, 4])])
def test_pure_neumann_solve_matches_oracle(case_id, prm):
    from workloads import pure_neumann_setup

    G = build_product(case_id, prm)
    g = build_oracle(case_id, prm)
    lv, ijk, ty = G.tiles()
    ct, b = pure_neumann_setup(lv, ijk, ty)
    G.upload_cell_types(ct)
    g.cell_types()[:] = ct
    solver = cmg.AMGSolver(COEFF, 0.5, 1.0, 1.0)
    solver.prepareTypesAndCoeffs(G)
    g.coarsen_types_and_coeffs(COEFF, 0.5)
    G.upload(1, b)
    g.channel(1)[:] = b
    it, rel = solver.solve(G, False, 100, 1e-6, 2, 10, 1, True)
    ito, relo = g.amg_solve(COEFF, max_iters=100, tol=1e-6, pure_neumann=True)
    assert rel <= 1e-6 and relo <= 1e-6 and abs(it - ito) <= 1
    m = (ty[:, None] == cmg.LEAF) & (G.download_cell_types() == cmg.INTERIOR)
    x, xo = G.download(0)[m], g.channel(0)[m]
    assert np.linalg.norm(x - xo) <= 1e-5 * np.linalg.norm(xo)


@pytest.mark.parametrize("case_id,prm", [(cmg.CASE_UNIFORM, [2, 2]), (cmg.CASE_CENTER_POINT, [2, 4])])
def test_fas_mu_cycle_solve_matches_oracle(case_id, prm):
    """AMGSolver::FASMuCycleSolve as the reference harness's "amg_vcycle": AMGSolver(coeff, 0.5, 0.5, 1),
    mu = 1, level_iters = 1 (tests/SolverTests.cu:1100-1112)."""
    from workloads import uniform_rhs

    G = build_product(case_id, prm)
    g = build_oracle(case_id, prm)
    G.set_leaf_cell_types_case(cmg.CASE_UNIFORM)
    g.set_leaf_cell_types_case(O.CASE_UNIFORM)
    solver = cmg.AMGSolver(COEFF, 0.5, 0.5, 1.0)
    solver.prepareTypesAndCoeffs(G)
    g.coarsen_types_and_coeffs(COEFF, 0.5)
    lv, ijk, ty = G.tiles()
    b = uniform_rhs(ty == cmg.LEAF, 0)
    G.upload(1, b)
    g.channel(1)[:] = b
    it, rel = solver.FASMuCycleSolve(1, G, False, 60, 1e-6, 1, 10)
    ito, relo = g.fas_mu_cycle_solve(COEFF, repeat_times=1, R_restrict=0.5, max_iters=60, tol=1e-6, level_iters=1, coarsest_iters=10)
    assert abs(it - ito) <= 1
    assert rel == pytest.approx(relo, rel=1e-3)
    m = ty == cmg.LEAF
    x, xo = G.download(0)[m], g.channel(0)[m]
    assert np.linalg.norm(x - xo) <= 1e-5 * np.linalg.norm(xo)


def test_gmg_damped_jacobi_matches_oracle():
    G, g, solver, b = _geo_pair(cmg.CASE_CENTER_POINT, [2, 4], O.GMG)
    it, rel = solver.dampedJacobiSolve(G, False, 40, 1e-12, 1.0)
    ito, relo = g.gmg_damped_jacobi_solve(max_iters=40, tol=1e-12, omega=1.0)
    assert it == ito == 40
    assert rel == pytest.approx(relo, rel=1e-4)
    lv, ijk, ty = G.tiles()
    m = ty == cmg.LEAF
    x, xo = G.download(0)[m], g.channel(0)[m]
    assert np.linalg.norm(x - xo) <= 1e-5 * np.linalg.norm(xo)
