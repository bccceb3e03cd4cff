"""Mixed-precision preconditioner: the cycle's smoothing sweeps read the operator from a
BF16 or FP16 copy (cmg_amg_solver_set_storage).

The 16-bit path widens every stored value to float and computes in FP32, so on a grid
whose coefficients were rounded to 16 bits beforehand it must equal the FP32 path bit
for bit -- sweep by sweep and for a whole solve.  On the real coefficients the mixed
solve must still reach the tolerance, within two PCG iterations of FP32, and agree with
the FP64 CSR solution of the exact operator to 1e-5 relative L2 (the tolerance of the
FP32 solve tests).
"""
import numpy as np
import pytest

import cmg
from workloads import COEFF, setup_shell, setup_uniform, shell_params

pytestmark = pytest.mark.gpu


def round_bf16(a):
    """float32 -> nearest bfloat16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32)


def round_fp16(a):
    return np.asarray(a, np.float32).astype(np.float16).astype(np.float32)


ROUND = {"bf16": round_bf16, "fp16": round_fp16}


def _rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("storage", ["bf16", "fp16"])
def test_16bit_sweeps_equal_fp32_sweeps_on_rounded_coefficients(storage):
    G, _, solver = setup_shell(shell_params(coarse=3, mid=4, fine=5), with_oracle=False)
    for a in range(4):
        G.upload(COEFF + a, ROUND[storage](G.download(COEFF + a)))
    rng = np.random.default_rng(5)
    n = G.num_tiles
    interior = G.download_cell_types() == cmg.INTERIOR
    x = np.where(interior, rng.standard_normal((n, 512)), 0.0).astype(np.float32)
    G.upload(3, rng.standard_normal((n, 512)).astype(np.float32))
    for level in range(3, G.max_level + 1):
        out = []
        for mode in ("fp32", storage):
            solver.set_storage(mode)
            G.upload(4, x)
            solver.gauss_seidel_masked(G, 2, 0, level, 4, 3)
            out.append(G.download(4))
        assert np.array_equal(out[0], out[1]), level


@pytest.mark.parametrize("storage", ["bf16", "fp16"])
def test_16bit_solve_equals_fp32_solve_on_rounded_coefficients(storage):
    G, _, solver = setup_shell(shell_params(coarse=3, mid=4, fine=5), with_oracle=False)
    for a in range(4):
        G.upload(COEFF + a, ROUND[storage](G.download(COEFF + a)))
    b = G.download(1)
    res = []
    for mode in ("fp32", storage):
        solver.set_storage(mode)
        G.upload(1, b)
        it, rel = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
        res.append((it, rel, G.download(0)))
    assert res[0][:2] == res[1][:2]
    assert np.array_equal(res[0][2], res[1][2])


@pytest.mark.parametrize("storage", ["bf16", "fp16"])
@pytest.mark.parametrize("grid", ["uniform64", "shell345"])
def test_mixed_solve_converges_to_the_fp64_solution(storage, grid):
    from test_gpu_parity import fp64_solution

    if grid == "uniform64":
        G, g, solver, b = setup_uniform(3)
    else:
        G, g, solver = setup_shell(shell_params(coarse=3, mid=4, fine=5))
        b = G.download(1)
        g.channel(1)[:] = b
    solver.set_storage("fp32")
    it32, rel32 = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
    solver.set_storage(storage)
    G.upload(1, b)
    it, rel = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
    assert rel <= 1e-6
    assert it <= it32 + 2, (it, it32)
    xs, rt, rc = fp64_solution(g, b, 0 if grid == "uniform64" else 1)
    assert _rel_l2(G.download(0)[rt, rc], xs) <= 1e-5


def test_true_residual_replacement():
    """Every `every` iterations the recurrence residual is replaced by b - A x (stencil in
    FP64).  A weak preconditioner (one sweep per level, two on the coarsest) makes the solve
    long enough for several replacements; it must still converge to the FP64 solution with
    about the iteration count of the plain recurrence.  With `every` beyond the iteration
    count the solve is the plain one, bit for bit."""
    from test_gpu_parity import fp64_solution

    G, g, solver, b = setup_uniform(3)
    solver.omega = 1.0
    solver.mu_cycle_repeat_times = 1
    it0, rel0 = solver.solve(G, False, 100, 1e-6, 1, 2, 1, False)
    x0 = G.download(0)
    assert solver.last_replacements() == 0
    G.upload(1, b)
    solver.set_residual_replacement(3)
    it1, rel1 = solver.solve(G, False, 100, 1e-6, 1, 2, 1, False)
    n = solver.last_replacements()
    assert it0 >= 7, it0
    assert n == (it1 - 1) // 3 and n >= 2, (n, it1)
    assert rel1 <= 1e-6 and abs(it1 - it0) <= 1, (it0, it1)
    xs, rt, rc = fp64_solution(g, b, 0)
    x1 = G.download(0)
    assert _rel_l2(x1[rt, rc], xs) <= 1e-5
    # the replaced residual is the true one: |b - A x| / |b| from the FP64 operator
    rp, ci, va, rt2, rc2 = g.assemble(COEFF)
    from oracle import oracle as O

    ax = O.csr_matvec(rp, ci, va, x1[rt2, rc2].astype(np.float64))
    bb = b[rt2, rc2].astype(np.float64)
    true_rel = np.linalg.norm(bb - ax) / np.linalg.norm(bb)
    assert true_rel <= 2e-6, true_rel
    G.upload(1, b)
    solver.set_residual_replacement(1000)
    it2, rel2 = solver.solve(G, False, 100, 1e-6, 1, 2, 1, False)
    assert solver.last_replacements() == 0
    assert (it2, rel2) == (it0, rel0) and np.array_equal(G.download(0), x0)


@pytest.mark.parametrize("grid", ["uniform32", "uniform64", "shell345"])
def test_direct_coarsest_solve(grid):
    """Level 0 solved exactly in double (FP64 Cholesky-based inverse of the root operator)
    inside the cluster step: the solve converges to the FP64 solution in no more PCG
    iterations than with the reference's coarsest sweeps."""
    from test_gpu_parity import fp64_solution

    if grid.startswith("uniform"):
        G, g, solver, b = setup_uniform(2 if grid == "uniform32" else 3)
    else:
        G, g, solver = setup_shell(shell_params(coarse=3, mid=4, fine=5))
        b = G.download(1)
        g.channel(1)[:] = b
    it0, rel0 = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
    solver.set_coarsest_direct(True)
    G.upload(1, b)
    it1, rel1 = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
    assert rel1 <= 1e-6 and it1 <= it0, (it0, it1)
    xs, rt, rc = fp64_solution(g, b, 0 if grid.startswith("uniform") else 1)
    assert _rel_l2(G.download(0)[rt, rc], xs) <= 1e-5
    # fewer coarsest sweeps than the reference's ten cannot beat the exact solve
    solver.set_coarsest_direct(False)
    G.upload(1, b)
    it2, _ = solver.solve(G, False, 100, 1e-6, 2, 2, 1, False)
    assert it1 <= it2


def test_mixed_mode_on_the_sphere_octree():
    """Config 3's whole mixed mode on the 3/4/5 sphere octree: BF16 operator, x and rhs storage,
    true residual every 10 iterations and the direct coarsest solve, against the FP64 solution."""
    from test_gpu_parity import fp64_solution

    G, g, solver = setup_shell(shell_params(coarse=3, mid=4, fine=5))
    b = G.download(1)
    g.channel(1)[:] = b
    solver.set_storage("bf16")
    solver.set_cycle_bf16(True)
    solver.set_residual_replacement(10)
    solver.set_coarsest_direct(True)
    it, rel = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
    assert rel <= 1e-6
    xs, rt, rc = fp64_solution(g, b, 1)
    assert _rel_l2(G.download(0)[rt, rc], xs) <= 1e-5


@pytest.mark.parametrize("grid", ["uniform64", "shell345"])
def test_bf16_cycle_storage_matches_the_oracle(grid):
    """x, rhs and saved x of levels >= 3 in BF16 planes (FP32 arithmetic): the solve follows the
    oracle run with the same roundings (og_set_x_bf16) to +-1 iteration and 1e-5, and the FP64
    solution to 1e-5, in the iteration count of the FP32 cycle within one."""
    from test_gpu_parity import fp64_solution

    if grid == "uniform64":
        G, g, solver, b = setup_uniform(3)
    else:
        G, g, solver = setup_shell(shell_params(coarse=3, mid=4, fine=5))
        b = G.download(1)
        g.channel(1)[:] = b
    it32, _ = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
    G.upload(1, b)
    solver.set_cycle_bf16(True)
    it, rel = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
    x = G.download(0)
    g.set_x_bf16(True)
    ito, relo = g.amg_solve(COEFF, max_iters=100, tol=1e-6)
    assert rel <= 1e-6 and abs(it - ito) <= 1 and abs(it - it32) <= 1, (it, ito, it32)
    m = G.tiles()[2] == cmg.LEAF
    assert _rel_l2(x[m], g.channel(0)[m]) <= 1e-5
    xs, rt, rc = fp64_solution(g, b, 0 if grid == "uniform64" else 1)
    assert _rel_l2(x[rt, rc], xs) <= 1e-5
