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
