"""Writes the golden fixtures of tests/golden from the CPU oracle (test infrastructure).

The reference stores no golden vectors for this path, so these fixtures pin the oracle's
own outputs on seeded inputs; tests check that the oracle still reproduces them (CPU) and
that the CUDA product agrees with them (GPU).

  uniform32.npz   32^3 uniform grid (levels 0-2), all cells INTERIOR, Dirichlet walls,
                  b = N(0,1) on LEAF cells from default_rng(0) (the smoke case):
                  x64 = FP64 Jacobi-CG solution of the assembled operator to 1e-12 (stored
                  as float32, LEAF tiles in tile order), oracle_iters = iterations of the
                  oracle's FP32 mu-cycle PCG to 1e-6.
  learned_h8.npz  the learned smoother's network, H = 8: seeded parameters and four sample
                  tiles, with the FP64 restatement's forward output, loss and gradient
                  (BF16 roundings emulated, energy loss).

Run from the repository root:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import learned_oracle as LO  # noqa: E402
from oracle import oracle as O  # noqa: E402

COEFF = 6


def uniform32_rhs(ty):
    rng = np.random.default_rng(0)
    leaf = ty == O.LEAF
    b = np.zeros((ty.size, 512), np.float32)
    b[leaf] = rng.standard_normal((int(leaf.sum()), 512)).astype(np.float32)
    return b


def build_uniform32():
    g = O.Grid(0.125, 10)
    g.set_tile(0, 0, 0, 0, O.LEAF)
    g.rebuild()
    g.refine_case(O.CASE_UNIFORM, [2, 2])
    g.alloc(16)
    g.set_leaf_cell_types_case(O.CASE_UNIFORM)
    g.coarsen_types_and_coeffs(COEFF, 0.5)
    return g


def uniform32():
    g = build_uniform32()
    _, _, ty = g.tiles()
    b = uniform32_rhs(ty)
    rp, ci, va, rt, rc = g.assemble(COEFF)
    x, its, rel = O.csr_solve(rp, ci, va, b[rt, rc].astype(np.float64), 1e-12, 20000, 0)
    x64 = np.zeros((ty.size, 512), np.float64)
    x64[rt, rc] = x
    g.channel(1)[:] = b
    oit, orel = g.amg_solve(COEFF, max_iters=100, tol=1e-6)
    return dict(x64=x64[ty == O.LEAF].astype(np.float32), oracle_iters=np.int32(oit), fp64_rel=np.float64(rel))


def learned_samples(n=4, seed=11):
    rng = np.random.default_rng(seed)
    types = np.full((n, 512), LO.INTERIOR, np.uint8)
    u = rng.uniform(size=(n, 512))
    types[u < 0.1] = LO.DIRICHLET
    types[(u >= 0.1) & (u < 0.15)] = LO.NEUMANN
    rho = (rng.standard_normal((n, 512)) * 10.0 ** rng.uniform(-2, 2, (n, 1))).astype(np.float32)
    diag = (rng.uniform(0.3, 6.0, (n, 512)) / 64.0).astype(np.float32)
    target = rng.standard_normal((n, 512)).astype(np.float32)
    L = LO.layout(8)
    p = (rng.standard_normal(L["n"]) * 0.15).astype(np.float32)
    return p, rho, diag, types, target


def learned_h8():
    p, rho, diag, types, target = learned_samples()
    fwd = LO.forward(p, 8, rho, diag, types)
    loss, grad = LO.loss_and_grad(p, 8, rho, diag, types, target, kind=1)
    return dict(params=p, rho=rho, diag=diag, types=types, target=target, forward=fwd.astype(np.float32),
                loss=np.float64(loss), grad=grad.astype(np.float32))


def main():
    np.savez_compressed(os.path.join(HERE, "uniform32.npz"), **uniform32())
    np.savez_compressed(os.path.join(HERE, "learned_h8.npz"), **learned_h8())


if __name__ == "__main__":
    main()
