"""Learned finest-level smoother: the per-tile network's forward pass and gradients
against the FP64 CPU restatement (oracle/learned_oracle.py), GPU training, and the
learned solve (flexible PCG, true-residual judge, plain fallback) against the plain one."""
import numpy as np
import pytest

import cmg
import learned
from oracle import learned_oracle as LO
from workloads import COEFF, setup_uniform, uniform_rhs

pytestmark = pytest.mark.gpu


def random_samples(n, seed):
    """Tiles with mixed cell types, residual scales over six decades, one all-zero tile and
    one tile without INTERIOR cells (both give a zero correction)."""
    rng = np.random.default_rng(seed)
    types = np.full((n, 512), cmg.INTERIOR, np.uint8)
    u = rng.uniform(size=(n, 512))
    types[u < 0.08] = cmg.DIRICHLET
    types[(u >= 0.08) & (u < 0.15)] = cmg.NEUMANN
    rho = (rng.standard_normal((n, 512)) * 10.0 ** rng.uniform(-3, 3, (n, 1))).astype(np.float32)
    diag = (rng.uniform(0.3, 6.0, (n, 512)) / 64.0).astype(np.float32)
    target = (rng.standard_normal((n, 512)) * 10.0 ** rng.uniform(-2, 2, (n, 1))).astype(np.float32)
    rho[1] = 0.0
    types[2] = cmg.NEUMANN
    return rho, diag, types, target


def random_params(H, seed, scale=0.15):
    rng = np.random.default_rng(seed)
    L = LO.layout(H)
    p = (rng.standard_normal(L["n"]) * scale).astype(np.float32)
    p[L["B1"]:L["W2"]] = rng.uniform(-0.1, 0.1, H)
    p[L["B2"]:L["W3"]] = rng.uniform(-0.1, 0.1, H)
    return p


@pytest.mark.parametrize("H,kind", [(8, "tcgen05"), (16, "tcgen05"), (8, "mma.sync"), (16, "mma.sync")])
def test_forward_matches_oracle(H, kind):
    """Both inference kernels (tcgen05 with TMEM accumulators, and mma.sync) against the oracle."""
    rho, diag, types, target = random_samples(12, 10 + H)
    net = cmg.LearnedNet(H, seed=1)
    p = random_params(H, 20 + H)
    net.set_params(p)
    net.set_samples(rho, diag, types, target)
    cmg.set_learned_inference(kind)
    try:
        out = net.forward()
    finally:
        cmg.set_learned_inference("mma.sync")
    ref = LO.forward(p, H, rho, diag, types)
    assert np.all(out[1] == 0) and np.all(out[2] == 0)
    assert np.all(out[(types & cmg.INTERIOR) == 0] == 0)
    for s in range(out.shape[0]):
        m = np.abs(ref[s]).max()
        if m == 0:
            continue
        # same BF16 roundings on both sides; FP32 against FP64 accumulation and rare
        # rounding-boundary flips of a BF16 activation remain
        assert np.abs(out[s] - ref[s]).max() <= 1e-2 * m, s


@pytest.mark.parametrize("H,kind", [(8, 0), (16, 0), (8, 1), (16, 1)])
def test_gradient_matches_oracle(H, kind):
    rho, diag, types, target = random_samples(10, 30 + H)
    net = cmg.LearnedNet(H, seed=2)
    p = random_params(H, 40 + H)
    net.set_params(p)
    net.set_loss(["mse", "energy"][kind])
    net.set_samples(rho, diag, types, target)
    loss, g = net.gradient()
    rl, rg = LO.loss_and_grad(p, H, rho, diag, types, target, kind=kind)
    assert abs(loss - rl) <= 1e-3 * rl
    L = LO.layout(H)
    for a, b in [("W1", "B1"), ("B1", "W2"), ("W2", "B2"), ("B2", "W3"), ("W3", "n")]:
        gs, rs = g[L[a]:L[b]], rg[L[a]:L[b]]
        assert np.linalg.norm(gs - rs) <= 2e-2 * np.linalg.norm(rs) + 1e-12, a
    # padded input channels 4..7 of W1 get exactly zero gradient
    gw1 = g[L["W1"]:L["B1"]].reshape(H, 27, 8)
    assert np.all(gw1[:, :, 4:] == 0)


def random_extra(n, seed):
    """Face coefficients (negative, cut faces smaller) and a residual halo with about a third of
    its cells absent (flag 0, value 0)."""
    rng = np.random.default_rng(seed)
    faces = (-rng.uniform(0.05, 1.0, (n, 3, 512)) / 64.0).astype(np.float32)
    val = (rng.standard_normal((n, 384)) * 10.0 ** rng.uniform(-3, 3, (n, 1))).astype(np.float32)
    flag = (rng.uniform(size=(n, 384)) > 0.33).astype(np.float32)
    return faces, np.concatenate([val * flag, flag], axis=1)


@pytest.mark.parametrize("H,kind", [(8, "tcgen05"), (16, "tcgen05"), (8, "mma.sync"), (16, "mma.sync")])
def test_forward_with_faces_and_halo_matches_oracle(H, kind):
    """The net's face-coefficient channels and the residual's 1-cell halo, both kernels."""
    rho, diag, types, target = random_samples(12, 50 + H)
    faces, halo = random_extra(12, 60 + H)
    net = cmg.LearnedNet(H, seed=1)
    p = random_params(H, 70 + H)
    net.set_params(p)
    net.set_samples(rho, diag, types, target, faces, halo)
    cmg.set_learned_inference(kind)
    try:
        out = net.forward()
    finally:
        cmg.set_learned_inference("mma.sync")
    ref = LO.forward(p, H, rho, diag, types, faces=faces, halo=halo)
    plain = LO.forward(p, H, rho, diag, types)
    assert np.all(out[(types & cmg.INTERIOR) == 0] == 0)
    moved = 0
    for s in range(out.shape[0]):
        m = np.abs(ref[s]).max()
        if m == 0:
            continue
        assert np.abs(out[s] - ref[s]).max() <= 1e-2 * m, s
        moved += np.abs(ref[s] - plain[s]).max() > 0.05 * m  # the extra inputs change the output
    assert moved >= 6


@pytest.mark.parametrize("H", [8, 16])
def test_gradient_with_faces_and_halo_matches_oracle(H):
    rho, diag, types, target = random_samples(10, 80 + H)
    faces, halo = random_extra(10, 90 + H)
    net = cmg.LearnedNet(H, seed=2)
    p = random_params(H, 100 + H)
    net.set_params(p)
    net.set_loss("energy")
    net.set_samples(rho, diag, types, target, faces, halo)
    loss, g = net.gradient()
    rl, rg = LO.loss_and_grad(p, H, rho, diag, types, target, kind=1, faces=faces, halo=halo)
    assert abs(loss - rl) <= 1e-3 * rl
    L = LO.layout(H)
    for a, b in [("W1", "B1"), ("B1", "W2"), ("W2", "B2"), ("B2", "W3"), ("W3", "n")]:
        gs, rs = g[L[a]:L[b]], rg[L[a]:L[b]]
        assert np.linalg.norm(gs - rs) <= 2e-2 * np.linalg.norm(rs) + 1e-12, a
    # the face channels 4..6 now carry gradient; channel 7 stays unused
    gw1 = g[L["W1"]:L["B1"]].reshape(H, 27, 8)
    assert np.any(gw1[:, :, 4:7] != 0) and np.all(gw1[:, :, 7] == 0)


@pytest.mark.parametrize("kind", ["mma.sync", "tcgen05"])
def test_net_on_the_grid_equals_net_on_samples(kind):
    """The learned solve's inputs read on the grid (face coefficients, the residual across faces
    from same-level LEAF neighbours) equal the training samples' (learned.collect_pairs), bit
    for bit: the same kernel on the same values."""
    from workloads import setup_shell, shell_params

    G, _, S = setup_shell(shell_params(coarse=3, mid=4, fine=5), with_oracle=False)
    lv, ijk, ty = G.tiles()
    L = int(lv.max())
    nb, _ = G.tables()
    types = G.download_cell_types()
    rng = np.random.default_rng(3)
    leaf = ty == cmg.LEAF
    inter = (types & cmg.INTERIOR) != 0
    r = np.where(inter & leaf[:, None], rng.standard_normal((G.num_tiles, 512)), 0.0).astype(np.float32)
    G.upload(1, r)
    net = cmg.LearnedNet(16, seed=5)
    net.set_params(random_params(16, 6))
    cmg.set_learned_inference(kind)
    try:
        net.apply_grid(G, L, 1, -1, COEFF, 4, overwrite=True)
        sel = learned.finest_leaf_tiles(G)
        faces = np.stack([G.download(COEFF + a) for a in range(3)], axis=1)[sel]
        halo = learned.tile_halo(r, types, ty, nb, sel)
        assert halo[:, 384:].sum() > 0  # the octree has LEAF neighbours across tile faces
        net.set_samples(r[sel], G.download(COEFF + 3)[sel], types[sel], None, faces, halo)
        out = net.forward()
    finally:
        cmg.set_learned_inference("mma.sync")
    assert np.array_equal(G.download(4)[sel], out)


def test_inference_kernels_agree():
    """tcgen05 and mma.sync inference on 300 tiles: the same products, summed in different orders."""
    rho, diag, types, target = random_samples(300, 77)
    net = cmg.LearnedNet(16, seed=8)
    net.set_params(random_params(16, 78))
    net.set_samples(rho, diag, types, target)
    out_ms = net.forward()
    cmg.set_learned_inference("tcgen05")
    try:
        out_tc = net.forward()
    finally:
        cmg.set_learned_inference("mma.sync")
    scale = np.abs(out_ms).max(axis=1, keepdims=True) + 1e-30
    assert np.all(np.abs(out_tc - out_ms) <= 1e-2 * scale)


def test_gradient_is_deterministic():
    rho, diag, types, target = random_samples(9, 5)
    net = cmg.LearnedNet(16, seed=4)
    net.set_samples(rho, diag, types, target)
    l1, g1 = net.gradient()
    l2, g2 = net.gradient()
    assert l1 == l2 and np.array_equal(g1, g2)


def _uniform_pairs(L, seeds, iters=(1, 2, 3)):
    G, _, solver, _ = setup_uniform(L, seed=seeds[0], with_oracle=False)
    lv, _, ty = G.tiles()
    rhs = [uniform_rhs(ty == cmg.LEAF, s) for s in seeds]
    return G, solver, learned.collect_pairs(G, solver, COEFF, rhs, iters=iters), ty


def test_pairs_satisfy_the_error_equation():
    """d = A^-1 rho: A d reproduces rho on the finest LEAF tiles."""
    G, solver, pairs, ty = _uniform_pairs(2, [7], iters=(2,))
    fine = learned.finest_leaf_tiles(G)
    d = np.zeros((G.num_tiles, 512), np.float32)
    d[fine] = pairs["d"]
    G.upload(13, d)
    G.full_neg_lap(13, COEFF, 14)
    ad = G.download(14)[fine]
    assert np.linalg.norm(ad - pairs["rho"]) <= 1e-5 * np.linalg.norm(pairs["rho"])


def test_training_reduces_loss():
    G, solver, pairs, ty = _uniform_pairs(2, [100, 101, 102, 103])
    net0 = cmg.LearnedNet(16, seed=0)
    net0.set_samples(pairs["rho"], pairs["diag"], pairs["types"], pairs["d"])
    l0, _ = net0.gradient()
    net, losses = learned.train(pairs, hidden=16, epochs=15, batch=64, lr=2e-3, seed=0)
    l1, _ = net.gradient()
    assert np.all(np.isfinite(losses))
    assert l1 < 0.7 * l0, (l0, l1, losses)


def test_learned_solve_with_tcgen05_inference():
    """The learned solve with the tcgen05 inference kernel: same iterations as with mma.sync
    and the same solution to FP32 rounding."""
    G, solver, pairs, ty = _uniform_pairs(2, [100, 101, 102])
    net, _ = learned.train(pairs, hidden=8, epochs=10, batch=128, lr=2e-3, seed=0, damping=0.5, loss="energy")
    b = uniform_rhs(ty == cmg.LEAF, 0)
    rows_ms = learned.compare(G, solver, net, [b])
    cmg.set_learned_inference("tcgen05")
    try:
        rows_tc = learned.compare(G, solver, net, [b])
    finally:
        cmg.set_learned_inference("mma.sync")
    assert not rows_tc[0][5] and rows_tc[0][4] <= 1e-5
    assert abs(rows_tc[0][2] - rows_ms[0][2]) <= 1
    assert rows_tc[0][6] <= 1e-4


def test_learned_solve_matches_plain():
    """An untrained net: flexible PCG still reaches the tolerance (or falls back), the true
    residual judges it, and x agrees with the plain solve."""
    G, _, solver, b = setup_uniform(3, seed=0, with_oracle=False)
    net = cmg.LearnedNet(16, seed=5)
    rows = learned.compare(G, solver, net, [b])
    ip, tp, il, tl, tr, fb, dx = rows[0]
    assert tr <= 4e-6
    assert dx <= 1e-4, rows
    assert il <= 100


def test_stalled_learned_solve_falls_back_to_plain():
    """A net whose correction swamps the cycle's (output layer x 1000) leaves the residual where
    it is: the solve stops as stalled after a few iterations (the residual norm fell by less
    than 2x over 4 of them), and the plain solve takes over with the plain result."""
    G, _, solver, b = setup_uniform(3, seed=0, with_oracle=False)
    ip, _ = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
    xp = G.download(0)
    net = cmg.LearnedNet(8, seed=3)
    p = net.params()
    p[-27 * 8:] *= 1000.0
    net.set_params(p)
    solver.set_learned(net)
    G.upload(1, b)
    it, rel = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
    tr, fb, lit = solver.learned_status()
    solver.set_learned(None)
    assert fb and lit <= 8, (fb, lit)
    assert it == ip and rel < 1e-6 and np.array_equal(G.download(0), xp)


def test_nonfinite_net_falls_back_to_plain():
    """A net whose output overflows makes the learned solve non-finite; the plain solve takes over."""
    G, _, solver, b = setup_uniform(2, seed=3, with_oracle=False)
    ip, _ = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
    xp = G.download(0)
    net = cmg.LearnedNet(8, seed=6)
    net.set_params(np.full(net.num_params, 3e37, np.float32))
    solver.set_learned(net)
    G.upload(1, b)
    it, rel = solver.solve(G, False, 100, 1e-6, 2, 10, 1, False)
    tr, fb, _ = solver.learned_status()
    assert fb and it == ip and rel < 1e-6
    assert np.array_equal(G.download(0), xp)


def test_trained_net_against_plain(capsys):
    """What the trained network gains: trained on other right-hand sides of the uniform 64^3
    grid (seeds 100-109), compared with the plain solve on the benchmark rhs (seed 0).
    The damped net (output x 0.5, energy loss) saves one of the plain solve's 8 PCG iterations."""
    G, solver, pairs, ty = _uniform_pairs(3, list(range(100, 110)), iters=(1, 2, 3, 5))
    net, losses = learned.train(pairs, hidden=8, epochs=30, batch=256, lr=2e-3, seed=0, damping=0.5, loss="energy")
    b = uniform_rhs(ty == cmg.LEAF, 0)
    rows = learned.compare(G, solver, net, [b, b])
    with capsys.disabled():
        print("\nlearned vs plain (uniform 64^3): losses", losses[0], losses[-1], "rows", rows)
    assert losses[-1] < 0.9 * losses[0]
    ip, tp, il, tl, tr, fb, dx = rows[-1]
    assert not fb and tr <= 4e-6 and dx <= 1e-4
    assert il < ip, rows


def test_moving_sphere_sequence():
    """The net trained at one sphere position, applied as the octree and cut-cell operator move
    with the sphere: every learned solve passes the true-residual judge (or falls back) and
    matches the plain solution."""
    from workloads import U, fourier_modes, setup_shell, shell_params

    centres = [(0.5 + 0.25 * np.cos(t), 0.5 + 0.25 * np.sin(t), 0.5) for t in (0.0, 0.3, 0.6)]
    G, _, solver = setup_shell(shell_params(3, 4, 5, centres[0], 0.1), spheres=[centres[0] + (0.1,)], with_oracle=False)
    rhs = []
    for seed in (7, 8, 9):
        k, amp, ph = fourier_modes(seed)
        G.face_velocity_fourier(U, k, amp, ph)
        G.divergence(U, COEFF, 1)
        rhs.append(G.download(1))
    pairs = learned.collect_pairs(G, solver, COEFF, rhs, iters=(1, 2, 3))
    net, _ = learned.train(pairs, hidden=8, epochs=10, batch=128, lr=2e-3, seed=0, damping=0.5, loss="energy")
    for c in centres:
        G, _, solver = setup_shell(shell_params(3, 4, 5, c, 0.1), spheres=[c + (0.1,)], with_oracle=False)
        b = G.download(1)
        ip, tp, il, tl, tr, fb, dx = learned.compare(G, solver, net, [b])[0]
        assert tr <= 1e-5 and dx <= 1e-3, (c, ip, il, tr, fb, dx)
