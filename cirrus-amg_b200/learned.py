"""Training data and training driver of the learned finest-level smoother.

The reference has no learned preconditioner; this is the learned form of its solve
(`AMGSolver::solve`, src/AMGSolver.cu:1399-1549) with a per-tile network added after
each FAS mu-cycle on the finest level's LEAF tiles (csrc/learned.cu).

Training pairs come from the plain solver: for a right-hand side b and k plain PCG
iterations from x = 0, r_k is the residual left in channel 1; one mu-cycle gives
z = M r_k; rho = r_k - A z is the residual the cycle leaves and d = A^-1 rho (a plain
solve to a tight tolerance) is the error it leaves.  The network learns d from rho on
each finest LEAF tile, with the tile's cell types and diagonal of A as extra inputs.
Training runs on the GPU (LearnedNet.train: the forward and backward kernels of
learned.cu with Adam).
"""
import numpy as np

import cmg


def finest_leaf_tiles(G):
    """Indices of the LEAF tiles on the grid's finest level."""
    lv, _, ty = G.tiles()
    return np.nonzero((lv == lv.max()) & (ty == cmg.LEAF))[0]


def collect_pairs(G, solver, coeff_ch, rhs_list, iters=(1, 2, 3, 5), z_ch=13, x0_ch=14, az_ch=15, exact_tol=1e-7,
                  exact_iters=300, level_iters=2, coarsest_iters=10, max_tiles=None, seed=0):
    """(rho, diag, types, d) of the finest LEAF tiles for every rhs in rhs_list ([n, 512] host
    arrays) and every iteration count in iters.  Channels 0-5 and z_ch, x0_ch, az_ch are
    overwritten.  max_tiles: a seeded random subset of that many tiles per pair at most."""
    fine = finest_leaf_tiles(G)
    lv, _, ty = G.tiles()
    leaf = ty == cmg.LEAF
    types = G.download_cell_types()
    diag = G.download(coeff_ch + 3)
    inter = (types & cmg.INTERIOR) != 0
    rng = np.random.default_rng(seed)
    out = {"rho": [], "diag": [], "types": [], "d": []}
    for b in rhs_list:
        for k in iters:
            G.upload(1, b)
            solver.solve(G, False, int(k), 1e-30, level_iters, coarsest_iters, 1, False)
            r = G.download(1)
            r[~leaf] = 0.0
            G.upload(1, r)
            solver.fas_mu_cycle(G, z_ch, 1, x0_ch, level_iters, coarsest_iters)
            G.full_neg_lap(z_ch, coeff_ch, az_ch)
            az = G.download(az_ch)
            rho = np.where(inter & leaf[:, None], r - az, 0.0).astype(np.float32)
            G.upload(1, rho)
            solver.solve(G, False, exact_iters, exact_tol, level_iters, coarsest_iters, 1, False)
            d = G.download(0)
            sel = fine
            if max_tiles is not None and sel.size > max_tiles:
                sel = np.sort(rng.choice(sel, max_tiles, replace=False))
            out["rho"].append(rho[sel])
            out["diag"].append(diag[sel])
            out["types"].append(types[sel])
            out["d"].append(d[sel])
    return {k: np.concatenate(v) for k, v in out.items()}


def train(pairs, hidden=16, epochs=20, batch=256, lr=2e-3, seed=0, net=None, damping=1.0, loss="mse"):
    """A LearnedNet trained on `pairs` (from collect_pairs); returns (net, per-epoch loss).
    damping scales the trained network's output (its last layer is linear): the step length
    of the learned correction inside the preconditioner.  loss: "mse" or "energy"."""
    if net is None:
        net = cmg.LearnedNet(hidden, seed)
    net.set_loss(loss)
    net.set_samples(pairs["rho"], pairs["diag"], pairs["types"], pairs["d"])
    losses = net.train(epochs, batch, lr, seed)
    if damping != 1.0:
        p = net.params()
        w3 = p.size - 27 * net.hidden
        p[w3:] *= damping
        net.set_params(p)
    return net, losses


def compare(G, solver, net, rhs_list, tol=1e-6, max_iters=100, level_iters=2, coarsest_iters=10):
    """Plain against learned solves of each rhs: per rhs (plain iters, plain ms, learned iters,
    learned ms, learned true relative residual, fell back, max |x_learned - x_plain| / max |x_plain|)."""
    rows = []
    for b in rhs_list:
        solver.set_learned(None)
        G.upload(1, b)
        ip, _ = solver.solve(G, False, max_iters, tol, level_iters, coarsest_iters, 1, False)
        tp = solver.last_solve_ms()
        xp = G.download(0)
        solver.set_learned(net)
        G.upload(1, b)
        il, _ = solver.solve(G, False, max_iters, tol, level_iters, coarsest_iters, 1, False)
        tl = solver.last_solve_ms()
        xl = G.download(0)
        tr, fb, _ = solver.learned_status()
        rows.append((ip, tp, il, tl, tr, fb, float(np.abs(xl - xp).max() / max(np.abs(xp).max(), 1e-30))))
    solver.set_learned(None)
    return rows
