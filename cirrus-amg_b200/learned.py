"""Training data and training driver of the learned finest-level smoother.

The reference has no learned preconditioner; this is the learned form of its solve
(`AMGSolver::solve`, src/AMGSolver.cu:1399-1549) with a per-tile network added after
each FAS mu-cycle on the finest level's LEAF tiles (csrc/learned.cu).

Training pairs come from the plain solver: for a right-hand side b and k plain PCG
iterations from x = 0, r_k is the residual left in channel 1; one mu-cycle gives
z = M r_k; rho = r_k - A z is the residual the cycle leaves and d = A^-1 rho (a plain
solve to a tight tolerance) is the error it leaves.  The network learns d from rho on
each finest LEAF tile, with the tile's cell types, the diagonal and face coefficients of A
and the residual across the tile's faces (a 1-cell halo) as extra inputs.
Training runs on the GPU (LearnedNet.train: the forward and backward kernels of
learned.cu with Adam).
"""
import numpy as np

import cmg


def finest_leaf_tiles(G):
    """Indices of the LEAF tiles on the grid's finest level."""
    lv, _, ty = G.tiles()
    return np.nonzero((lv == lv.max()) & (ty == cmg.LEAF))[0]


def halo_index():
    """For halo entry r*128 + side*64 + a*8 + b (face of axis r on side `side`, 0: -, 1: +):
    the face-neighbour slot in the tables (-x, -y, -z, +x, +y, +z) and the neighbour's cell
    across that face (its boundary layer)."""
    slot = np.zeros(384, np.int64)
    cell = np.zeros(384, np.int64)
    for r in range(3):
        for side in range(2):
            e = 0 if side else 7
            for a in range(8):
                for b in range(8):
                    h = r * 128 + side * 64 + a * 8 + b
                    slot[h] = r + 3 * side
                    cell[h] = [e * 64 + a * 8 + b, a * 64 + e * 8 + b, a * 64 + b * 8 + e][r]
    return slot, cell


def tile_halo(rho, types, ty, nb, tiles):
    """[len(tiles), 768]: the residual rho across each tile's six faces from same-level LEAF
    neighbours (0 elsewhere), then 1/0 flags for INTERIOR cells of such neighbours; the
    layout the net's kernels read (NetExtra)."""
    slot, cell = halo_index()
    q = nb[tiles][:, slot]  # [m, 384] neighbour tile per entry
    has = q >= 0
    qs = np.where(has, q, 0)
    leafn = has & (ty[qs] == cmg.LEAF)
    inter = (types[qs, cell[None, :]] & cmg.INTERIOR) != 0
    flag = leafn & inter
    val = np.where(flag, rho[qs, cell[None, :]], 0.0)
    return np.concatenate([val, flag.astype(np.float32)], axis=1).astype(np.float32)


def collect_pairs(G, solver, coeff_ch, rhs_list, iters=(1, 2, 3, 5), z_ch=13, x0_ch=14, az_ch=15, exact_tol=1e-7,
                  exact_iters=300, level_iters=2, coarsest_iters=10, max_tiles=None, seed=0):
    """(rho, diag, types, d, faces, halo) of the finest LEAF tiles for every rhs in rhs_list
    ([n, 512] host arrays) and every iteration count in iters; faces: the tiles' -x/-y/-z face
    coefficients, halo: rho across their faces (tile_halo).  Channels 0-5 and z_ch, x0_ch,
    az_ch are overwritten.  max_tiles: a seeded random subset of that many tiles per pair at most."""
    fine = finest_leaf_tiles(G)
    lv, _, ty = G.tiles()
    nb, _ = G.tables()
    leaf = ty == cmg.LEAF
    types = G.download_cell_types()
    diag = G.download(coeff_ch + 3)
    faces = np.stack([G.download(coeff_ch + a) for a in range(3)], axis=1)  # [n, 3, 512]
    inter = (types & cmg.INTERIOR) != 0
    rng = np.random.default_rng(seed)
    out = {"rho": [], "diag": [], "types": [], "d": [], "faces": [], "halo": []}
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
            out["faces"].append(faces[sel])
            out["halo"].append(tile_halo(rho, types, ty, nb, sel))
    return {k: np.concatenate(v) for k, v in out.items()}


def train(pairs, hidden=16, epochs=20, batch=256, lr=2e-3, seed=0, net=None, damping=1.0, loss="mse"):
    """A LearnedNet trained on `pairs` (from collect_pairs); returns (net, per-epoch loss).
    damping scales the trained network's output (its last layer is linear): the step length
    of the learned correction inside the preconditioner.  loss: "mse" or "energy"."""
    if net is None:
        net = cmg.LearnedNet(hidden, seed)
    net.set_loss(loss)
    net.set_samples(pairs["rho"], pairs["diag"], pairs["types"], pairs["d"], pairs.get("faces"), pairs.get("halo"))
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
