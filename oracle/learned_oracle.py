"""FP64 CPU restatement of the learned finest-level smoother's network (test infrastructure only).

Imported by tests/ -- never by the product.  The reference has no learned preconditioner;
this module restates the network that cirrus-amg_b200/csrc/learned.cu runs on BF16 tensor
cores, so that its forward pass, loss and gradients can be checked:

  features per 8^3 tile (channels-last) with a 1-cell border:
      0: rho / S (S = RMS of rho over INTERIOR cells)   1: INTERIOR   2: DIRICHLET
      3: diag / D on INTERIOR cells (D = max |diag| over INTERIOR cells)
      4-6: the -x/-y/-z face coefficients / D on INTERIOR cells (0 without face data)   7: 0
      border: channel 0 the neighbour's rho / S and channel 1 its flag across each face (the
      sample's halo), 0 without halo data; the hidden layers are zero-padded
  a1 = relu(conv(x, W1) + b1); a2 = relu(conv(a1, W2) + b2); f = conv(a2, W3)
  correction = (S / D) f on INTERIOR cells
  loss = sum over tiles and INTERIOR cells of (f - target D / S)^2 / (n 512), or with the
         energy loss e^T L e per tile (L: the tile's 7-point Laplacian, zero outside)

Every convolution is 3x3x3 with tap = dx*9 + dy*3 + dz.  The GPU path rounds the
features, the weights and the activations a1, a2, 2 (f - t), dz2, dz1 to BF16 and
accumulates in FP32; `emulate_bf16=True` applies the same roundings here (in FP64
arithmetic otherwise), which is what the gradient check compares against.
"""
import numpy as np

DIRICHLET, INTERIOR, NEUMANN = 1, 2, 4


def bf16(x):
    """Round to the nearest BF16 (ties to even) via FP32, as __float2bfloat16_rn does."""
    f = np.ascontiguousarray(np.asarray(x, dtype=np.float64).astype(np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32).astype(np.float64)


def layout(H):
    W1 = 0
    B1 = W1 + H * 216
    W2 = B1 + H
    B2 = W2 + H * 27 * H
    W3 = B2 + H
    return dict(W1=W1, B1=B1, W2=W2, B2=B2, W3=W3, n=W3 + 27 * H)


def unpack(p, H):
    L = layout(H)
    p = np.asarray(p, dtype=np.float64)
    return (p[L["W1"]:L["B1"]].reshape(H, 27, 8), p[L["B1"]:L["W2"]], p[L["W2"]:L["B2"]].reshape(H, 27, H),
            p[L["B2"]:L["W3"]], p[L["W3"]:L["n"]].reshape(1, 27, H))


def _taps():
    return [(t // 9, (t // 3) % 3, t % 3) for t in range(27)]


def _padded(x):
    """x [n, 8, 8, 8, C] zero-padded to [n, 10, 10, 10, C]; an x already [n, 10, ...] as is."""
    if x.shape[1] == 10:
        return x
    xp = np.zeros((x.shape[0], 10, 10, 10, x.shape[4]))
    xp[:, 1:9, 1:9, 1:9] = x
    return xp


def conv(x, W):
    """x [n, 8, 8, 8, Cin] (or padded [n, 10, 10, 10, Cin]), W [Cout, 27, Cin] -> [n, 8, 8, 8, Cout];
    out[v] = sum_t x[v + off(t)] W[:, t]."""
    n = x.shape[0]
    xp = _padded(x)
    out = np.zeros((n, 8, 8, 8, W.shape[0]))
    for t, (dx, dy, dz) in enumerate(_taps()):
        out += np.einsum("sijkc,nc->sijkn", xp[:, dx:dx + 8, dy:dy + 8, dz:dz + 8], W[:, t, :])
    return out


def conv_input_grad(d, W):
    """Gradient of conv's input: da[u] = sum_t W[:, t]^T d[u - off(t)] (zero outside the tile)."""
    n = d.shape[0]
    dp = np.zeros((n, 10, 10, 10, d.shape[4]))
    dp[:, 1:9, 1:9, 1:9] = d
    out = np.zeros((n, 8, 8, 8, W.shape[2]))
    for t, (dx, dy, dz) in enumerate(_taps()):
        out += np.einsum("sijkn,nc->sijkc", dp[:, 2 - dx:10 - dx, 2 - dy:10 - dy, 2 - dz:10 - dz], W[:, t, :])
    return out


def conv_weight_grad(x, d):
    """Gradient of conv's weights: gW[n, t, c] = sum_v x[v + off(t), c] d[v, n]."""
    xp = _padded(x)
    g = np.zeros((d.shape[4], 27, x.shape[4]))
    for t, (dx, dy, dz) in enumerate(_taps()):
        g[:, t, :] = np.einsum("sijkc,sijkn->nc", xp[:, dx:dx + 8, dy:dy + 8, dz:dz + 8], d)
    return g


def halo_positions():
    """Padded-grid index (i, j, k) of halo entry r*128 + side*64 + a*8 + b: the cell (a, b) of
    the face of axis r on side `side` (0: -, 1: +)."""
    pos = np.zeros((384, 3), np.int64)
    for r in range(3):
        for side in range(2):
            for a in range(8):
                for b in range(8):
                    e = 9 if side else 0
                    pos[r * 128 + side * 64 + a * 8 + b] = [(e, a + 1, b + 1), (a + 1, e, b + 1), (a + 1, b + 1, e)][r]
    return pos


def features(rho, diag, types, emulate_bf16=True, faces=None, halo=None):
    """Per-tile features as a padded [n, 10, 10, 10, 8] volume; rho, diag [n, 512] float32,
    types [n, 512] uint8 (cell i*64 + j*8 + k); faces [n, 3, 512], halo [n, 768] (optional)."""
    rho = np.asarray(rho, dtype=np.float32).reshape(-1, 512)
    diag = np.asarray(diag, dtype=np.float32).reshape(-1, 512)
    types = np.asarray(types, dtype=np.uint8).reshape(-1, 512)
    n = rho.shape[0]
    inter = (types & INTERIOR) != 0
    r = np.where(inter, rho, 0.0).astype(np.float64)
    cnt = inter.sum(1)
    D = np.where(inter, np.abs(diag), 0.0).max(1).astype(np.float64)
    ss = (r * r).sum(1)
    ok = (cnt > 0) & (ss > 0) & (D > 0)
    S = np.where(ok, np.sqrt(ss / np.maximum(cnt, 1)), 0.0)
    x = np.zeros((n, 512, 8))
    Ssafe = np.where(ok, S, 1.0)[:, None]
    Dsafe = np.where(ok, D, 1.0)[:, None]
    x[:, :, 0] = r / Ssafe
    x[:, :, 1] = inter
    x[:, :, 2] = (types & DIRICHLET) != 0
    x[:, :, 3] = np.where(inter, diag / Dsafe, 0.0)
    if faces is not None:
        fc = np.asarray(faces, dtype=np.float32).reshape(n, 3, 512).astype(np.float64)
        for a in range(3):
            x[:, :, 4 + a] = np.where(inter, fc[:, a] / Dsafe, 0.0)
    xp = np.zeros((n, 10, 10, 10, 8))
    xp[:, 1:9, 1:9, 1:9] = x.reshape(n, 8, 8, 8, 8)
    if halo is not None:
        hl = np.asarray(halo, dtype=np.float32).reshape(n, 768).astype(np.float64)
        pos = halo_positions()
        val, flag = hl[:, :384], hl[:, 384:]
        xp[:, pos[:, 0], pos[:, 1], pos[:, 2], 0] = np.where(flag != 0, val / Ssafe, 0.0)
        xp[:, pos[:, 0], pos[:, 1], pos[:, 2], 1] = flag
    if emulate_bf16:
        xp = bf16(xp)
    return xp, S, D, inter, ok


def forward(p, H, rho, diag, types, emulate_bf16=True, faces=None, halo=None):
    """Correction (S/D) f on INTERIOR cells, [n, 512]."""
    x, S, D, inter, ok = features(rho, diag, types, emulate_bf16, faces, halo)
    f, _ = _forward_net(p, H, x, emulate_bf16)
    sc = np.where(ok, S / np.where(ok, D, 1.0), 0.0)[:, None]
    return np.where(inter & ok[:, None], sc * f.reshape(-1, 512), 0.0)


def _forward_net(p, H, x, emulate_bf16):
    W1, b1, W2, b2, W3 = unpack(p, H)
    r = bf16 if emulate_bf16 else (lambda a: a)
    W1, W2, W3 = r(W1), r(W2), r(W3)
    a1 = r(np.maximum(conv(x, W1) + b1, 0.0))
    a2 = r(np.maximum(conv(a1, W2) + b2, 0.0))
    f = conv(a2, W3)[..., 0]
    return f, (x, a1, a2, W1, W2, W3)


def tile_laplacian(e):
    """7-point Laplacian of [n, 512] cell values within each tile: 6 e - (neighbours inside the tile)."""
    g = np.asarray(e, dtype=np.float64).reshape(-1, 8, 8, 8)
    p = np.zeros((g.shape[0], 10, 10, 10))
    p[:, 1:9, 1:9, 1:9] = g
    nb = (p[:, :-2, 1:-1, 1:-1] + p[:, 2:, 1:-1, 1:-1] + p[:, 1:-1, :-2, 1:-1] + p[:, 1:-1, 2:, 1:-1] +
          p[:, 1:-1, 1:-1, :-2] + p[:, 1:-1, 1:-1, 2:])
    return (6.0 * g - nb).reshape(-1, 512)


def loss_and_grad(p, H, rho, diag, types, target, emulate_bf16=True, kind=0, faces=None, halo=None):
    """Mean loss and its gradient (layout of `layout(H)`); kind 0: sum e^2 per tile,
    kind 1: e^T L e with L = tile_laplacian."""
    x, S, D, inter, ok = features(rho, diag, types, emulate_bf16, faces, halo)
    n = x.shape[0]
    f, (x, a1, a2, W1, W2, W3) = _forward_net(p, H, x, emulate_bf16)
    r = bf16 if emulate_bf16 else (lambda a: a)
    tgt = np.asarray(target, dtype=np.float64).reshape(-1, 512) * np.where(ok, D / np.where(ok, S, 1.0), 0.0)[:, None]
    m = inter & ok[:, None]
    e = np.where(m, f.reshape(-1, 512) - tgt, 0.0)
    g = np.where(m, tile_laplacian(e), 0.0) if kind == 1 else e
    scale = 1.0 / (n * 512)
    loss = (e * g).sum() * scale
    dy = r(2.0 * g).reshape(n, 8, 8, 8, 1)
    gW3 = conv_weight_grad(a2, dy)
    dz2 = r(conv_input_grad(dy, W3) * (a2 > 0))
    gW2 = conv_weight_grad(a1, dz2)
    gb2 = dz2.sum((0, 1, 2, 3))
    dz1 = r(conv_input_grad(dz2, W2) * (a1 > 0))
    gW1 = conv_weight_grad(x, dz1)
    gb1 = dz1.sum((0, 1, 2, 3))
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel()]) * scale
    return loss, g


# ---------------------------------------------------------------------------------------
# The residual network (hidden = 32): conv 8->32, four residual blocks of two 3x3x3 convs
# at 32 channels, conv 32->1.
#   x1 = relu(conv(x0, W0) + b0)
#   block k: h_k = relu(conv(x_k, Wa_k) + ba_k); x_{k+1} = relu(x_k + conv(h_k, Wb_k) + bb_k)
#   f = conv(x5, Wo)
# The GPU rounds x0, the weights, x_k, h_k, 2 (f - t) and every back-propagated gradient
# that enters a convolution (the ReLU-masked pre-activation gradients) to BF16.
# ---------------------------------------------------------------------------------------
DEEP_BLOCKS = 4
DEEP_C = 32


def layout_deep():
    C, o = DEEP_C, {}
    o["W0"] = 0
    o["B0"] = C * 216
    base = o["B0"] + C
    blk = 2 * (C * 27 * C) + 2 * C
    for k in range(DEEP_BLOCKS):
        o[f"Wa{k}"] = base + k * blk
        o[f"Ba{k}"] = o[f"Wa{k}"] + C * 27 * C
        o[f"Wb{k}"] = o[f"Ba{k}"] + C
        o[f"Bb{k}"] = o[f"Wb{k}"] + C * 27 * C
    o["WO"] = base + DEEP_BLOCKS * blk
    o["n"] = o["WO"] + 27 * C
    return o


def unpack_deep(p):
    L, C = layout_deep(), DEEP_C
    p = np.asarray(p, dtype=np.float64)
    W0 = p[L["W0"]:L["B0"]].reshape(C, 27, 8)
    b0 = p[L["B0"]:L["B0"] + C]
    blocks = []
    for k in range(DEEP_BLOCKS):
        blocks.append((p[L[f"Wa{k}"]:L[f"Ba{k}"]].reshape(C, 27, C), p[L[f"Ba{k}"]:L[f"Wb{k}"]],
                       p[L[f"Wb{k}"]:L[f"Bb{k}"]].reshape(C, 27, C), p[L[f"Bb{k}"]:L[f"Bb{k}"] + C]))
    Wo = p[L["WO"]:L["n"]].reshape(1, 27, C)
    return W0, b0, blocks, Wo


def _forward_deep(p, x0, emulate_bf16):
    W0, b0, blocks, Wo = unpack_deep(p)
    r = bf16 if emulate_bf16 else (lambda a: a)
    W0, Wo = r(W0), r(Wo)
    blocks = [(r(Wa), ba, r(Wb), bb) for Wa, ba, Wb, bb in blocks]
    xs = [r(np.maximum(conv(x0, W0) + b0, 0.0))]
    hs = []
    for Wa, ba, Wb, bb in blocks:
        h = r(np.maximum(conv(xs[-1], Wa) + ba, 0.0))
        hs.append(h)
        xs.append(r(np.maximum(conv(h, Wb) + bb + xs[-1], 0.0)))
    f = conv(xs[-1], Wo)[..., 0]
    return f, (W0, blocks, Wo, xs, hs)


def forward_deep(p, rho, diag, types, emulate_bf16=True, faces=None, halo=None):
    """Correction (S/D) f of the residual network on INTERIOR cells, [n, 512]."""
    x, S, D, inter, ok = features(rho, diag, types, emulate_bf16, faces, halo)
    f, _ = _forward_deep(p, x, emulate_bf16)
    sc = np.where(ok, S / np.where(ok, D, 1.0), 0.0)[:, None]
    return np.where(inter & ok[:, None], sc * f.reshape(-1, 512), 0.0)


def loss_and_grad_deep(p, rho, diag, types, target, emulate_bf16=True, kind=0, faces=None, halo=None):
    """Mean loss of the residual network and its gradient (layout of `layout_deep()`)."""
    x0, S, D, inter, ok = features(rho, diag, types, emulate_bf16, faces, halo)
    n = x0.shape[0]
    f, (W0, blocks, Wo, xs, hs) = _forward_deep(p, x0, emulate_bf16)
    r = bf16 if emulate_bf16 else (lambda a: a)
    tgt = np.asarray(target, dtype=np.float64).reshape(-1, 512) * np.where(ok, D / np.where(ok, S, 1.0), 0.0)[:, None]
    m = inter & ok[:, None]
    e = np.where(m, f.reshape(-1, 512) - tgt, 0.0)
    g = np.where(m, tile_laplacian(e), 0.0) if kind == 1 else e
    scale = 1.0 / (n * 512)
    loss = (e * g).sum() * scale
    dy = r(2.0 * g).reshape(n, 8, 8, 8, 1)
    L = layout_deep()
    grad = np.zeros(L["n"])
    grad[L["WO"]:L["n"]] = conv_weight_grad(xs[-1], dy).ravel()
    d = r(conv_input_grad(dy, Wo) * (xs[-1] > 0))  # gradient of block 3's pre-activation
    for k in range(DEEP_BLOCKS - 1, -1, -1):
        Wa, ba, Wb, bb = blocks[k]
        grad[L[f"Bb{k}"]:L[f"Bb{k}"] + DEEP_C] = d.sum((0, 1, 2, 3))
        grad[L[f"Wb{k}"]:L[f"Bb{k}"]] = conv_weight_grad(hs[k], d).ravel()
        da = r(conv_input_grad(d, Wb) * (hs[k] > 0))
        grad[L[f"Ba{k}"]:L[f"Wb{k}"]] = da.sum((0, 1, 2, 3))
        grad[L[f"Wa{k}"]:L[f"Ba{k}"]] = conv_weight_grad(xs[k], da).ravel()
        d = r((d + conv_input_grad(da, Wa)) * (xs[k] > 0))
    grad[L["B0"]:L["B0"] + DEEP_C] = d.sum((0, 1, 2, 3))
    grad[L["W0"]:L["B0"]] = conv_weight_grad(x0, d).ravel()
    return loss, grad * scale
