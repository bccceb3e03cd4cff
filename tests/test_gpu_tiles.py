"""A view of the reference's own device tiles (cmg_grid_gather_device_tiles /
cmg_grid_scatter_device_tiles): raw PoissonTile<float,15> structs (src/PoissonTile.h:34-39,
44880 bytes: float mData[15][736], uint8 mCellType[512] at byte 44352) anywhere in device
memory, reached through a list of tile addresses."""
import numpy as np
import pytest

import cmg
from workloads import setup_shell, shell_params

pytestmark = pytest.mark.gpu

TILE, TYPES, STRIDE = 44880, 44352, 736


def test_gather_and_scatter_through_tile_addresses():
    import torch

    G, _, _ = setup_shell(shell_params(coarse=3, mid=4, fine=5), with_oracle=False)
    n = G.num_tiles
    rng = np.random.default_rng(12)
    tiles = np.full((n, TILE), 0xAB, np.uint8)  # neighbour infos, flags: must stay untouched
    data = rng.standard_normal((n, 15, STRIDE)).astype(np.float32)
    tiles[:, :15 * STRIDE * 4] = data.reshape(n, -1).view(np.uint8)
    types = rng.choice(np.array([cmg.DIRICHLET, cmg.INTERIOR, cmg.NEUMANN], np.uint8), size=(n, 512))
    tiles[:, TYPES:TYPES + 512] = types
    # tile t of the grid lives in slot perm[t] of the buffer
    perm = rng.permutation(n)
    host = np.empty_like(tiles)
    host[perm] = tiles
    buf = torch.from_numpy(host.reshape(-1)).cuda()
    ptrs = [buf.data_ptr() + int(perm[t]) * TILE for t in range(n)]

    G.gather_device_tiles(ptrs, 0, 15, True)
    for c in range(15):
        assert np.array_equal(G.download(c), data[:, c, :512]), c
    assert np.array_equal(G.download_cell_types(), types)

    x = rng.standard_normal((n, 512)).astype(np.float32)
    G.upload(0, x)
    G.scatter_device_tiles(ptrs, 0, 1)
    out = buf.cpu().numpy().reshape(n, TILE)[perm]
    expected = tiles.copy()
    expected[:, :512 * 4] = x.view(np.uint8)
    assert np.array_equal(out, expected)


def test_tile_view_rejects_a_wrong_tile_size():
    G, _, _ = setup_shell(shell_params(coarse=3, mid=4, fine=5), with_oracle=False)
    arr = (cmg.ctypes.c_void_p * G.num_tiles)(*([16] * G.num_tiles))
    assert cmg.lib().cmg_grid_gather_device_tiles(G.h, arr, 44000, 0, 1, 0) != 0
