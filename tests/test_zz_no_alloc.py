"""cmg_amg_dot_noalloc: the allocation-free dot product, called through the C ABI and
compared with cmg_amg_dot on two calls in a row.  Collected last (file name) so it also
runs after every other GPU test has used the device."""
import ctypes

import numpy as np
import pytest

import cmg
from workloads import setup_shell, setup_uniform, shell_params

pytestmark = pytest.mark.gpu


def _dot_noalloc(G, a, b):
    out = ctypes.c_double(0.0)
    rc = cmg.lib().cmg_amg_dot_noalloc(G.h, a, b, ctypes.byref(out))
    return rc, out.value


def _random_planes(G, seed):
    rng = np.random.default_rng(seed)
    for ch in (1, 4):
        G.upload(ch, rng.standard_normal((G.num_tiles, 512)).astype(np.float32))


@pytest.mark.parametrize("grid", ["uniform64", "shell345"])
def test_noalloc_dot_matches_dot_on_two_calls(grid):
    if grid == "uniform64":
        G, _, _, _ = setup_uniform(3, with_oracle=False)
    else:
        G, _, _ = setup_shell(shell_params(coarse=3, mid=4, fine=5), with_oracle=False)
    _random_planes(G, 5)
    want = G.dot(1, 4)
    for _ in range(2):
        rc, got = _dot_noalloc(G, 1, 4)
        assert rc == 0, cmg.lib().cmg_last_error()
        assert got == pytest.approx(want, rel=1e-12, abs=1e-12)
    assert _dot_noalloc(G, 1, 1)[1] == pytest.approx(G.dot(1, 1), rel=1e-12)


def test_noalloc_dot_rejects_grids_beyond_its_scratch():
    # uniform 256^3: 32768 LEAF tiles, twice the fixed scratch; rejected before any device work
    G = cmg.HADeviceGrid(0.125, 10, 2)
    G.set_tile_host(0, (0, 0, 0), cmg.LEAF)
    G.rebuild()
    G.refine_case(cmg.CASE_UNIFORM, [5, 5])
    rc, _ = _dot_noalloc(G, 0, 1)
    assert rc == 1  # CMG_ERR_INVALID
    assert b"16384" in cmg.lib().cmg_last_error()
