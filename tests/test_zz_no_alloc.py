"""cmg_amg_dot_noalloc: the allocation-free dot product, called through the C ABI.

Some callers cannot allocate device memory at the point of the call: a simulator that
hands the whole GPU to its own memory pool at start-up, and a time-critical loop that
must not call cudaFree (which synchronises the device).  This entry point keeps its
scratch in a fixed static device array instead.  The tests check, on two calls in a row,
that it returns exactly cmg_amg_dot's result (the same summation order, so the same
bits), that many calls leave the device's free memory unchanged, and that grids beyond
the fixed scratch are refused.  The file name makes pytest collect it last, so it also
runs after every other GPU test has used the device."""
import ctypes
import struct

import numpy as np
import pytest

import cmg
from workloads import setup_shell, setup_uniform, shell_params

pytestmark = pytest.mark.gpu


def _dot_noalloc(G, a, b):
    out = ctypes.c_double(0.0)
    rc = cmg.lib().cmg_amg_dot_noalloc(G.h, a, b, ctypes.byref(out))
    return rc, out.value


def _bits(x):
    return struct.pack("<d", x)


def _random_planes(G, seed):
    rng = np.random.default_rng(seed)
    for ch in (1, 4):
        G.upload(ch, rng.standard_normal((G.num_tiles, 512)).astype(np.float32))


def _grid(name):
    if name == "uniform64":
        G, _, _, _ = setup_uniform(3, with_oracle=False)
    else:
        G, _, _ = setup_shell(shell_params(coarse=3, mid=4, fine=5), with_oracle=False)
    _random_planes(G, 5)
    return G


@pytest.mark.parametrize("grid", ["uniform64", "shell345"])
def test_noalloc_dot_equals_dot_bit_for_bit_on_two_calls(grid):
    G = _grid(grid)
    for a, b in ((1, 4), (1, 1)):
        want = G.dot(a, b)
        for _ in range(2):
            rc, got = _dot_noalloc(G, a, b)
            assert rc == 0, cmg.lib().cmg_last_error()
            assert _bits(got) == _bits(want), (got, want)


def test_noalloc_dot_allocates_nothing():
    import torch

    G = _grid("shell345")
    rc, want = _dot_noalloc(G, 1, 4)  # first call: the scratch address lookup
    assert rc == 0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(200):
        rc, got = _dot_noalloc(G, 1, 4)
        assert rc == 0 and _bits(got) == _bits(want)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] >= free0


def test_noalloc_dot_rejects_grids_beyond_its_scratch():
    # uniform 256^3: 32768 LEAF tiles, twice the fixed scratch; rejected before any device work
    G = cmg.HADeviceGrid(0.125, 10, 2)
    G.set_tile_host(0, (0, 0, 0), cmg.LEAF)
    G.rebuild()
    G.refine_case(cmg.CASE_UNIFORM, [5, 5])
    rc, _ = _dot_noalloc(G, 0, 1)
    assert rc == 1  # CMG_ERR_INVALID
    assert b"16384" in cmg.lib().cmg_last_error()
