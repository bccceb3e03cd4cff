"""'HAGR' v1 grid blobs (HADeviceGrid::dumpBinaryBlob / loadBinaryBlob, src/HAGrid.h:687-853)."""
import struct

import numpy as np
import pytest

import cmg
from workloads import setup_shell, shell_params

pytestmark = pytest.mark.gpu

TILE_BYTES, TYPES_AT, STRIDE = 44880, 44352, 736


def _reference_blob(records, h0=0.125, num_levels=10, hashes=None):
    """A blob written from the reference's struct layout: records = [(level, type, (i,j,k), data[15][512], types[512])]."""
    head = struct.pack("<IIIiIIf4xQ", 0x52474148, 1, num_levels, max(r[0] for r in records), TILE_BYTES, 12, h0, len(records))
    head += b"".join(struct.pack("<I", 8 if hashes is None else hashes[l]) for l in range(num_levels))
    body = b""
    for level, ty, c, data, types in records:
        tile = bytearray(TILE_BYTES)
        for ch in range(15):
            tile[ch * STRIDE * 4: ch * STRIDE * 4 + 2048] = np.asarray(data[ch], np.float32).tobytes()
        tile[TYPES_AT: TYPES_AT + 512] = np.asarray(types, np.uint8).tobytes()
        body += struct.pack("<IB3i", level, ty, *c) + bytes(tile)
    return head + body


def test_load_pins_the_reference_layout_and_dump_reproduces_it():
    data = (np.arange(15)[:, None] * 1000 + np.arange(512)[None, :]).astype(np.float32)
    types = (np.arange(512) % 3 == 0) * 2 + 1
    blob = _reference_blob([(0, cmg.LEAF, (0, 0, 0), data, types)])
    G = cmg.HADeviceGrid.loadBinaryBlob(blob, num_channels=16)
    assert G.num_tiles == 1
    for ch in range(15):
        assert np.array_equal(G.download(ch)[0], data[ch])
    assert not G.download(15).any()
    assert np.array_equal(G.download_cell_types()[0], types.astype(np.uint8))
    assert G.dumpBinaryBlob() == blob


def test_round_trip_of_the_sphere_octree():
    G, _, _ = setup_shell(shell_params(coarse=3, mid=4, fine=5), with_oracle=False)
    rng = np.random.default_rng(2)
    planes = [rng.standard_normal((G.num_tiles, 512)).astype(np.float32) for _ in range(16)]
    for ch, p in enumerate(planes):
        G.upload(ch, p)
    blob = G.dumpBinaryBlob()
    H = cmg.HADeviceGrid.loadBinaryBlob(blob, num_channels=16)
    for a, b in zip(G.tiles(), H.tiles()):
        assert np.array_equal(a, b)
    assert np.array_equal(G.download_cell_types(), H.download_cell_types())
    for ch in range(15):
        assert np.array_equal(H.download(ch), planes[ch])
    assert not H.download(15).any()
    G.fill(15, 0.0)
    assert H.dumpBinaryBlob() == blob


@pytest.mark.parametrize("damage", ["magic", "truncated", "tile_size"])
def test_load_rejects_damaged_blobs(damage):
    data = np.zeros((15, 512), np.float32)
    blob = bytearray(_reference_blob([(0, cmg.LEAF, (0, 0, 0), data, np.full(512, 2))]))
    if damage == "magic":
        blob[0] ^= 0xFF
    elif damage == "truncated":
        blob = blob[:-100]
    else:
        blob[16] ^= 0x01
    with pytest.raises(cmg.CmgError):
        cmg.HADeviceGrid.loadBinaryBlob(bytes(blob))
