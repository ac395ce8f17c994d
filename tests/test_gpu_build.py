"""The GPU build (vt_bvh_build_device) produces the host build's trees word
for word: the binned-SAH binary tree (and so the reference's buildArrayBvh
tree: node words and triangle order) and its 8-wide encoding (node words and
triangle records), for random soups, planar grids (SAH ties and the balanced
fallback), coincident centroids (the large-node fallback), every leaf size and
bin counts from 2 to 256, and both strides."""
import time

import numpy as np
import pytest
import torch

import oracle
from vitrum_b200 import _native as N
from vitrum_b200 import bvh as vb
from vitrum_b200 import scenes

pytestmark = pytest.mark.gpu


def both(pos, idx, **opts):
    host = vb.build_compressed_wide_bvh(pos, idx, **opts)
    hn, hr = host.export_binary()
    dp = torch.from_numpy(np.ascontiguousarray(pos, np.float32).reshape(-1)).cuda()
    di = torch.from_numpy(np.ascontiguousarray(idx, np.uint32).reshape(-1).view(np.int32)).cuda()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    dev = vb.build_compressed_wide_bvh_device(dp.data_ptr(), dp.numel(), di.data_ptr(), di.numel(), **opts)
    dt = time.perf_counter() - t0
    dn, dr = dev.export_binary()
    hw, hrec = host.export_wide()
    dw, drec = dev.export_wide()
    host.close()
    dev.close()
    # the 8-wide encodings too (records compared bit for bit)
    assert np.array_equal(hw, dw) and np.array_equal(hrec.view(np.uint32), drec.view(np.uint32))
    return (hn, hr), (dn, dr), dt


def soup(n, seed, sigma=0.02):
    s = scenes.random_triangles(n, seed=seed, sigma=sigma)
    return s.positions, s.indices


@pytest.mark.parametrize("n", [1, 3, 5, 17, 100, 4096, 65536])
def test_random_soups(cuda, n):
    pos, idx = soup(n, 100 + n)
    (hn, hr), (dn, dr), _ = both(pos, idx)
    assert np.array_equal(hn, dn) and np.array_equal(hr, dr)


@pytest.mark.parametrize("leaf,bins", [(1, 16), (2, 8), (3, 2), (4, 16), (4, 5), (2, 32), (4, 64), (1, 256)])
def test_options(cuda, leaf, bins):
    pos, idx = soup(3000, 7)
    (hn, hr), (dn, dr), _ = both(pos, idx, maxLeafTriangles=leaf, binCount=bins)
    assert np.array_equal(hn, dn) and np.array_equal(hr, dr)


def test_stride_three(cuda):
    pos, idx = soup(2000, 8)
    p3 = np.ascontiguousarray(pos[:, :3])
    i3 = np.ascontiguousarray(idx[:, :3])
    (hn, hr), (dn, dr), _ = both(p3, i3, positionStride=3, indexStride=3)
    assert np.array_equal(hn, dn) and np.array_equal(hr, dr)


def test_planar_grid_and_box_room(cuda):
    sc, _ = scenes.box_room(wall_cells=32, box_cells=16)
    flat = oracle.flatten_scene(sc)
    (hn, hr), (dn, dr), _ = both(flat[0], flat[1])
    assert np.array_equal(hn, dn) and np.array_equal(hr, dr)


def test_coincident_centroids_large_fallback(cuda):
    # 6000 copies of one triangle: no split improves SAH, every node takes the
    # balanced fallback, the root's sort is larger than the shared-memory sort
    pos = np.array([[0, 0, 0, 0], [1, 0, 0, 0], [0, 1, 0, 0]], np.float32)
    idx = np.tile(np.array([[0, 1, 2, 0]], np.uint32), (6000, 1))
    (hn, hr), (dn, dr), _ = both(pos, idx)
    assert np.array_equal(hn, dn) and np.array_equal(hr, dr)


def test_errors_match_host(cuda):
    pos = np.array([[0, 0, 0, 0], [1, 0, 0, 0], [0, 1, 0, 0]], np.float32)
    idx = np.tile(np.array([[0, 1, 2, 0]], np.uint32), (64, 1))
    with pytest.raises(N.VtError):
        both(pos, idx, maxDepth=2)               # depth cap cannot hold leaves of 4
    bad = np.array([[0, 1, 7, 0]], np.uint32)
    dp = torch.from_numpy(pos.reshape(-1)).cuda()
    di = torch.from_numpy(bad.reshape(-1).view(np.int32)).cuda()
    with pytest.raises(N.VtError):
        vb.build_compressed_wide_bvh_device(dp.data_ptr(), dp.numel(), di.data_ptr(), di.numel())


def test_large_build_time(cuda):
    pos, idx = soup(1 << 21, 5)
    (hn, hr), (dn, dr), dt = both(pos, idx)
    print(f"2,097,152 triangles: device build (binary tree and 8-wide encoding on the GPU, copies for the "
          f"publication proofs) {dt * 1e3:.0f} ms")
    assert np.array_equal(hn, dn) and np.array_equal(hr, dr)
