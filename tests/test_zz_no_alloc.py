"""The allocation-free closest-hit call, checked against the ordinary one.

vt_bvh_trace_closest_noalloc serves callers that cannot allocate device
memory (a host with a fixed, pre-reserved device budget, or host-array callers
such as the Node addon on a path where no cudaMalloc may happen).  Its scratch
is one library-wide device array, so this test makes two calls in a row on
different ray batches -- the second sees whatever the first left in the array
-- and each must equal what vt_bvh_trace_closest returns for the same rays.
A further test checks the property the call exists for: after the set-up
call, full-size calls leave the device's free memory unchanged.  Runs last
(file name) and passes alone or after the other tests.
"""
import ctypes

import numpy as np
import pytest

from vitrum_b200 import _native as N
from vitrum_b200 import bvh as vb
from vitrum_b200 import scenes

pytestmark = pytest.mark.gpu

MAX_RAYS = 65536
HIT = vb.HIT_DTYPE


def _noalloc(bvh, rays):
    rays = np.ascontiguousarray(rays, dtype=np.float32)
    out = np.empty(rays.shape[0], dtype=HIT)
    N.call("vt_bvh_trace_closest_noalloc", bvh.handle, ctypes.c_void_p(rays.ctypes.data), rays.shape[0],
           ctypes.c_void_p(out.ctypes.data))
    return out


def test_noalloc_matches_trace_closest_on_two_calls(cuda):
    soup = scenes.random_triangles(20000, seed=77)
    g = vb.build_compressed_wide_bvh(soup.positions, soup.indices)
    first = scenes.sphere_rays(MAX_RAYS, seed=78)          # the full staging capacity
    second = scenes.sphere_rays(12345, seed=79)            # smaller: stale tail from the first call
    for rays in (first, second):
        want = g.intersect_first_hit(rays)
        got = _noalloc(g, rays)
        assert np.array_equal(got["prim"], want["prim"])
        hit = want["prim"] >= 0
        assert hit.sum() > 0.5 * rays.shape[0]
        # same kernels, same inputs: identical records (tolerance of the parity tests: 1e-5 rel / abs)
        assert np.allclose(got["t"][hit], want["t"][hit], rtol=1e-5, atol=0)
        assert np.allclose(got["u"][hit], want["u"][hit], rtol=0, atol=1e-5)
        assert np.allclose(got["v"][hit], want["v"][hit], rtol=0, atol=1e-5)
    g.close()


def test_noalloc_rejects_batches_beyond_its_scratch(cuda):
    soup = scenes.random_triangles(100, seed=80)
    g = vb.build_compressed_wide_bvh(soup.positions, soup.indices)
    rays = scenes.sphere_rays(MAX_RAYS + 1, seed=81)
    with pytest.raises(N.VtError) as e:
        _noalloc(g, rays)
    assert e.value.status == 2 and "65536" in str(e.value)
    assert _noalloc(g, rays[:0]).size == 0
    g.close()


def test_noalloc_calls_leave_free_device_memory_unchanged(cuda):
    import torch
    soup = scenes.random_triangles(5000, seed=82)
    g = vb.build_compressed_wide_bvh(soup.positions, soup.indices)
    rays = scenes.sphere_rays(MAX_RAYS, seed=83)
    _noalloc(g, rays[:0])          # set-up call: loads the module, resolves the scratch address
    want = _noalloc(g, rays)       # and one full call, so every kernel it launches is loaded
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        got = _noalloc(g, rays)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert np.array_equal(got["prim"], want["prim"])
    # an allocation the size of the staging (3 MiB) would show here
    assert free1 == free0, (free0, free1)
    g.close()
