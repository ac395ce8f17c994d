"""Shared-memory staging of the top of the tree in the traversal kernel.

With staging on, every traversal CTA first copies the root and the next two
8-wide levels below it (breadth-first prefix) into shared memory with one bulk
copy and reads those nodes from there.  Where a node is read from does not
change what the traversal computes, so hits, instance ids and rendered images
must be bit-identical with staging on and off, on single-level and two-level
(TLAS root) scenes.
"""
import numpy as np
import pytest

from vitrum_b200 import _native as N
from vitrum_b200 import scenes
from vitrum_b200.engine import Engine

pytestmark = pytest.mark.gpu


def _rays_through(cam, n, seed, extent):
    # from around the eye towards points around the camera target
    u = scenes.uniform(seed, 31, 6 * n).reshape(n, 6)
    o = np.asarray(cam.eye, np.float64) + (u[:, 0:3] - 0.5) * 0.1 * extent
    tgt = np.asarray(cam.target, np.float64) + (u[:, 3:6] * 2 - 1) * extent
    d = tgt - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 4:7] = d
    rays[:, 7] = 1e30
    return rays


@pytest.mark.parametrize("kind", ["box_room", "instanced"])
def test_staging_is_bit_identical(cuda, kind):
    if kind == "box_room":
        sc, cam = scenes.box_room()
        extent = 0.5
    else:
        sc, cam = scenes.instanced_cloud(n_instances=64, seed=3, n_points=4, sphere_levels=(1, 2),
                                         torus_segments=(24, 8), cube_cells=(3, 5), extent=4.0)
        extent = 4.0
    out = {}
    for stage in (False, True):
        e = Engine(max_bounces=4)
        e.set_scene(sc)
        # 4 CTAs per SM leaves room for the staged nodes at any stack depth
        e.set_tuning(wave_paths=1 << 16, trace_blocks_per_sm=4, stage_hot_nodes=stage)
        assert e.tuning["stage_hot_nodes"] == (1 if stage else 0)
        hits, inst = e.trace_rays(_rays_through(cam, 1 << 16, 7, extent))
        e.render_frame(cam, 48, 40, samples=4, frame_seed=11)
        out[stage] = (hits, inst, e.capture_frame().copy())
        e.dispose()
    h0, i0, f0 = out[False]
    h1, i1, f1 = out[True]
    assert (h0["prim"] >= 0).mean() > 0.3
    assert np.array_equal(h0.view(np.uint8), h1.view(np.uint8))
    assert np.array_equal(i0, i1)
    assert np.array_equal(f0.view(np.uint32), f1.view(np.uint32))


def test_set_tuning_validation(cuda):
    sc, cam = scenes.box_room()
    e = Engine(max_bounces=2)
    e.set_scene(sc)
    for bad in (dict(wave_paths=10), dict(trace_blocks_per_sm=17), dict(trace_blocks_per_sm=-1), dict(sort_rays=4),
                dict(nrc_infer_tiles=5)):
        with pytest.raises(N.VtError):
            e.set_tuning(**bad)
    e.set_tuning(wave_paths=1 << 18, sort_by_material=True, trace_blocks_per_sm=6, stage_hot_nodes=True)
    # nrc_infer_tiles reads 0 on an engine without the radiance cache
    assert e.tuning == {"wave_paths": 1 << 18, "sort_by_material": 1, "trace_blocks_per_sm": 6, "stage_hot_nodes": 1,
                        "sort_rays": 0, "nrc_infer_tiles": 0}
    e.render_frame(cam, 16, 16, samples=2)
    e.dispose()
