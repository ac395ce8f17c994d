"""The engine builds its scenes on the GPU (scene_build "gpu", the default):
the binned-SAH trees, their SAH-optimal 8-wide encodings and, for instanced
scenes, the top level over the instance bounds (the reference's buildTlas
rules) with its instance records.  The device arrays equal those of the host
pipeline (scene_build "host") word for word -- single-level scenes, instanced
scenes with planar meshes whose bounds hold signed zeros, top-level rebuilds and
refits after instance updates, and mesh updates -- and a debug engine's
structural proofs accept every tree the GPU publishes."""
import dataclasses
import time

import numpy as np
import pytest

from vitrum_b200 import scenes
from vitrum_b200.engine import Engine, Instance, Mesh

pytestmark = pytest.mark.gpu


def export(sc, build, debug=False, width=0):
    e = Engine(max_bounces=2, scene_build=build, debug=debug, bvh_width=width)
    t0 = time.perf_counter()
    e.set_scene(sc)
    dt = time.perf_counter() - t0
    words, recs = e.export_scene()
    tl = e.export_tlas() if sc.instances else None
    return e, words, recs, tl, dt


def same(a, b):
    ew, er = a[1], b[1]
    assert np.array_equal(a[1], b[1])
    assert np.array_equal(a[2].view(np.uint32), b[2].view(np.uint32))
    if a[3] is not None:
        assert all(np.array_equal(x, y) for x, y in zip(a[3], b[3]))


def test_single_level_box_room(cuda):
    sc, _ = scenes.box_room(wall_cells=64, box_cells=32)
    g, h = export(sc, "gpu"), export(sc, "host")
    same(g, h)
    print(f"box room {sc.triangle_count} triangles: set_scene GPU {g[4] * 1e3:.0f} ms, host {h[4] * 1e3:.0f} ms")
    g[0].dispose()
    h[0].dispose()


@pytest.mark.parametrize("width", [4, 6])
def test_collapse_widths_gpu_equals_host(cuda, width):
    """Narrower SAH-optimal collapses (at most `width` children per wide node):
    the GPU encoding equals the host's word for word, a debug engine's proofs
    accept it, and the first hits are those of the full-width tree."""
    sc, cam = scenes.box_room(wall_cells=32, box_cells=16)
    g, h = export(sc, "gpu", debug=True, width=width), export(sc, "host", width=width)
    same(g, h)
    full = export(sc, "gpu")
    assert g[1].size > full[1].size  # more, narrower nodes
    rays = np.concatenate([scenes.sphere_rays(20000, seed=31, radius=2.0, target_half=0.4)])
    rays[:, :3] += 0.5
    a, _ = g[0].trace_rays(rays)
    b, _ = full[0].trace_rays(rays)
    assert np.array_equal(a["prim"], b["prim"]) and np.array_equal(a["t"], b["t"])
    for x in (g, h, full):
        x[0].dispose()


def test_bvh_shape_autotune(cuda):
    """vt_engine_autotune_bvh tries leaf sizes and widths, keeps the fastest and
    leaves the scene set in that shape: a frame renders as a fresh engine
    created with that shape renders it."""
    sc, cam = scenes.box_room(wall_cells=16, box_cells=8)
    e = Engine(max_bounces=3)
    trials = e.autotune_bvh(sc, cam, 64, 64, samples=4)
    assert len(trials) == 6
    assert {(t["bvh_width"], t["bvh_max_leaf"]) for t in trials} >= {(8, 1), (8, 2), (8, 3), (8, 4)}
    kept = (8, 2)  # the starting shape; a candidate replaces it only when 0.5 % faster
    best_ms = trials[0]["frame_ms"]
    for t in trials[1:4]:
        if t["frame_ms"] < best_ms * 0.995:
            kept, best_ms = (8, t["bvh_max_leaf"]), t["frame_ms"]
    for t in trials[4:]:
        if t["frame_ms"] < best_ms * 0.995:
            kept, best_ms = (t["bvh_width"], kept[1]), t["frame_ms"]
    best = {"bvh_width": kept[0], "bvh_max_leaf": kept[1]}
    e.render_frame(cam, 32, 32, samples=8)
    img = e.capture_frame()
    f = Engine(max_bounces=3, bvh_width=best["bvh_width"], bvh_max_leaf=best["bvh_max_leaf"])
    f.set_scene(sc)
    f.render_frame(cam, 32, 32, samples=8)
    assert np.array_equal(img, f.capture_frame())
    with pytest.raises(Exception):
        Engine(bvh_width=9)
    e.dispose()
    f.dispose()


def planar_cloud():
    sc, cam = scenes.instanced_cloud(n_instances=96, seed=9, n_points=4, sphere_levels=(1, 2),
                                     torus_segments=(24, 8), cube_cells=(3, 5), extent=6.0)
    # a flat quad at y = 0 placed without rotation: its bounds hold exact zeros
    quad = Mesh(np.array([[-1, 0, -1], [1, 0, -1], [1, 0, 1], [-1, 0, 1]], np.float32),
                np.array([[0, 1, 2], [0, 2, 3]], np.uint32), 0)
    meshes = list(sc.meshes) + [quad]
    q = len(meshes) - 1
    eye = np.eye(4, dtype=np.float32)
    flip = np.diag([-1.0, 1.0, 1.0, 1.0]).astype(np.float32)
    extra = [Instance(q, eye, 0), Instance(q, flip, 0), Instance(q, eye, 1)]
    return dataclasses.replace(sc, meshes=meshes, instances=list(sc.instances) + extra), cam


def test_instanced_scene_and_updates(cuda):
    sc, _ = planar_cloud()
    g, h = export(sc, "gpu"), export(sc, "host")
    same(g, h)
    rng = np.random.default_rng(3)
    moved = []
    for inst in sc.instances:
        t = np.array(inst.local_to_world, np.float32).copy()
        t[:3, 3] += rng.normal(0, 0.5, 3).astype(np.float32)
        moved.append(dataclasses.replace(inst, local_to_world=t))
    for rebuild in (False, True):
        for eng in (g[0], h[0]):
            eng.update_instances(moved, rebuild=rebuild)
        same((None, *g[0].export_scene(), g[0].export_tlas()), (None, *h[0].export_scene(), h[0].export_tlas()))
    p, t = scenes.icosphere(2)
    new_mesh = Mesh((p * 0.7).astype(np.float32), t, 0)
    for eng in (g[0], h[0]):
        eng.update_mesh(0, new_mesh, rebuild=True)
    same((None, *g[0].export_scene(), g[0].export_tlas()), (None, *h[0].export_scene(), h[0].export_tlas()))
    g[0].dispose()
    h[0].dispose()


def test_debug_engine_proves_gpu_trees(cuda):
    for sc in (scenes.box_room(wall_cells=16, box_cells=8)[0], planar_cloud()[0]):
        e = Engine(max_bounces=2, scene_build="gpu", debug=True)
        e.set_scene(sc)  # the structural proofs run on every tree and raise on a violation
        e.dispose()


def test_scene_build_option_validation(cuda):
    with pytest.raises(KeyError):
        Engine(scene_build="cpu")
