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


def export(sc, build, debug=False):
    e = Engine(max_bounces=2, scene_build=build, debug=debug)
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
