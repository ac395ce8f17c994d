"""Mesh updates of a two-level scene (vt_update_mesh), the reference's
rebuildPrimitiveBlas (shared-bvh/src/scenePack.ts:1763) with its in-place
splice (same sizes) and its resized splice (later meshes rebased,
:1006-1100).  After an update the engine must answer exactly what an engine
given the changed scene from scratch answers: closest hits do not depend on
where a bottom level sits in the concatenated arrays, so hits, instance ids
and images agree (exact up to float ties)."""
import dataclasses

import numpy as np
import pytest

from vitrum_b200 import _native as N
from vitrum_b200 import scenes
from vitrum_b200.engine import Engine, Mesh

from test_gpu_instance_update import rays_at, small_cloud

pytestmark = pytest.mark.gpu


def check_same(e, sc, cam, rays):
    h, ii = e.trace_rays(rays)
    e.render_frame(cam, 32, 24, samples=8, frame_seed=5)
    img = e.capture_frame().copy()
    f = Engine(max_bounces=4)
    f.set_scene(sc)
    hf, iif = f.trace_rays(rays)
    f.render_frame(cam, 32, 24, samples=8, frame_seed=5)
    imgf = f.capture_frame().copy()
    f.dispose()
    assert (hf["prim"] >= 0).mean() > 0.2
    same = (h["prim"] == hf["prim"]) & (ii == iif)
    assert same.mean() > 0.9999, same.mean()
    assert np.allclose(h["t"][same], hf["t"][same], rtol=1e-6)
    assert np.isclose(img, imgf, rtol=1e-4, atol=1e-6).mean() > 0.999


@pytest.mark.parametrize("rebuild", [False, True])
def test_mesh_updates_equal_a_fresh_scene(cuda, rebuild):
    sc, cam = small_cloud()
    rays = rays_at(1 << 16, 17)
    e = Engine(max_bounces=4)
    e.set_scene(sc)
    e.render_frame(cam, 32, 24, samples=2)
    meshes = list(sc.meshes)
    # 1) same topology, moved vertices (in-place splice when the tree keeps its size)
    m0 = meshes[0]
    p = np.asarray(m0.positions, np.float32) * np.float32(1.3) + np.float32(0.05)
    meshes[0] = Mesh(p, m0.indices, m0.material)
    # 2) a different mesh in the middle (resized splice: later meshes rebased)
    k = len(meshes) // 2
    p2, t2 = scenes.icosphere(3)
    meshes[k] = Mesh(p2 * np.float32(0.8), t2, meshes[k].material)
    # 3) the last mesh shrinks to a few triangles
    p3, t3 = scenes.box_mesh((-0.5, -0.5, -0.5), (0.5, 0.5, 0.5), 1)
    meshes[-1] = Mesh(p3, t3, meshes[-1].material)
    cur = list(sc.meshes)
    for i in (0, k, len(meshes) - 1):  # one mesh at a time, each compared with a fresh scene
        cur[i] = meshes[i]
        e.update_mesh(i, meshes[i], rebuild=rebuild)
        check_same(e, dataclasses.replace(sc, meshes=list(cur)), cam, rays)
    assert e.stats()["triangle_count"] == sum(len(m.indices) for m in meshes)
    # and instance updates still work on the spliced arrays
    from test_gpu_instance_update import moved
    n_mat = len(sc.materials)
    new = [dataclasses.replace(i, material=i.material % n_mat) for i in moved(sc.instances, 4)]
    e.update_instances(new, rebuild=rebuild)
    check_same(e, dataclasses.replace(sc, meshes=list(meshes), instances=new), cam, rays)
    e.dispose()


def test_mesh_update_validation(cuda):
    sc, cam = small_cloud()
    e = Engine(max_bounces=4)  # as the fresh engine of check_same
    e.set_scene(sc)
    m = sc.meshes[0]
    with pytest.raises(N.VtError):
        e.update_mesh(len(sc.meshes), m)                                   # no such mesh
    with pytest.raises(N.VtError):
        e.update_mesh(0, Mesh(m.positions, np.full_like(m.indices, 10 ** 6), m.material))  # index out of range
    bad = np.asarray(m.positions, np.float32).copy()
    bad[0, 0] = np.nan
    with pytest.raises(N.VtError):
        e.update_mesh(0, Mesh(bad, m.indices, m.material))                 # non-finite vertex
    with pytest.raises(N.VtError):
        e.update_mesh(0, Mesh(m.positions, m.indices, 10 ** 6))            # no such material
    # the failed calls changed nothing
    check_same(e, sc, cam, rays_at(1 << 12, 3))
    assert "mesh-updates" in e.capabilities["features"]
    e.dispose()
    room, _ = scenes.box_room(wall_cells=4, box_cells=2)
    e = Engine(max_bounces=2)
    e.set_scene(room)
    with pytest.raises(N.VtError):
        e.update_mesh(0, room.meshes[0])                                   # flat scene: set it again
    e.dispose()
