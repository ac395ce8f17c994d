"""Instance updates without bottom-level rebuilds (vt_update_instances):
refitTlasTransforms (shared-bvh/src/scenePack.ts:1310; refitTlas,
tlas.ts:990-1012) keeps the top level's topology and takes the moved
instances' bounds, rebuildTlasReuseBlas (scenePack.ts:1635) builds a new top
level.  Either way the engine must then answer exactly what an engine given
the moved scene from scratch answers: the traversal's closest hits do not
depend on the tree's shape, so hits, instance ids and images agree (exact up
to float ties)."""
import dataclasses

import numpy as np
import pytest

from vitrum_b200 import _native as N
from vitrum_b200 import scenes
from vitrum_b200.engine import Engine, Instance

pytestmark = pytest.mark.gpu


def small_cloud():
    return scenes.instanced_cloud(n_instances=48, seed=5, n_points=4, sphere_levels=(1, 2), torus_segments=(24, 8),
                                  cube_cells=(3, 5), extent=4.0)


def moved(insts, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    out = []
    for k, inst in enumerate(insts):
        M = np.asarray(inst.local_to_world, np.float64).copy()
        M[:3, 3] += rng.uniform(-1.5, 1.5, 3) * scale
        if k % 3 == 0:  # and re-orient some
            c, s = np.cos(0.7 * k), np.sin(0.7 * k)
            M[:3, :3] = M[:3, :3] @ np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]])
        out.append(Instance(inst.mesh, M.astype(np.float32), (inst.material + k) % 7))
    return out


def rays_at(n, seed, extent=4.0):
    u = scenes.uniform(seed, 40, 5 * n).reshape(n, 5)
    z = 2 * u[:, 0] - 1
    ph = 2 * np.pi * u[:, 1]
    r = np.sqrt(1 - z * z)
    o = 2.5 * extent * np.stack([r * np.cos(ph), r * np.sin(ph), z], 1)
    tgt = (np.stack([u[:, 2], u[:, 3], u[:, 4]], 1) * 2 - 1) * extent
    d = tgt - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 4:7] = d
    rays[:, 7] = np.inf
    return rays


@pytest.mark.parametrize("rebuild", [False, True])
def test_update_equals_a_fresh_scene(cuda, rebuild):
    sc, cam = small_cloud()
    n_mat = len(sc.materials)
    new = moved(sc.instances, 3)
    new = [Instance(i.mesh, i.local_to_world, i.material % n_mat) for i in new]
    rays = rays_at(1 << 16, 9)
    e = Engine(max_bounces=4)
    e.set_scene(sc)
    e.render_frame(cam, 32, 24, samples=2)
    for step in range(2):                 # two updates in a row
        e.update_instances(new, rebuild=rebuild)
        h, ii = e.trace_rays(rays)
        e.render_frame(cam, 32, 24, samples=8, frame_seed=5)
        img = e.capture_frame().copy()
        f = Engine(max_bounces=4)
        f.set_scene(dataclasses.replace(sc, instances=new))
        hf, iif = f.trace_rays(rays)
        f.render_frame(cam, 32, 24, samples=8, frame_seed=5)
        imgf = f.capture_frame().copy()
        f.dispose()
        assert (hf["prim"] >= 0).mean() > 0.2
        same = (h["prim"] == hf["prim"]) & (ii == iif)
        assert same.mean() > 0.9999, same.mean()
        assert np.allclose(h["t"][same], hf["t"][same], rtol=1e-6)
        assert np.isclose(img, imgf, rtol=1e-4, atol=1e-6).mean() > 0.999
        new = moved(new, 11 + step, scale=0.5)
        new = [Instance(i.mesh, i.local_to_world, i.material % n_mat) for i in new]
    e.dispose()


def test_update_validation(cuda):
    sc, cam = small_cloud()
    e = Engine(max_bounces=2)
    e.set_scene(sc)
    with pytest.raises(N.VtError):
        e.update_instances(sc.instances[:-1])                       # membership is fixed
    bad = list(sc.instances)
    bad[0] = Instance(bad[0].mesh, np.zeros((4, 4), np.float32), 0)  # not invertible
    with pytest.raises(N.VtError):
        e.update_instances(bad)
    bad[0] = Instance(99, np.eye(4, dtype=np.float32), 0)            # no such mesh
    with pytest.raises(N.VtError):
        e.update_instances(bad)
    e.dispose()
    room, _ = scenes.box_room(wall_cells=4, box_cells=2)
    e = Engine(max_bounces=2)
    e.set_scene(room)
    with pytest.raises(N.VtError):
        e.update_instances([])                                      # no instances in this scene
    e.dispose()
