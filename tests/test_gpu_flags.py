"""Material flags of the reference's traceClosest / traceAny
(pt-webgpu/src/wgsl/pathTrace/intersection.wgsl.ts:462-528): back faces of
single-sided surfaces are skipped by every ray, castShadow: false geometry by
shadow rays; both are decided inside traversal (no retrace)."""
import math

import numpy as np
import pytest

import oracle
from vitrum_b200 import scenes
from vitrum_b200.engine import Camera, Engine, Material, Mesh, PointLight, Scene

pytestmark = pytest.mark.gpu


def rays_along_z(z0, dz, n=64):
    g = (np.arange(n) + 0.5) / n - 0.5
    r = np.zeros((n, 8), np.float32)
    r[:, 0] = g * 0.8
    r[:, 1] = g[::-1] * 0.8
    r[:, 2] = z0
    r[:, 3] = 0.0
    r[:, 6] = dz
    r[:, 7] = np.inf
    return r


def test_single_sided_back_faces_are_skipped(cuda):
    front, ft = scenes.grid_quad((-1, -1, 0), (2, 0, 0), (0, 2, 0), 2)      # normal +z, single-sided
    back, bt = scenes.grid_quad((-1, -1, -1), (2, 0, 0), (0, 2, 0), 2)      # z = -1, double-sided
    sc = Scene(meshes=[Mesh(front, ft, 0), Mesh(back, bt, 1)],
               materials=[Material(double_sided=False), Material()])
    e = Engine()
    e.set_scene(sc)
    h, _ = e.trace_rays(rays_along_z(2.0, -1.0))       # towards -z: front face of the quad
    assert (h["prim"] < 8).all() and np.allclose(h["t"], 2.0)
    h, _ = e.trace_rays(rays_along_z(-0.5, 1.0))       # towards +z from behind: passes through
    assert (h["prim"] < 0).all()
    h, _ = e.trace_rays(rays_along_z(-0.5, -1.0))      # towards -z from between: the back wall
    assert (h["prim"] >= 8).all() and np.allclose(h["t"], 0.5)
    e.dispose()


@pytest.mark.parametrize("cast", [True, False])
def test_cast_shadow_false_is_ignored_by_shadow_rays(cuda, cast):
    rho, I, h = 0.8, 4.0, 1.0
    floor, tf = scenes.grid_quad((-5, 0, -5), (0, 0, 10), (10, 0, 0), 4)
    occ, to = scenes.grid_quad((-4.9, 0.5, -4.9), (0, 0, 9.8), (9.8, 0, 0), 1)  # covers the floor below the light
    sc = Scene(meshes=[Mesh(floor, tf, 0), Mesh(occ, to, 1)],
               materials=[Material(base_color=(rho,) * 3, specular_intensity=0.0),
                          Material(base_color=(0.0,) * 3, cast_shadow=cast, specular_intensity=0.0)],
               point_lights=[PointLight((0.0, h, 0.0), (I, I, I))])
    # camera between the floor and the occluder, looking at the floor under the occluder
    cam = Camera(eye=(0.0, 0.25, 3.0), target=(0.0, 0.0, 0.0), fov_y_deg=30.0, near=0.01, far=100.0)
    e = Engine(max_bounces=1)
    e.set_scene(sc)
    e.render_frame(cam, 24, 24, samples=64)
    img = e.capture_frame()[..., 0]
    lit = img[16:, :].mean()
    if cast:
        assert lit < 1e-3, lit
    else:
        assert lit > 0.05, lit
    e.dispose()


def test_flags_match_cpu_oracle(cuda):
    # box room whose walls are single-sided (seen from inside: front faces) and
    # whose tall box does not cast shadows
    sc, cam = scenes.box_room(wall_cells=8, box_cells=4)
    for k in range(3):
        sc.materials[k].double_sided = False
    sc.materials[3].cast_shadow = False
    W = H = 20
    n, B = 256, 4
    e = Engine(max_bounces=B, oracle_accumulation=True)
    e.set_scene(sc)
    e.render_frame(cam, W, H, samples=n)
    gm, gv = e.capture_moments()
    s, q = oracle.pt_render(sc, cam, W, H, n, B)
    cm = s / n
    cv = np.maximum(q / n - cm * cm, 0) * n / (n - 1)
    z = np.abs(gm - cm) / (np.sqrt((gv + cv) / n) + 1e-9)
    assert (z > 4).sum() <= 3
    assert abs(gm.mean() / cm.mean() - 1) < 1e-2
    e.dispose()
