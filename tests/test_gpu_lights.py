"""Light families of the reference integrator beyond area meshes and points
(pt-webgpu/src/wgsl/pathTrace/kernel.wgsl.ts:1203-1675): directional (delta
and disc, with MIS for escaped BSDF rays) and rectangle lights, against
known answers and the CPU oracle."""
import math

import numpy as np
import pytest

import oracle
from vitrum_b200 import scenes
from vitrum_b200.engine import Camera, DirectionalLight, Engine, Material, Mesh, RectLight, Scene

pytestmark = pytest.mark.gpu


def plane_scene(**lights):
    p, t = scenes.grid_quad((-5, 0, -5), (0, 0, 10), (10, 0, 0), 4)   # normal +y
    # a pure Lambertian (specular factor 0; roughness 0 keeps the multiple-scattering
    # lobe that the F0 = 0 layer still carries below 1e-4 of the diffuse term)
    mat = Material(base_color=(0.8, 0.8, 0.8), specular_intensity=0.0, roughness=0.0)
    return Scene(meshes=[Mesh(p, t, 0)], materials=[mat], **lights)


CAM = Camera(eye=(0.0, 3.0, 0.01), target=(0.0, 0.0, 0.0), fov_y_deg=50.0, near=0.01, far=100.0)


def test_delta_directional_on_lambert_plane(cuda):
    # L = rho / pi * E * cos(theta) everywhere on the plane
    E, th = 3.0, math.radians(30)
    d = (math.sin(th), -math.cos(th), 0.0)
    e = Engine(max_bounces=1)
    e.set_scene(plane_scene(directional_lights=[DirectionalLight(d, (E, E, E))]))
    e.render_frame(CAM, 16, 16, samples=4)
    img = e.capture_frame()[..., :3]
    want = 0.8 / math.pi * E * math.cos(th)
    assert np.abs(img / want - 1).max() < 1e-4
    e.dispose()


def test_disc_sun_converges_to_delta(cuda):
    E, th = 3.0, math.radians(30)
    d = (math.sin(th), -math.cos(th), 0.0)
    e = Engine(max_bounces=1)
    e.set_scene(plane_scene(directional_lights=[DirectionalLight(d, (E, E, E), angular_radius=0.02)]))
    e.render_frame(CAM, 16, 16, samples=256)
    img = e.capture_frame()[..., :3]
    want = 0.8 / math.pi * E * math.cos(th)
    assert abs(img.mean() / want - 1) < 5e-3
    e.dispose()


@pytest.mark.parametrize("kind", ["disc", "rect", "both"])
def test_lights_match_cpu_oracle(cuda, kind):
    sc, cam = scenes.box_room(wall_cells=8, box_cells=4)
    sc.meshes = sc.meshes[:-1]            # drop the ceiling emitter
    if kind in ("disc", "both"):
        sc.meshes = [m for i, m in enumerate(sc.meshes) if i != 1]   # open ceiling: the sun shines in
        sc.directional_lights = [DirectionalLight((0.2, -1.0, -0.3), (4.0, 3.8, 3.5), angular_radius=0.05)]
    if kind in ("rect", "both"):
        sc.rect_lights = [RectLight((0.3, 0.95, 0.3), (0.4, 0.0, 0.0), (0.0, 0.0, 0.4), (8.0, 8.0, 8.0))]
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
    identical = np.isclose(gm, cm, rtol=1e-4, atol=1e-7).mean()
    print(f"{kind}: {identical:.3f} identical, max z {z.max():.2f}, mean {gm.mean():.4f} vs {cm.mean():.4f}")
    assert gm.mean() > 0
    assert (z > 4).sum() <= 3
    assert abs(gm.mean() / cm.mean() - 1) < 1e-2
    e.dispose()


def test_rect_light_is_invisible_from_behind_and_to_shadows(cuda):
    # a rect light facing down: seen from below it emits, from above it is transparent
    r = RectLight((-1, 1, -1), (2, 0, 0), (0, 0, 2), (5.0, 5.0, 5.0))  # edge_u x edge_v = (2,0,0)x(0,0,2) -> -y
    sc = plane_scene(rect_lights=[r])
    e = Engine(max_bounces=1)
    e.set_scene(sc)
    up = np.zeros((1, 8), np.float32)
    up[0, :3] = (0.0, 0.5, 0.0)
    up[0, 4:7] = (0.0, 1.0, 0.0)
    up[0, 7] = np.inf
    h, _ = e.trace_rays(up)
    assert h["prim"][0] >= 0 and abs(h["t"][0] - 0.5) < 1e-6     # front face visible from below
    down = up.copy()
    down[0, :3] = (0.0, 2.0, 0.0)
    down[0, 4:7] = (0.0, -1.0, 0.0)
    h, _ = e.trace_rays(down)
    assert abs(h["t"][0] - 2.0) < 1e-6                              # passes through to the plane
    e.dispose()
