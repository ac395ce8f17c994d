"""Light families of the reference integrator beyond area meshes and points
(pt-webgpu/src/wgsl/pathTrace/kernel.wgsl.ts:1203-1675): directional (delta
and disc, with MIS for escaped BSDF rays), spot lights (cone with penumbra,
decay and range), and analytic rectangle and disc lights (area sampling plus
analytic hits of BSDF rays, never occluders), against known answers and the
CPU oracle."""
import dataclasses
import math

import numpy as np
import pytest

import oracle
from vitrum_b200 import scenes
from vitrum_b200.engine import (Camera, DirectionalLight, DiscLight, Engine, Material, Mesh, RectLight, Scene,
                                SpotLight)

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


@pytest.mark.parametrize("kind", ["disc", "rect", "both", "spot", "disc_area"])
def test_lights_match_cpu_oracle(cuda, kind):
    sc, cam = scenes.box_room(wall_cells=8, box_cells=4)
    sc.meshes = sc.meshes[:-1]            # drop the ceiling emitter
    if kind in ("disc", "both"):
        sc.meshes = [m for i, m in enumerate(sc.meshes) if i != 1]   # open ceiling: the sun shines in
        sc.directional_lights = [DirectionalLight((0.2, -1.0, -0.3), (4.0, 3.8, 3.5), angular_radius=0.05)]
    if kind in ("rect", "both"):
        sc.rect_lights = [RectLight((0.3, 0.95, 0.3), (0.4, 0.0, 0.0), (0.0, 0.0, 0.4), (8.0, 8.0, 8.0))]
    if kind == "spot":
        sc.spot_lights = [SpotLight((0.5, 0.9, 0.5), (0.1, -1.0, 0.05), (3.0, 2.8, 2.5), angle=0.6, penumbra=0.4),
                          SpotLight((0.2, 0.5, 0.8), (1.0, -0.3, -0.5), (1.0, 1.0, 1.2), angle=0.3, distance=1.5,
                                    decay=1.0)]
    if kind == "disc_area":
        sc.disc_lights = [DiscLight((0.5, 0.97, 0.5), (0.0, -1.0, 0.0), 0.15, (9.0, 8.5, 8.0)),
                          DiscLight((0.05, 0.5, 0.5), (1.0, 0.2, 0.0), 0.1, (2.0, 2.0, 3.0))]
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


def _plane_points(cam, W, H, n=8):
    """Per pixel, n x n sub-sample points where the camera rays meet the y = 0 plane."""
    ivp = oracle.inverse_view_proj(cam, W, H).astype(np.float64)
    sub = (np.arange(n) + 0.5) / n
    jx, jy = np.meshgrid(sub, sub)
    out = np.zeros((H, W, n * n, 3))
    for y in range(H):
        for x in range(W):
            ndc = np.stack([(x + jx) / W * 2 - 1, 1 - (y + jy) / H * 2], -1).reshape(-1, 2)
            near = np.c_[ndc, -np.ones(len(ndc)), np.ones(len(ndc))] @ ivp.T
            far = np.c_[ndc, np.ones(len(ndc)), np.ones(len(ndc))] @ ivp.T
            o = near[:, :3] / near[:, 3:]
            d = far[:, :3] / far[:, 3:] - o
            out[y, x] = o + d * (-o[:, 1] / d[:, 1])[:, None]
    return out


@pytest.mark.parametrize("penumbra,distance,decay", [(0.0, 0.0, 2.0), (0.5, 0.0, 2.0), (0.3, 2.5, 0.0),
                                                     (0.0, 0.0, 1.0)])
def test_spot_light_on_lambert_plane(cuda, penumbra, distance, decay):
    # L = rho/pi * I * smoothstep(cos outer, cos inner, cos theta) * falloff(d) * cos(incidence)
    rho, I, h, angle = 0.8, 4.0, 1.0, 0.5
    sc = plane_scene(spot_lights=[SpotLight((0.0, h, 0.0), (0.0, -1.0, 0.0), (I, I, I), angle=angle,
                                            penumbra=penumbra, distance=distance, decay=decay)])
    cam = Camera(eye=(0.0, 3.0, 0.01), target=(0.0, 0.0, 0.0), fov_y_deg=50.0, near=0.01, far=100.0)
    W = H = 16
    e = Engine(max_bounces=1)
    e.set_scene(sc)
    e.render_frame(cam, W, H, samples=4096)
    img = e.capture_frame()[..., 0].astype(np.float64)
    e.dispose()
    P = _plane_points(cam, W, H)
    d = np.sqrt(P[..., 0] ** 2 + P[..., 2] ** 2 + h * h)
    c = h / d                                            # cone cosine and incidence cosine
    co, ci = math.cos(angle), math.cos(angle * (1 - penumbra))
    t = np.clip((c - co) / max(ci - co, 1e-6), 0, 1)
    cone = np.where(c >= co, t * t * (3 - 2 * t), 0.0)
    fall = d ** -decay if decay > 0 else np.ones_like(d)
    if distance > 0:
        fall = fall * np.clip(1 - (d / distance) ** 4, 0, 1) * (d <= distance)
    want = (rho / math.pi * I * cone * fall * c).mean(axis=-1)
    # pixels that the cone edge crosses average a step over jittered samples;
    # compare the others (the penumbra's steep ramp leaves ~0.5 % sampling noise)
    inside = c >= co
    mixed = inside.any(axis=-1) & ~inside.all(axis=-1)
    err = np.abs(img - want)[~mixed] / want.max()
    assert img.max() > 0 and mixed.sum() < img.size // 2 and err.max() < 1.5e-2, err.max()


@pytest.mark.parametrize("bounces", [1, 2])
def test_disc_light_on_axis_known_answer(cuda, bounces):
    # irradiance under the centre of a disc of radius r at height h: E = pi L r^2 / (h^2 + r^2);
    # the camera looks down through the disc's back (not an occluder, not visible from behind)
    rho, Le, r, h = 0.8, 5.0, 0.5, 1.0
    sc = plane_scene(disc_lights=[DiscLight((0.0, h, 0.0), (0.0, -1.0, 0.0), r, (Le, Le, Le))])
    cam = Camera(eye=(0.0, 10.0, 0.001), target=(0.0, 0.0, 0.0), fov_y_deg=0.2, near=0.01, far=100.0)
    e = Engine(max_bounces=bounces)
    e.set_scene(sc)
    e.render_frame(cam, 8, 8, samples=4096)
    got = float(e.capture_frame()[..., 0].mean())
    e.dispose()
    want = rho / math.pi * math.pi * Le * r * r / (h * h + r * r)
    assert abs(got / want - 1) < 1e-2, (got, want)


def test_analytic_area_lights_are_seen_only_from_the_front(cuda):
    # a rect light facing down: a camera below sees its radiance; one above sees
    # the lit plane through it; traced rays never hit it
    r = RectLight((-1, 1, -1), (2, 0, 0), (0, 0, 2), (5.0, 5.0, 5.0))  # edge_u x edge_v = (2,0,0)x(0,0,2) -> -y
    sc = plane_scene(rect_lights=[r])
    e = Engine(max_bounces=1)
    e.set_scene(sc)
    up = np.zeros((1, 8), np.float32)
    up[0, :3] = (0.0, 0.5, 0.0)
    up[0, 4:7] = (0.0, 1.0, 0.0)
    up[0, 7] = np.inf
    h, _ = e.trace_rays(up)
    assert h["prim"][0] == -1                                       # not geometry
    below = Camera(eye=(0.0, 0.5, 0.0), target=(0.0, 2.0, 0.001), fov_y_deg=20.0, near=0.01, far=100.0)
    e.render_frame(below, 8, 8, samples=4)
    assert np.allclose(e.capture_frame()[..., :3], 5.0)            # front face: its radiance
    above = Camera(eye=(0.0, 3.0, 0.001), target=(0.0, 0.0, 0.0), fov_y_deg=2.0, near=0.01, far=100.0)
    e.reset()
    e.render_frame(above, 8, 8, samples=2048)
    img = e.capture_frame()[..., 0]
    # the plane below the light's centre: E = L * solid-angle-projected area of the square
    a = 1.0 / math.sqrt(2.0)
    want = 0.8 / math.pi * 5.0 * 4 * (a * math.atan(a) * 2 / 2)      # 4 quadrants, unit offsets at height 1
    assert abs(img.mean() / want - 1) < 0.02, (img.mean(), want)
    e.dispose()


def test_spot_and_disc_validation(cuda):
    bad = [dict(spot_lights=[SpotLight((0, 1, 0), (0, 0, 0), (1, 1, 1), angle=0.5)]),
           dict(spot_lights=[SpotLight((0, 1, 0), (0, -1, 0), (1, 1, 1), angle=0.0)]),
           dict(spot_lights=[SpotLight((0, 1, 0), (0, -1, 0), (1, 1, 1), angle=0.5, penumbra=1.5)]),
           dict(spot_lights=[SpotLight((0, 1, 0), (0, -1, 0), (1, 1, 1), angle=0.5, decay=-1.0)]),
           dict(disc_lights=[DiscLight((0, 1, 0), (0, -1, 0), 0.0, (1, 1, 1))]),
           dict(disc_lights=[DiscLight((0, 1, 0), (0, 0, 0), 0.5, (1, 1, 1))])]
    for kw in bad:
        e = Engine(max_bounces=1)
        with pytest.raises(Exception):
            e.set_scene(plane_scene(**kw))
        e.dispose()


def test_procedural_sky_matches_cpu_oracle(cuda):
    # Preetham daylight baked into the environment (vt_bake_preetham_sky), importance
    # sampled with its sun disc: device vs CPU oracle over a box room without a ceiling
    sc, cam = scenes.box_room(wall_cells=8, box_cells=4)
    sc.meshes = [m for i, m in enumerate(sc.meshes[:-1]) if i != 1]
    sc.environment = scenes.preetham_sky((0.3, 0.8, -0.4), turbidity=3.0, intensity=0.05)
    W = H = 20
    n, B = 256, 3
    e = Engine(max_bounces=B, oracle_accumulation=True)
    e.set_scene(sc)
    e.render_frame(cam, W, H, samples=n)
    gm, gv = e.capture_moments()
    e.dispose()
    s, q = oracle.pt_render(sc, cam, W, H, n, B)
    cm = s / n
    cv = np.maximum(q / n - cm * cm, 0) * n / (n - 1)
    z = np.abs(gm - cm) / (np.sqrt((gv + cv) / n) + 1e-9)
    assert gm.mean() > 0 and (z > 4).sum() <= 3
    assert abs(gm.mean() / cm.mean() - 1) < 1e-2


def test_environment_rotation_equals_shifted_map(cuda):
    # rotationY = 2 pi k / W looks the map up k columns further (rotateYNeg,
    # connectCore.wgsl.ts:27-30): the same image as the map with its columns shifted
    from vitrum_b200.engine import Environment
    sc, cam = scenes.box_room(wall_cells=8, box_cells=4)
    sc.meshes = [m for i, m in enumerate(sc.meshes[:-1]) if i != 1]   # no ceiling, no emitter
    rng = np.random.default_rng(4)
    env = (rng.uniform(0.0, 1.0, (8, 16, 3)) ** 4 * 6).astype(np.float32)
    k = 3
    rot = dataclasses.replace(sc, environment=Environment(env, rotation_y=2 * math.pi * k / 16))
    shift = dataclasses.replace(sc, environment=Environment(np.roll(env, -k, axis=1)))
    out = []
    for s in (rot, shift):
        e = Engine(max_bounces=3, oracle_accumulation=True)
        e.set_scene(s)
        e.render_frame(cam, 20, 20, samples=2048)
        out.append(e.capture_moments())
        e.dispose()
    (ma, va), (mb, vb) = out
    z = np.abs(ma - mb) / (np.sqrt((va + vb) / 2048) + 1e-9)
    assert ma.mean() > 0 and (z > 4).sum() <= 3 and abs(ma.mean() / mb.mean() - 1) < 1.5e-2
    s, _ = oracle.pt_render(rot, cam, 20, 20, 512, 3)
    assert abs((s / 512).mean() / ma.mean() - 1) < 4e-2
