"""Multi-light NEE + MIS consistency (the reference's multiLightMis.test.ts
known answers, pt-webgpu/src/__tests__/multiLightMis.test.ts:190-263): with
one light entry chosen per vertex and both strategies MIS-weighted, the image
lit by two lights equals the sum of the images lit by each alone (within the
Monte Carlo error), and scaling every light's power scales the image.
Exercised with an emissive mesh, an analytic rectangle, an analytic disc, a
spot and a directional sun in a box room."""
import dataclasses

import numpy as np
import pytest

from vitrum_b200 import scenes
from vitrum_b200.engine import DirectionalLight, DiscLight, Engine, Material, RectLight, SpotLight

pytestmark = pytest.mark.gpu

W = H = 24


def room():
    # the glass box made diffuse: caustics (light reached only through a delta
    # interface) make single samples heavy-tailed, which these mean tests avoid
    sc, cam = scenes.box_room(wall_cells=8, box_cells=4)
    mats = list(sc.materials)
    mats[4] = Material(base_color=(0.7, 0.7, 0.7), specular_intensity=0.0)
    return dataclasses.replace(sc, materials=mats), cam


def lights(kind, scale=1.0):
    s = scale
    return {
        "rect": dict(rect_lights=[RectLight((0.3, 0.95, 0.3), (0.4, 0.0, 0.0), (0.0, 0.0, 0.4), (6 * s,) * 3)]),
        # (no direction from the room meets both analytic lights: BSDF rays count
        # only the nearest analytic light they cross, as the reference does)
        "disc": dict(disc_lights=[DiscLight((0.5, 0.95, 0.85), (0.1, -1.0, -0.1), 0.1, (10 * s, 9 * s, 8 * s))]),
        "spot": dict(spot_lights=[SpotLight((0.5, 0.9, 0.6), (0.0, -1.0, -0.2), (2 * s,) * 3, angle=0.7,
                                            penumbra=0.3)]),
    }[kind]


def render(sc, cam, spp=4096, seed=3):
    """FP64 mean and variance of `spp` samples.  The frame seed is shifted past
    the sample indices, so different seeds draw disjoint key sets (the key is
    seed ^ sample index)."""
    e = Engine(max_bounces=4, oracle_accumulation=True, max_samples_per_pixel=1 << 16)
    e.set_scene(sc)
    e.render_frame(cam, W, H, samples=spp, frame_seed=seed << 20)
    m, v = e.capture_moments()
    e.dispose()
    return m, v


def with_lights(sc, *kinds, scale=1.0, keep_mesh_light=False):
    kw = dict(rect_lights=[], disc_lights=[], spot_lights=[])
    for k in kinds:
        kw.update({a: kw[a] + b for a, b in lights(k, scale).items()})
    out = dataclasses.replace(sc, **kw)
    if not keep_mesh_light:
        out = dataclasses.replace(out, meshes=sc.meshes[:-1])  # drop the ceiling emitter
    return out


@pytest.mark.parametrize("a,b", [("rect", "disc"), ("disc", "spot"), ("rect", "spot")])
def test_two_lights_sum(cuda, a, b):
    """Eight renders of each image.  Light reaching the camera through the
    metal surfaces makes the image mean heavy-tailed (one 4096-sample render
    of disc + spot lands anywhere within about 5 % of the sum), so the
    difference of the image means is judged against its standard error over
    the renders, which then resolves a bias of about 3 % of the sum."""
    sc, cam = room()
    scenes_ = [with_lights(sc, a), with_lights(sc, b), with_lights(sc, a, b)]
    reps, n = 8, 16384
    means = np.zeros((reps, 3))
    for i in range(reps):
        out = [render(s, cam, spp=n, seed=3 * i + k + 3) for k, s in enumerate(scenes_)]
        means[i] = [m.mean() for m, _ in out]
        if i == 0:
            (ma, va), (mb, vb), (mab, vab) = out
            z = (mab - ma - mb) / (np.sqrt((va + vb + vab) / n) + 1e-9)
    d = means[:, 2] - means[:, 0] - means[:, 1]
    tot = (means[:, 0] + means[:, 1]).mean()
    se = d.std(ddof=1) / np.sqrt(reps)
    print(f"{a}+{b}: difference {d.mean() / tot:+.4f} +- {se / tot:.4f} of the sum; first render |z|>4: "
          f"{(np.abs(z) > 4).sum()}")
    assert abs(d.mean()) < 4 * se + 1e-3 * tot and se < 0.0075 * tot
    assert (z < -4).sum() <= 3


def test_mesh_emitter_and_analytic_light_sum(cuda):
    sc, cam = room()
    mesh_only, v1 = render(with_lights(sc, keep_mesh_light=True), cam, seed=6)
    rect_only, v2 = render(with_lights(sc, "rect"), cam, seed=7)
    both, v3 = render(with_lights(sc, "rect", keep_mesh_light=True), cam, seed=8)
    assert abs(both.mean() / (mesh_only.mean() + rect_only.mean()) - 1) < 0.025


def test_power_scales_the_image(cuda):
    # one light entry per vertex is chosen uniformly, so the same random numbers
    # trace the same paths: doubling every emitter doubles every pixel
    sc, cam = room()
    m1, _ = render(with_lights(sc, "rect", "disc", "spot"), cam, spp=64, seed=9)
    m2, _ = render(with_lights(sc, "rect", "disc", "spot", scale=2.0), cam, spp=64, seed=9)
    assert m1.mean() > 0
    assert np.allclose(m2, 2.0 * m1, rtol=1e-5, atol=1e-7)


def test_directional_and_area_light_sum(cuda):
    sc, cam = room()
    open_top = dataclasses.replace(sc, meshes=[m for i, m in enumerate(sc.meshes[:-1]) if i != 1])
    sun = [DirectionalLight((0.2, -1.0, -0.3), (4.0, 3.8, 3.5), angular_radius=0.05)]
    ms, vs = render(dataclasses.replace(open_top, directional_lights=sun), cam, seed=10)
    md, vd = render(dataclasses.replace(open_top, disc_lights=lights("disc")["disc_lights"]), cam, seed=11)
    mb, vb = render(dataclasses.replace(open_top, directional_lights=sun,
                                        disc_lights=lights("disc")["disc_lights"]), cam, seed=12)
    assert abs(mb.mean() / (ms.mean() + md.mean()) - 1) < 0.025
