"""Unbiasedness at the workloads' own sizes: the box room at 512x512 (5
bounces) and the 1024-instance cloud at 480x270 (8 bounces), rendered at 64
spp (and 4096 spp) and compared with a 65,536-spp FP64-accumulated render of the
same scene (disjoint RNG keys), pixel by pixel on luminance and per 16 x 16
tile.

The z-score of a pixel is standardised by the oracle's per-sample variance,
z = (m - m_ref) / sqrt(v_ref (1/n + 1/65536)): a render's own variance is zero
wherever its n samples happen to agree (a pixel that rarely sees an object past
the sky), which would turn any difference into an arbitrary z.

A path-traced pixel's samples are skewed and heavy-tailed (rare bright paths),
so at 64 spp its mean is not Gaussian at 4 sigma, and the expected number of
pixels beyond each side is computed from the oracle's per-pixel skewness and
excess kurtosis (vt_capture_luminance_moments):
- where g1 = skewness / sqrt(n) <= 0.5 and g2 = kurtosis / n <= 1, by the
  second-order Edgeworth expansion of the standardised mean, P(Z > x) = Q(x) +
  phi(x) [g1 He2(x) / 6 + g2 He3(x) / 24 + g1^2 He5(x) / 72];
- elsewhere (heavy tails) by the two-point model with that kurtosis (the
  sample is 0 or one rare large value of probability p, kurtosis ~ 1/p): the
  count of rare values among n is binomial, so Z > 4 needs a few more of them
  than n p, and Z < -4 is all but impossible.
Each count is held within a binomial bound of its expectation (expected +
4 sqrt(expected) + 4); the lower side is summed over both kinds of pixel.

- Scenes: the workloads (near-mirror metal, smooth glass: paths that reach
  a light only through them are found by BSDF sampling alone, and most
  pixels' excess kurtosis runs to the thousands) and Lambertian variants
  (every material made Lambert with its base colour), plus the cloud lit by
  its sky alone.
- Per 16 x 16 tile at 64 spp, the tile mean's cumulants sum the pixels'.
- Per pixel at 4096 spp for the two scenes of finite per-sample variance (the
  Lambertian room and the sky-lit cloud).  The cloud's point lights give the
  next-event term I cos / d^2 an unbounded variance where a surface passes
  close to one; 65,536 oracle samples cannot resolve that tail, so at 4096
  spp its pixels exceed +4 sigma more often than the oracle's moments predict
  (152 of 24,848 measured).  Those scenes are held at 64 spp and per tile.
"""
import dataclasses
import math

import numpy as np
import pytest

from vitrum_b200 import scenes
from vitrum_b200.engine import Engine, Material

pytestmark = pytest.mark.gpu

ORACLE_SPP = 65536
# keys are seed ^ sample index: the oracle's [2^24, 2^24 + 2^16), the 64-spp
# render's [2^16, 2^16 + 64) and the 4096-spp render's [2^17, 2^17 + 4096) are disjoint
ORACLE_SEED = 1 << 24
SEEDS = {64: 1 << 16, 4096: 1 << 17}
TILE = 16

_CACHE = {}


def lambertian(sc):
    mats = [m if any(c > 0 for c in m.emission) else Material(base_color=m.base_color, specular_intensity=0.0)
            for m in sc.materials]
    return dataclasses.replace(sc, materials=mats)


SCENES = {
    "room": lambda: (*scenes.box_room(), 512, 512, 5),
    "room_lambert": lambda: (lambertian(scenes.box_room()[0]), scenes.box_room()[1], 512, 512, 5),
    "cloud": lambda: (*scenes.instanced_cloud(), 480, 270, 8),
    "cloud_lambert": lambda: (lambertian(scenes.instanced_cloud()[0]), scenes.instanced_cloud()[1], 480, 270, 8),
    "cloud_sky_lambert": lambda: (dataclasses.replace(lambertian(scenes.instanced_cloud()[0]), point_lights=[]),
                                  scenes.instanced_cloud()[1], 480, 270, 8),
}


def moments(sc, cam, W, H, B, spp, seed):
    e = Engine(max_bounces=B, oracle_accumulation=True, max_samples_per_pixel=1 << 17)
    e.set_scene(sc)
    done = 0
    while done < spp:
        k = min(4096, spp - done)
        e.render_frame(cam, W, H, samples=k, frame_seed=seed)
        done += k
    out = e.capture_luminance_moments()
    e.dispose()
    return out


def oracle(name):
    key = (name, "oracle")
    if key not in _CACHE:
        sc, cam, W, H, B = SCENES[name]()
        _CACHE[key] = moments(sc, cam, W, H, B, ORACLE_SPP, ORACLE_SEED)
    return _CACHE[key]


def render(name, spp):
    key = (name, spp)
    if key not in _CACHE:
        sc, cam, W, H, B = SCENES[name]()
        _CACHE[key] = moments(sc, cam, W, H, B, spp, SEEDS[spp])
    return _CACHE[key]


def tails(g1, g2, x=4.0):
    """Second-order Edgeworth tail probabilities (below -x, above +x) of a
    standardised statistic with skewness g1 and excess kurtosis g2."""
    q = 0.5 * math.erfc(x / math.sqrt(2.0))
    phi = math.exp(-x * x / 2) / math.sqrt(2 * math.pi)
    he2, he3, he5 = x * x - 1, x ** 3 - 3 * x, x ** 5 - 10 * x ** 3 + 15 * x
    even = g2 * he3 / 24 + g1 * g1 * he5 / 72
    return (np.clip(q + phi * (-g1 * he2 / 6 + even), 0, 1), np.clip(q + phi * (g1 * he2 / 6 + even), 0, 1))


def bound(e):
    return e + 4.0 * math.sqrt(e) + 4.0


def two_point_tails(kurt, n, x=4.0):
    """Tail probabilities (below -x, above +x) of the standardised mean of n
    samples drawn from a two-point distribution with excess kurtosis `kurt`."""
    from scipy.stats import binom
    q = 1.0 / (np.maximum(kurt, 0.0) + 6.0)  # p (1 - p) from (1 - 6 p (1 - p)) / (p (1 - p)) = kurt
    p = np.clip((1 - np.sqrt(np.maximum(1 - 4 * q, 0))) / 2, 1e-12, 0.5)
    mu, sd = n * p, np.sqrt(n * p * (1 - p))
    return binom.cdf(np.ceil(mu - x * sd) - 1, n, p), binom.sf(np.floor(mu + x * sd), n, p)


def pixel_stats(name, spp):
    ref, got = oracle(name), render(name, spp)
    om, ov, skew, kurt = (ref[..., k] for k in range(4))
    m = got[..., 0]
    live = ov > 0
    # deterministic pixels (every oracle sample equal: sky seen directly, black) agree exactly
    assert np.allclose(m[~live], om[~live], rtol=1e-6, atol=1e-9)
    z = (m - om)[live] / np.sqrt(ov[live] * (1.0 / spp + 1.0 / ORACLE_SPP))
    g1, g2 = skew[live] / math.sqrt(spp), kurt[live] / spp
    valid = (np.abs(g1) <= 0.5) & (g2 <= 1.0)
    p_lo, p_hi = tails(g1[valid], g2[valid])
    h_lo, h_hi = two_point_tails(kurt[live][~valid], spp)
    out = dict(n=int(z.size), n_valid=int(valid.sum()),
               lo=int((z < -4).sum()), e_lo=float(p_lo.sum() + h_lo.sum()),
               hi=int((z[valid] > 4).sum()), e_hi=float(p_hi.sum()),
               hi_heavy=int((z[~valid] > 4).sum()), e_hi_heavy=float(h_hi.sum()),
               ratio=float(m.mean() / om.mean()))
    print(f"{name} {spp} spp, per pixel: {out['n']} pixels; below -4 sigma {out['lo']} (expected "
          f"{out['e_lo']:.1f}); above +4 sigma {out['hi']} of {out['n_valid']} Edgeworth pixels (expected "
          f"{out['e_hi']:.1f}) and {out['hi_heavy']} of {out['n'] - out['n_valid']} heavy-tailed ones (two-point "
          f"model {out['e_hi_heavy']:.1f}); image mean ratio {out['ratio']:.5f}; excess kurtosis median "
          f"{np.median(kurt[live]):.1f}")
    return out


def tile_stats(name, spp):
    ref, got = oracle(name), render(name, spp)
    H, W = ref.shape[:2]
    h, w = H // TILE * TILE, W // TILE * TILE

    def tiles(a):
        return a[:h, :w].reshape(h // TILE, TILE, w // TILE, TILE).sum(axis=(1, 3))
    om, ov, skew, kurt = (ref[..., k] for k in range(4))
    P = TILE * TILE
    dm = tiles(got[..., 0] - om) / P
    var = tiles(ov) * (1.0 / spp + 1.0 / ORACLE_SPP) / P ** 2
    k3 = tiles(skew * ov ** 1.5) / spp ** 2 / P ** 3   # third cumulant of the tile mean
    k4 = tiles(kurt * ov ** 2) / spp ** 3 / P ** 4     # fourth cumulant
    live = var > 0
    z = dm[live] / np.sqrt(var[live])
    g1, g2 = k3[live] / var[live] ** 1.5, k4[live] / var[live] ** 2
    valid = (np.abs(g1) <= 0.5) & (g2 <= 1.0)
    p_lo, p_hi = tails(g1[valid], g2[valid])
    out = dict(n=int(z.size), lo=int((z < -4).sum()), e_lo=float(p_lo.sum()), hi=int((z[valid] > 4).sum()),
               e_hi=float(p_hi.sum()), hi_heavy=int((z[~valid] > 4).sum()), n_heavy=int((~valid).sum()))
    print(f"{name} {spp} spp, {TILE}x{TILE} tiles: {out['n']} tiles; below -4 sigma {out['lo']} (expected "
          f"{out['e_lo']:.2f}); above +4 sigma {out['hi']} (expected {out['e_hi']:.2f}) and {out['hi_heavy']} of "
          f"{out['n_heavy']} skewed tiles; |z| max {np.abs(z).max():.2f}")
    return out


@pytest.mark.parametrize("name", ["room_lambert", "cloud_sky_lambert", "cloud_lambert", "room", "cloud"])
def test_tile_means_within_4_sigma(cuda, name):
    t = tile_stats(name, 64)
    assert t["lo"] <= bound(t["e_lo"]) and t["hi"] <= bound(t["e_hi"])
    assert t["hi_heavy"] <= max(4, 0.01 * t["n_heavy"])


@pytest.mark.parametrize("name,spp", [("room_lambert", 64), ("cloud_sky_lambert", 64), ("cloud_lambert", 64),
                                      ("room", 64), ("cloud", 64), ("room_lambert", 4096),
                                      ("cloud_sky_lambert", 4096)])
def test_pixel_means_within_4_sigma(cuda, name, spp):
    s = pixel_stats(name, spp)
    assert s["lo"] <= bound(s["e_lo"])
    assert s["hi"] <= bound(s["e_hi"]) and s["hi_heavy"] <= bound(s["e_hi_heavy"])
    assert abs(s["ratio"] - 1) < (2e-3 if name.endswith("lambert") else 5e-3)
