"""The procedural-sky bake (vt_bake_preetham_sky, host code) against the numpy
restatement of the reference's bake (oracle/sky.py): the sky and haze texels
to float precision, the sun disc's total power exactly and its texels to the
accuracy of the two coverage quadratures (CPU; no GPU needed)."""
import math

import numpy as np
import pytest

from oracle import sky as osky
from vitrum_b200 import scenes


@pytest.mark.parametrize("sun,T,g", [((0.3, 0.8, 0.2), 2.0, 0.8), ((-0.5, 0.2, 0.7), 6.0, 0.6),
                                      ((0.0, 1.0, 0.0), 3.0, 0.8), ((0.8, 0.05, -0.3), 10.0, 0.9)])
def test_bake_matches_oracle(sun, T, g):
    got = scenes.preetham_sky(sun, turbidity=T, mie_directional_g=g, width=128, height=64).rgb.astype(np.float64)
    want = osky.bake_preetham_sky(sun, turbidity=T, mie_directional_g=g, width=128, height=64)
    s = np.asarray(sun, np.float64) / np.linalg.norm(sun)
    th = (np.arange(64) + 0.5) / 64 * math.pi
    ph = ((np.arange(128) + 0.5) / 128 - 0.5) * 2 * math.pi
    TH, PH = np.meshgrid(th, ph, indexing="ij")
    d = np.stack([np.sin(TH) * np.cos(PH), np.cos(TH), np.sin(TH) * np.sin(PH)], -1)
    far = np.arccos(np.clip(d @ s, -1, 1)) > 0.2            # texels away from the sun disc
    assert np.allclose(got[far], want[far], rtol=2e-5, atol=1e-7)
    # the sun: same total (solid-angle weighted), texels within the quadratures' accuracy
    meas = (math.pi / 64) * (2 * math.pi / 128) * np.maximum(np.sin(TH), 1e-6)
    lum = lambda a: 0.2126 * a[..., 0] + 0.7152 * a[..., 1] + 0.0722 * a[..., 2]
    near = ~far
    assert abs((lum(got) * meas)[near].sum() / (lum(want) * meas)[near].sum() - 1) < 1e-3
    assert abs(lum(got).max() / lum(want).max() - 1) < 2e-2
    assert np.all(got >= 0) and np.all(got[np.cos(TH) < -0.05] == 0)


def test_sky_is_symmetric_about_the_sun_azimuth():
    # sun in the x-y plane: the map is mirror-symmetric in z (columns about the middle)
    env = scenes.preetham_sky((0.6, 0.5, 0.0), width=128, height=64).rgb
    assert np.allclose(env[:, 64:], env[:, 63::-1], rtol=1e-4, atol=1e-6)
