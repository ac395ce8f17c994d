"""Numpy restatement of the procedural-sky bake (TEST INFRASTRUCTURE ONLY: the
checker of vt_bake_preetham_sky).

Follows bakePreethamSkyEquirect (shared-samplers/src/preethamSky.ts:151-313):
Perez sky luminance and chromaticity relative to the zenith (preethamSky.ts:51-120),
Henyey-Greenstein haze, and the sun disc deposited by the reference's
solarDiscTexelCoverage recipe (solarDiscCoverage.ts:44-178: per row, a
theta quadrature with the disc's analytic longitude half-width at each theta,
intervals intersected with the columns, rescaled to the cap's solid angle and
divided by dtheta dphi sin(theta_centre)).  Float64 throughout."""
import math

import numpy as np

SUN_RADIUS = 0.00436


def _perez(c, gamma, k):
    c = np.maximum(c, 1e-4)
    return (1 + k[0] * np.exp(k[1] / c)) * (1 + k[2] * np.exp(k[3] * gamma) + k[4] * np.cos(gamma) ** 2)


def _coverage(width, height, s):
    th_s = math.acos(max(-1.0, min(1.0, s[1])))
    sin_s = math.hypot(s[0], s[2])
    sun_phi = (math.atan2(s[2], s[0]) + math.pi) % (2 * math.pi)
    cos_r = math.cos(SUN_RADIUS)
    dth, dph = math.pi / height, 2 * math.pi / width
    cov = np.zeros((height, width))
    tmin, tmax = max(0.0, th_s - SUN_RADIUS), min(math.pi, th_s + SUN_RADIUS)
    r0, r1 = max(0, math.floor(tmin / dth)), min(height - 1, math.ceil(tmax / dth) - 1)

    def add(row, lo, hi, w):
        for x in range(max(0, math.floor(lo / dph)), min(width - 1, math.ceil(hi / dph) - 1) + 1):
            ov = min(hi, (x + 1) * dph) - max(lo, x * dph)
            if ov > 0:
                cov[row, x] += w * ov

    def span(row, half, w):
        if half >= math.pi:
            add(row, 0.0, 2 * math.pi, w)
            return
        start = (sun_phi - half) % (2 * math.pi)
        end = start + 2 * half
        add(row, start, min(end, 2 * math.pi), w)
        if end > 2 * math.pi:
            add(row, 0.0, end - 2 * math.pi, w)

    for row in range(r0, r1 + 1):
        lo, hi = max(row * dth, tmin), min((row + 1) * dth, tmax)
        if hi <= lo:
            continue
        n = max(16, min(512, math.ceil((hi - lo) / (SUN_RADIUS / 64))))
        step = (hi - lo) / n
        for k in range(n):
            th = lo + (k + 0.5) * step
            w = math.sin(th) * step
            h = math.sin(th) * sin_s
            if h <= 2.220446049250313e-16:
                if math.cos(th) * s[1] >= cos_r:
                    span(row, math.pi, w)
                continue
            thr = (cos_r - math.cos(th) * s[1]) / h
            if thr <= -1:
                span(row, math.pi, w)
            elif thr < 1:
                span(row, math.acos(thr), w)
    total = cov.sum()
    cap = 2 * math.pi * (1 - cos_r)
    rows = np.arange(height)
    measure = dth * dph * np.maximum(np.sin((rows + 0.5) * dth), 1e-6)
    return cov * (cap / total) / measure[:, None]


def bake_preetham_sky(sun_direction=(0.0, 1.0, 0.0), turbidity=2.0, rayleigh=1.0, mie_coefficient=0.005,
                      mie_directional_g=0.8, intensity=1.0, width=256, height=128):
    s = np.asarray(sun_direction, np.float32).astype(np.float64)
    ln = math.sqrt((s * s).sum())
    s = np.array([0.0, 1.0, 0.0]) if ln < 1e-8 else s / ln
    T = max(1.5, min(30.0, float(np.float32(turbidity))))
    mie = 200 * max(0.0, float(np.float32(mie_coefficient)))
    g = max(-0.999999, min(0.999999, float(np.float32(mie_directional_g))))
    ts = math.acos(max(-1.0, min(1.0, s[1])))
    Y_z = max(1e-5, (4.0453 * T - 4.971) * math.tan((4 / 9 - T / 120) * (math.pi - 2 * ts)) - 0.2155 * T + 2.4192)
    Y_z *= max(0.0, float(np.float32(rayleigh))) * max(0.0, float(np.float32(intensity)))
    t2, t3 = ts * ts, ts ** 3
    x_z = ((0.00166 * t3 - 0.00375 * t2 + 0.00209 * ts) * T * T + (-0.02903 * t3 + 0.06377 * t2 - 0.03202 * ts
           + 0.00394) * T + (0.11693 * t3 - 0.21196 * t2 + 0.06052 * ts + 0.25886))
    y_z = ((0.00275 * t3 - 0.0061 * t2 + 0.00317 * ts) * T * T + (-0.04214 * t3 + 0.0897 * t2 - 0.04153 * ts
           + 0.00516) * T + (0.15346 * t3 - 0.26756 * t2 + 0.0667 * ts + 0.26688))
    kY = [0.17872 * T - 1.46303, -0.3554 * T + 0.42749, -0.02266 * T + 5.32505, 0.12064 * T - 2.57705,
          -0.06696 * T + 0.37027]
    kx = [-0.01925 * T - 0.25922, -0.06651 * T + 0.00081, -0.00041 * T + 0.21247, -0.06409 * T - 0.89887,
          -0.00325 * T + 0.04517]
    ky = [-0.01669 * T - 0.26078, -0.09495 * T + 0.00921, -0.00792 * T + 0.21023, -0.04405 * T - 1.65369,
          -0.01092 * T + 0.05291]
    nY, nx, ny = (_perez(1.0, ts, k) for k in (kY, kx, ky))
    th = (np.arange(height) + 0.5) / height * math.pi
    ph = ((np.arange(width) + 0.5) / width - 0.5) * 2 * math.pi
    TH, PH = np.meshgrid(th, ph, indexing="ij")
    ct = np.cos(TH)
    cg = np.clip(np.sin(TH) * np.cos(PH) * s[0] + ct * s[1] + np.sin(TH) * np.sin(PH) * s[2], -1, 1)
    gamma = np.arccos(cg)
    c = np.maximum(ct, 1e-4)
    Y = Y_z * _perez(c, gamma, kY) / nY
    x = x_z * _perez(c, gamma, kx) / nx
    y = y_z * _perez(c, gamma, ky) / ny
    fade = np.minimum(1.0, (ct + 0.05) / 0.05)
    sky = np.maximum(0.0, Y) * fade
    d = 1 + g * g - 2 * g * cg
    haze = mie * (1 - g * g) / (4 * math.pi * d * np.sqrt(d)) * 4 * math.pi * Y_z * fade
    sun = _coverage(width, height, s) * 500 * Y_z
    tot = sky + haze + sun
    use_sky = (sky > 1e-12) | (tot < 1e-12)
    cx, cy = np.where(use_sky, x, x_z), np.where(use_sky, y, y_z)
    X, Z = tot / cy * cx, tot / cy * (1 - cx - cy)
    rgb = np.stack([3.2406 * X - 1.5372 * tot - 0.4986 * Z, -0.9689 * X + 1.8758 * tot + 0.0415 * Z,
                    0.0557 * X - 0.204 * tot + 1.057 * Z], -1)
    rgb = np.maximum(rgb, 0.0)
    rgb[ct < -0.05] = 0.0
    return rgb
