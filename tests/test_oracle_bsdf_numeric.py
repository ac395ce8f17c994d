"""The CPU oracle's BSDF pinned by the reference's numerical BSDF tests (CPU).

Ported checks (closed-form or quadrature targets, evaluated on the oracle's
own functions in the shading frame, normal +z):
  pt-webgpu/src/__tests__/roughDielectricNumerical.test.ts
    :104-121  the visible-normal density integrates to one
    :142-170  exact Smith G1 on a roughness x angle grid
    :172-210  transmitted densities integrate to the sampled event frequency
    :213-265  the Walter refraction Jacobian equals a finite difference
    :267-297  rough dielectric reflection + transmission <= 1
    :333-355  finite at normal, grazing, TIR and the delta boundary
  pt-webgpu/src/__tests__/energyConservation.test.ts
    :296-335  Lambert integral = albedo (1 %)
    :337-370  GGX white furnace <= 1 (+1e-2), metallic 0
  pt-webgpu/src/__tests__/ggxMultiscatterFurnace.test.ts
    :148-168  the white metal with the multiple-scattering lobe in (0.9, 1.15)
    :509-566  VNDF: D (wo.h) / (n.wo) over the sampled density = 1 / G1(wo)
    :583-611  VNDF reflections mostly above the horizon (< 8 % below)
    :613-680  VNDF estimator identity f cos / pdf = F G1(wi)
    :730-773  dielectric Fresnel: [0, 1], normal incidence, grazing, TIR
The oracle computes in f32 (as the device does), so the bars are the
reference's where f32 allows them and stated beside each check otherwise.
"""
import math

import numpy as np
import pytest

import oracle

TWO_PI = 2 * math.pi


def direction(cos_t, phi=0.0, hemi=1.0):
    s = math.sqrt(max(0.0, 1 - cos_t * cos_t))
    return np.array([s * math.cos(phi), s * math.sin(phi), hemi * cos_t])


def hemisphere_grid(hemi, steps):
    """Midpoint (theta, phi) grid over one hemisphere: directions and solid-angle weights."""
    dt, dp = 0.5 * math.pi / steps, TWO_PI / steps
    th = (np.arange(steps) + 0.5) * dt
    ph = (np.arange(steps) + 0.5) * dp
    T, P = np.meshgrid(th, ph, indexing="ij")
    d = np.stack([np.sin(T) * np.cos(P), np.sin(T) * np.sin(P), hemi * np.cos(T)], -1).reshape(-1, 3)
    return d, (np.sin(T) * dt * dp).reshape(-1)


def integrate(hemi, f, steps):
    d, w = hemisphere_grid(hemi, steps)
    return float((f(d) * w).sum())


def dielectric(roughness, eta):
    return oracle.material12(base=(1, 1, 1), roughness=roughness, metallic=0.0, transmission=1.0,
                             ior=max(eta, 1 / eta), specular=1.0)


def test_smith_g1_exact_on_grid():
    for r in (0.04, 0.1, 0.2, 0.5, 0.9):
        alpha = float(np.float32(max(r * r, 1e-3)))
        for c in (0.999999, 0.95, 0.5, 0.1, 0.001):
            cf = float(np.float32(c))
            tan2 = (1 - cf * cf) / (cf * cf)
            want = 2 / (1 + math.sqrt(1 + alpha * alpha * tan2))
            got = oracle.smith_g1(cf, alpha)
            assert 0 <= got <= 1 and abs(got - want) <= 2e-6 * want + 1e-7, (r, c, got, want)


@pytest.mark.parametrize("r", [0.2, 0.5, 0.9])
def test_visible_normal_density_integrates_to_one(r):
    mat = dielectric(r, 1.5)

    def over_slopes(wo, steps):
        du = 2 / steps
        u = -1 + (np.arange(steps) + 0.5) * du
        s = np.tan(0.5 * math.pi * u)
        jac = 0.5 * math.pi * (1 + s * s)
        SX, SY = np.meshgrid(s, s, indexing="ij")
        JX, JY = np.meshgrid(jac, jac, indexing="ij")
        wm = np.stack([SX, SY, np.ones_like(SX)], -1).reshape(-1, 3)
        wm /= np.linalg.norm(wm, axis=1, keepdims=True)
        solid = 1 / (1 + SX * SX + SY * SY) ** 1.5
        p = oracle.vndf_pdf(mat, wo, wm).astype(np.float64).reshape(SX.shape)
        return float((p * solid * JX * JY).sum() * du * du)

    for cos_o in (1.0, 0.7, 0.25):
        wo = direction(cos_o)
        coarse, fine = over_slopes(wo, 256), over_slopes(wo, 512)
        extrap = fine + (fine - coarse) / 3
        assert abs(fine - coarse) < 2e-3 and abs(extrap - fine) < 7e-4, (r, cos_o, coarse, fine)
        assert abs(extrap - 1) < 1e-3, (r, cos_o, extrap)  # reference: 5e-4 in FP64; f32 density here


@pytest.mark.parametrize("r", [0.2, 0.4, 0.75])
def test_transmission_density_matches_sampled_frequency(r):
    n = 1 << 18
    for eta in (1 / 1.5, 1.5, 2.0):
        mat = dielectric(r, eta)
        for cos_o in (1.0, 0.5):
            wo = direction(cos_o)
            # the midpoint rule needs ~2048 steps to resolve the r = 0.2 lobe to 1e-4
            steps = 2048 if r < 0.3 else 1024
            mixture = integrate(-1, lambda d: oracle.bsdf_eval(mat, eta, wo, d)[1].astype(np.float64), steps)
            wi, w, pdf, fl = oracle.bsdf_sample(mat, eta, wo, n, seed=int(1000 * r + 10 * eta + cos_o))
            sampled = float(((wi[:, 2] < -1e-8) & ((fl & 1) == 1)).mean())
            # binomial sd <= 1e-3 at 2^18 samples; the reference's bar is 5e-3 (toBeCloseTo(., 2))
            assert abs(mixture - sampled) < 2e-3, (r, eta, cos_o, mixture, sampled)


def test_walter_jacobian_matches_finite_difference():
    eta, r = 1.5, 0.42
    mat = dielectric(r, eta)
    alpha = float(np.float32(r * r))
    wo = direction(0.73, 0.31)

    def refract(wm):
        i = -wo
        ei = 1 / eta
        ndi = wm @ i
        k = 1 - ei * ei * (1 - ndi * ndi)
        v = i * ei - wm * (ei * ndi + math.sqrt(k))
        return v / np.linalg.norm(v)

    for u1, u2 in ((0.11, 0.23), (0.43, 0.77), (0.81, 0.36)):
        wm = oracle.ggx_vndf(wo, alpha, np.array([[u1, u2]]))[0].astype(np.float64)
        wm /= np.linalg.norm(wm)
        wi = refract(wm)
        assert wi[2] < 0
        ref_axis = np.array([0, 1, 0]) if abs(wm[1]) < 0.9 else np.array([1, 0, 0])
        t = np.cross(wm, ref_axis)
        t /= np.linalg.norm(t)
        b = np.cross(wm, t)
        eps = 1e-5
        pert = lambda ax, a: (wm + a * ax) / np.linalg.norm(wm + a * ax)
        du = (refract(pert(t, eps)) - refract(pert(t, -eps))) / (2 * eps)
        dv = (refract(pert(b, eps)) - refract(pert(b, -eps))) / (2 * eps)
        j_fd = 1 / abs(np.cross(du, dv) @ wi)          # d omega_m / d omega_i
        _, pdf = oracle.bsdf_eval(mat, eta, wo, wi[None])
        om = float(abs(wo @ wm))
        ev = oracle.diel_event_probs(mat, eta, float(wo[2]), om)
        p_m = float(oracle.vndf_pdf(mat, wo, wm[None])[0])
        j_oracle = float(pdf[0]) / (float(ev[2]) * p_m)
        assert abs(j_oracle - j_fd) <= 2e-3 * j_fd, (u1, u2, j_oracle, j_fd)  # f32 half vector


def test_rough_dielectric_energy_at_most_one():
    for r in (0.4, 0.7, 1.0):
        for eta in (1.25, 1.5, 2.0):
            mat = dielectric(r, eta)
            for cos_o in (1.0, 0.7, 0.3):
                wo = direction(cos_o, 0.17)

                def energy(steps):
                    up = integrate(1, lambda d: oracle.bsdf_eval(mat, eta, wo, d)[0][:, 0].astype(np.float64), steps)
                    dn = integrate(-1, lambda d: oracle.bsdf_eval(mat, eta, wo, d)[0][:, 0].astype(np.float64), steps)
                    return up + dn

                coarse, fine = energy(256), energy(512)
                extrap = fine + (fine - coarse) / 3
                assert abs(fine - coarse) < 3e-3, (r, eta, cos_o, coarse, fine)
                assert 0 <= extrap <= 1 + 5e-4, (r, eta, cos_o, extrap)


def test_sampling_finite_at_grazing_tir_and_delta():
    cases = [(1.0, 1.5, 1.0), (0.2, 1.5, 1e-4), (0.5, 1 / 1.5, 0.2), (1e-7, 2.0, 0.999), (0.0, 1.5, 0.6)]
    for r, eta, cos_o in cases:
        mat = dielectric(r, eta)
        wo = direction(cos_o)
        wi, w, pdf, fl = oracle.bsdf_sample(mat, eta, wo, 2048, seed=7)
        assert np.isfinite(wi).all() and np.isfinite(w).all() and np.isfinite(pdf).all(), (r, eta, cos_o)
        fc, p = oracle.bsdf_eval(mat, eta, wo, wi)
        assert np.isfinite(fc).all() and np.isfinite(p).all()
    # the smooth interface is a delta: no density for a transmitted direction
    mat = dielectric(0.0, 1.5)
    _, p = oracle.bsdf_eval(mat, 1.5, np.array([0, 0, 1.0]), np.array([[0, 0, -1.0]]))
    assert p[0] == 0


def test_lambert_integral_equals_albedo():
    for a in (0.5, 0.9, 1.0):
        mat = oracle.material12(base=(a, a, a), roughness=1.0, specular=0.0)
        for cos_o in (1.0, 0.6):
            e = integrate(1, lambda d: oracle.bsdf_eval(mat, 1.5, direction(cos_o), d)[0][:, 0].astype(np.float64),
                          256)
            assert abs(e - a) / a < 0.01, (a, cos_o, e)


def _furnace(mat, wo, seed):
    _, w, _, fl = oracle.bsdf_sample(mat, 1.5, wo, 1 << 18, seed=seed)
    return float(np.where((fl & 1) == 1, w[:, 0], 0).mean())


def test_ggx_white_furnace_at_most_one():
    # energyConservation.test.ts:337-370: white base colour, metallic 0 (GGX
    # specular over the diffuse base), wo along the normal: <= 1 + 1e-2
    wo = np.array([0.0, 0.0, 1.0])
    for r in (0.1, 0.3, 0.5, 0.7, 0.9):
        e = _furnace(oracle.material12(base=(1, 1, 1), roughness=r, metallic=0.0), wo, int(r * 1000))
        assert e <= 1 + 1e-2, (r, e)
    # ggxMultiscatterFurnace.test.ts:148-168: the white metal with the
    # multiple-scattering lobe stays within (0.9, 1.15) at every roughness and
    # above its single-scattering energy
    for r in (0.1, 0.3, 0.5, 0.7, 0.9):
        e = _furnace(oracle.material12(base=(1, 1, 1), roughness=r, metallic=1.0), wo, int(r * 1000) + 1)
        assert 0.9 < e < 1.15, (r, e)


def test_vndf_sampler_matches_its_density():
    rng = np.random.default_rng(5)
    wo = np.array([0.3, 0.0, 0.85])
    wo /= np.linalg.norm(wo)
    for r in (0.1, 0.5, 0.9):
        alpha = float(np.float32(max(r * r, 1e-3)))
        mat = oracle.material12(roughness=r, metallic=1.0)
        h = oracle.ggx_vndf(wo, alpha, rng.random((10000, 2))).astype(np.float64)
        p = oracle.vndf_pdf(mat, wo, h).astype(np.float64)
        ok = p > 1e-12
        assert ok.mean() > 0.95
        D = np.array([oracle.ggx_d(float(z), alpha) for z in h[ok, 2]])
        est = D * np.maximum(h[ok] @ wo, 0) / wo[2] / p[ok]
        inv_g1 = 1 / oracle.smith_g1(float(wo[2]), alpha)
        assert np.abs(est - inv_g1).max() <= 1e-4 * inv_g1, r     # pointwise (energyConservation :509-566)
        # reflection estimator identity f cos / pdf = F G1(wi), F = 1
        wi = 2 * (h @ wo)[:, None] * h - wo
        up = ok & (wi[:, 2] > 1e-5)
        g1i = np.array([oracle.smith_g1(float(z), alpha) for z in wi[up, 2]])
        g1o = oracle.smith_g1(float(wo[2]), alpha)
        Du = np.array([oracle.ggx_d(float(z), alpha) for z in h[up, 2]])
        f_cos = Du * g1o * g1i / (4 * wo[2] * wi[up, 2]) * wi[up, 2]
        pdf_refl = p[up] / (4 * (h[up] @ wo))
        assert np.abs(f_cos / pdf_refl - g1i).max() <= 1e-4, r  # energyConservation :613-680 (1e-3 there)
    # below-horizon fraction of VNDF reflections (energyConservation :583-611)
    wo = np.array([0.3, 0.0, 0.9])
    wo /= np.linalg.norm(wo)
    h = oracle.ggx_vndf(wo, 0.25, rng.random((10000, 2))).astype(np.float64)
    wi = 2 * (h @ wo)[:, None] * h - wo
    assert (wi[:, 2] < 0).mean() < 0.08


def test_dielectric_fresnel_limits():
    for eta in (1.1, 1.33, 1.5, 2.0):
        mat = oracle.material12(transmission=1.0, ior=eta)
        want = ((eta - 1) / (eta + 1)) ** 2
        assert abs(oracle.diel_fresnel(mat, 1.0, eta) - want) < 1e-6
    mat = oracle.material12(transmission=1.0, ior=1.5)
    assert abs(oracle.diel_fresnel(mat, 0.0, 1.5) - 1.0) < 1e-6                 # grazing, no TIR
    cos_c = math.sqrt(1 - (1 / 1.5) ** 2)
    assert oracle.diel_fresnel(mat, 0.5 * cos_c, 1 / 1.5) == 1.0                 # glass -> air beyond critical
    for c in np.linspace(0, 1, 101):
        f = oracle.diel_fresnel(mat, float(c), 1.5)
        assert -1e-9 <= f <= 1 + 1e-9
