"""The BSDF tables and the CPU path tracer's BSDF against known answers (CPU).

1. The Kulla-Conty tables in vitrum_b200/csrc/ggx_albedo_lut.h are what the
   generator's recipe computes, and agree with the values the reference embeds
   (pt-webgpu/src/wgsl/pathTrace/material.wgsl.ts:2852-2869, read as text into
   tests/golden/ggx_albedo_reference.json) to 3e-4.
2. White-furnace checks of the oracle's BSDF in a uniform unit environment
   around a convex sphere (the reference's mcConvergence.test.ts /
   ggxMultiscatterFurnace.test.ts known answers): a pure Lambertian returns its
   albedo, a white GGX metal with the multiple-scattering lobe returns ~1 at
   every roughness (within the reference's furnace bounds), and white glass
   (smooth or rough) neither creates energy nor loses more than rough single
   scattering does.
"""
import importlib.util
import json
import os
import re

import numpy as np
import pytest

import oracle
from vitrum_b200 import scenes
from vitrum_b200.engine import Camera, Environment, Material, Mesh, Scene

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LUT_H = os.path.join(ROOT, "vitrum_b200", "csrc", "ggx_albedo_lut.h")


def _header_tables():
    text = open(LUT_H).read()

    def grab(name):
        body = text.split("#define " + name)[1].split("#define")[0]
        return np.array([float(v) for v in re.findall(r"(\d+\.\d+)f", body)])

    return grab("VT_GGX_E_VALUES").reshape(8, 8), grab("VT_GGX_EAVG_VALUES")


def _generator():
    spec = importlib.util.spec_from_file_location("gen_ggx_albedo",
                                                  os.path.join(ROOT, "vitrum_b200", "csrc", "gen_ggx_albedo.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_table_matches_reference_values():
    e, eavg = _header_tables()
    ref = json.load(open(os.path.join(ROOT, "tests", "golden", "ggx_albedo_reference.json")))
    assert np.abs(e.ravel() - np.array(ref["e_ss"])).max() <= 3e-4
    assert np.abs(eavg - np.array(ref["e_avg"])).max() <= 3e-4


def test_table_is_the_generator_recipe():
    gen = _generator()
    e, eavg = _header_tables()
    for i in (0, 3, 7):
        for j in range(8):
            got = gen.directional_albedo(gen.grid_roughness(i), gen.grid_roughness(j))
            assert abs(round(got, 4) - e[i, j]) <= 1.5e-4, (i, j, got, e[i, j])
    mus = (np.arange(gen.N_MU_AVG) + 0.5) / gen.N_MU_AVG
    r = gen.grid_roughness(7)
    avg = 2.0 * np.mean([gen.directional_albedo(r, m) * m for m in mus])
    assert abs(round(avg, 4) - eavg[7]) <= 1.5e-4


def _furnace(material, bounces, spp=64, W=16):
    p, t = scenes.icosphere(3)
    sc = Scene(meshes=[Mesh(p, t, 0)], materials=[material],
               environment=Environment(np.ones((8, 16, 3), np.float32)))
    cam = Camera(eye=(0.0, 0.0, 3.0), target=(0.0, 0.0, 0.0), fov_y_deg=40.0, near=0.01, far=10.0)
    s, _ = oracle.pt_render(sc, cam, W, W, spp, bounces, seed=5)
    img = s / spp
    c = W // 4
    return img[c:W - c, c:W - c].mean(axis=(0, 1))  # pixels inside the sphere's silhouette


def test_lambertian_returns_its_albedo():
    got = _furnace(Material(base_color=(0.8, 0.5, 0.2), specular_intensity=0.0), bounces=2, spp=256)
    assert np.allclose(got, (0.8, 0.5, 0.2), rtol=0.01), got


@pytest.mark.parametrize("roughness", [0.2, 0.6, 1.0])
def test_white_metal_with_multiple_scattering_is_near_one(roughness):
    # The tables are the single-scatter albedo under the Schlick-GGX G1 while
    # the BSDF uses the exact Smith G1, so mid roughness over-compensates by a
    # few percent, as in the reference; its furnace harness accepts [0.9, 1.15].
    got = _furnace(Material(base_color=(1, 1, 1), metallic=1.0, roughness=roughness), bounces=2, spp=256)
    assert np.all(got > 0.9) and np.all(got < 1.15), got


def test_dielectric_coated_diffuse_conserves_energy():
    got = _furnace(Material(base_color=(1, 1, 1), roughness=0.5), bounces=2, spp=256)
    assert np.all(got > 0.9) and np.all(got < 1.05), got


@pytest.mark.parametrize("roughness", [0.0, 0.4])
def test_white_glass_conserves_energy(roughness):
    got = _furnace(Material(base_color=(1, 1, 1), roughness=roughness, transmission=1.0, ior=1.5),
                   bounces=8, spp=256)
    lo = 0.96 if roughness == 0.0 else 0.85
    assert np.all(got > lo) and np.all(got < 1.02), got
