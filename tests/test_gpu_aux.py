"""Auxiliary frame outputs (the normal / depth, albedo, motion and variance
textures the reference's kernel writes beside the radiance,
packages/pt-webgpu/src/wgsl/pathTrace/kernel.wgsl.ts:936-960) against closed
forms on a plane, and the luminance variance against the engine's FP64
moments."""
import ctypes

import numpy as np
import pytest

from vitrum_b200 import _native as N
from vitrum_b200.engine import Camera, Engine, Material, Mesh, Scene

pytestmark = pytest.mark.gpu

W, H = 64, 48
ALBEDO = (0.3, 0.5, 0.7)


def plane_scene(emitter=False, grey=False):
    """A 100 x 100 quad in the plane z = 0 (normal +z); optionally a small
    emitting quad above it at z = 1 facing down."""
    p = np.array([[-50, -50, 0], [50, -50, 0], [50, 50, 0], [-50, 50, 0]], np.float32)
    t = np.array([[0, 1, 2], [0, 2, 3]], np.uint32)
    mats = [Material(base_color=(0.5, 0.5, 0.5) if grey else ALBEDO, specular_intensity=0.0)]
    meshes = [Mesh(p, t, 0)]
    if emitter:
        q = np.array([[-0.3, -0.3, 1], [-0.3, 0.3, 1], [0.3, 0.3, 1], [0.3, -0.3, 1]], np.float32)
        mats.append(Material(base_color=(0, 0, 0), emission=(40.0, 40.0, 40.0), specular_intensity=0.0))
        meshes.append(Mesh(q, t, 1))
    return Scene(meshes=meshes, materials=mats)


def unproject(cam, x, y):
    """Camera ray (near-plane origin, unit direction) through viewport point
    (x, y) in pixels, the engine's raygen in float64."""
    view, proj = cam.matrices(W / H)
    vp = proj.reshape(4, 4).T.astype(np.float64) @ view.reshape(4, 4).T.astype(np.float64)
    inv = np.linalg.inv(vp)
    nx, ny = x / W * 2 - 1, 1 - y / H * 2
    n = inv @ np.array([nx, ny, -1.0, 1.0])
    f = inv @ np.array([nx, ny, 1.0, 1.0])
    o, fa = n[:3] / n[3], f[:3] / f[3]
    d = fa - o
    return o, d / np.linalg.norm(d)


def plane_distance(cam, x, y):
    o, d = unproject(cam, x, y)
    t = -o[2] / d[2]
    return t  # |P - o| for a unit direction


def test_first_hit_normal_depth_albedo(cuda):
    cam = Camera(eye=(0.0, 0.0, 2.0), target=(0.0, 0.0, 0.0), fov_y_deg=40.0)
    e = Engine(max_bounces=2)
    e.set_scene(plane_scene())
    e.render_frame(cam, W, H, samples=4, frame_seed=11)
    nd = e.capture_aux("normal_depth")
    al = e.capture_aux("albedo")
    mo = e.capture_aux("motion")
    assert np.array_equal(nd[..., :3], np.broadcast_to(np.float32([0.5, 0.5, 1.0]), (H, W, 3)))
    assert np.allclose(al, np.float32([*ALBEDO, 1.0]), atol=0, rtol=0)
    # no previous camera: the frame's own matrices, zero motion
    assert np.array_equal(mo, np.broadcast_to(np.float32([0, 0, 0, 1]), (H, W, 4)))
    # the depth of a jittered sample lies within the pixel footprint's range
    for y in range(0, H, 7):
        for x in range(0, W, 9):
            c = [plane_distance(cam, x + a, y + b) for a in (0, 1) for b in (0, 1)]
            assert min(c) * (1 - 1e-5) <= nd[y, x, 3] <= max(c) * (1 + 1e-5), (x, y, nd[y, x, 3], c)
    e.dispose()


def test_motion_of_a_translated_camera(cuda):
    a = Camera(eye=(0.0, 0.0, 2.0), target=(0.0, 0.0, 0.0), fov_y_deg=40.0)
    b = Camera(eye=(0.1, 0.0, 2.0), target=(0.1, 0.0, 0.0), fov_y_deg=40.0)
    e = Engine(max_bounces=2)
    e.set_scene(plane_scene())
    e.render_frame(a, W, H, samples=2, frame_seed=3)
    e.render_frame(b, W, H, samples=2, frame_seed=4, prev_camera=a)
    mo = e.capture_aux("motion")
    # a point at distance 2 in front of both cameras: ndc_x moves by -(k / aspect) * 0.1 / 2
    k = 1.0 / np.tan(np.radians(40.0) / 2)
    want_x = -(k / (W / H)) * 0.1 / 2 * 0.5 * W
    assert np.allclose(mo[..., 0], want_x, atol=2e-3), (mo[..., 0].min(), mo[..., 0].max(), want_x)
    assert np.allclose(mo[..., 1], 0.0, atol=2e-3)
    assert np.array_equal(mo[..., 2:], np.broadcast_to(np.float32([0, 1]), (H, W, 2)))
    # the previous camera applies to one frame: the next frame without one has no motion
    e.render_frame(b, W, H, samples=2, frame_seed=4)
    assert np.array_equal(e.capture_aux("motion")[..., :2], np.zeros((H, W, 2), np.float32))
    e.dispose()


def test_miss_defaults(cuda):
    away = Camera(eye=(0.0, 0.0, 2.0), target=(0.0, 0.0, 4.0), fov_y_deg=40.0)
    e = Engine(max_bounces=2)
    e.set_scene(plane_scene())
    e.render_frame(away, W, H, samples=2, frame_seed=1)
    assert np.array_equal(e.capture_aux("normal_depth"), np.broadcast_to(np.float32([0.5, 1, 0.5, 0]), (H, W, 4)))
    assert np.array_equal(e.capture_aux("albedo"), np.zeros((H, W, 4), np.float32))
    assert np.array_equal(e.capture_aux("motion"), np.broadcast_to(np.float32([0, 0, 0, 1]), (H, W, 4)))
    e.dispose()


def test_luminance_variance_matches_fp64_moments(cuda):
    """Grey materials and a white emitter: every sample's luminance equals its
    red channel (Rec. 709 weights sum to 1), so the float32 luminance variance
    is the FP64 per-sample variance of red rescaled from n - 1 to n."""
    cam = Camera(eye=(0.0, -1.5, 1.5), target=(0.0, 0.0, 0.0), fov_y_deg=50.0)
    e = Engine(max_bounces=3, oracle_accumulation=True)
    e.set_scene(plane_scene(emitter=True, grey=True))
    for k in range(3):
        e.render_frame(cam, W, H, samples=16, frame_seed=21)
    n = 48
    v32 = e.capture_aux("variance")
    assert np.array_equal(v32[..., 1:], np.zeros((H, W, 3), np.float32))
    mean, var = e.capture_moments()
    want = var[..., 0] * (n - 1) / n
    err = np.abs(v32[..., 0] - want)
    tol = 2e-3 * want + 2e-5 * (1.0 + mean[..., 0] ** 2)
    assert (err <= tol).all(), float((err - tol).max())
    assert want.max() > 0.01  # the scene is not trivially noise-free
    e.reset()
    e.render_frame(cam, W, H, samples=1, frame_seed=22)
    assert np.array_equal(e.capture_aux("variance")[..., 0], np.zeros((H, W), np.float32))  # one sample each
    e.dispose()


def test_aux_validation(cuda):
    e = Engine(max_bounces=2)
    e.set_scene(plane_scene())
    with pytest.raises(N.VtError):
        e.capture_aux("normal_depth")  # before any frame
    e.render_frame(Camera(eye=(0.0, 0.0, 2.0), target=(0.0, 0.0, 0.0)), 8, 8, samples=1)
    buf = np.empty(8 * 8 * 4, np.float32)
    for kind, cap in ((4, buf.size), (-1, buf.size), (0, buf.size - 1)):
        with pytest.raises(N.VtError):
            N.call("vt_capture_aux", e.handle, kind, ctypes.c_void_p(buf.ctypes.data), cap)
    m = (ctypes.c_float * 16)(*np.eye(4, dtype=np.float32).reshape(-1))
    with pytest.raises(N.VtError):
        N.call("vt_set_previous_camera", e.handle, m, None)
    bad = (ctypes.c_float * 16)(*([float("nan")] * 16))
    with pytest.raises(N.VtError):
        N.call("vt_set_previous_camera", e.handle, bad, m)
    assert "aux-outputs" in e.capabilities["features"]
    e.dispose()
