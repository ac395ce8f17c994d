"""CPU oracle for the ray-tracing hot path -- TEST INFRASTRUCTURE ONLY.

This package is the checker.  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg import it; the product package
``vitrum_b200`` never does, and its CUDA path fails loudly when its own
extension is missing instead of falling back here.

The C restatement (``bvh_oracle.c``) follows the reference's shared-bvh CPU
code (file:line citations in that file's header).  ``liborc.so`` is built by
``make -C oracle`` (``__graft_entry__.build()`` runs it).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

LEAF_FLAG = 0xFFFF0000


def build_library() -> str:
    """Compile liborc.so in place (gcc; no reference sources involved)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "liborc.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liborc.so")
        src = os.path.join(_HERE, "bvh_oracle.c")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            build_library()
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        L.orc_last_error.restype = ctypes.c_char_p
        L.orc_hw_threads.restype = ctypes.c_int
        L.orc_build_array_bvh.restype = ctypes.c_long
        L.orc_build_array_bvh.argtypes = [P, ctypes.c_long, ctypes.c_int, P, ctypes.c_long, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P]
        L.orc_collapse_wide.restype = ctypes.c_long
        L.orc_collapse_wide.argtypes = [P, ctypes.c_long, ctypes.c_long, ctypes.c_long, P, P, P, P, P, P]
        L.orc_first_hit_batch.restype = ctypes.c_int
        L.orc_first_hit_batch.argtypes = [P, P, P, P, ctypes.c_long, P, ctypes.c_int, P, ctypes.c_int, P,
                                          ctypes.c_long, P, ctypes.c_long, P, P, P, P, ctypes.c_int]
        L.orc_count_visits.restype = ctypes.c_int
        L.orc_count_visits.argtypes = [P, P, P, P, ctypes.c_long, P, ctypes.c_int, P, ctypes.c_int, P,
                                       ctypes.c_long, P, P, ctypes.c_int, ctypes.c_int]
        L.orc_brute_first_hit.restype = ctypes.c_int
        L.orc_brute_first_hit.argtypes = [P, ctypes.c_int, P, ctypes.c_int, ctypes.c_long, P, ctypes.c_long,
                                          P, P, P, P]
        L.orc_triangle_fp64.restype = ctypes.c_int
        L.orc_triangle_fp64.argtypes = [P, P, P, P, P, ctypes.c_double, P, P]
        L.orc_watertight_f32.restype = ctypes.c_int
        L.orc_watertight_f32.argtypes = [P, P, P, P, P, ctypes.c_float, P, P, P, P]
        L.orc_first_hit_wt_batch.restype = ctypes.c_int
        L.orc_first_hit_wt_batch.argtypes = [P, P, P, P, ctypes.c_long, P, ctypes.c_int, P, ctypes.c_int, P,
                                             ctypes.c_long, P, ctypes.c_long, P, P, P, ctypes.c_int]
        L.orc_build_tlas.restype = ctypes.c_long
        L.orc_build_tlas.argtypes = [P, ctypes.c_long, ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P]
        L.orc_wide_stack_entries.restype = ctypes.c_long
        L.orc_wide_stack_entries.argtypes = [P, P, ctypes.c_long]
        _LIB = L
    return _LIB


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def hw_threads() -> int:
    return int(lib().orc_hw_threads())


class BinaryBvh:
    """Result of the binary build: packed nodes plus triangle permutation."""

    def __init__(self, nodes, reordered_to_source, indices, idx_stride):
        self.nodes = nodes                      # (n, 8) uint32, buildArrayBvh.ts:13-27 layout
        self.reordered_to_source = reordered_to_source
        tri = reordered_to_source.astype(np.int64)
        idx = indices.reshape(-1, idx_stride)
        ro = np.zeros_like(idx)
        ro[:, :3] = idx[tri, :3]
        self.reordered_indices = ro.reshape(-1)  # reorderedIndices, padding lanes zero
        self.idx_stride = idx_stride

    @property
    def node_count(self):
        return self.nodes.shape[0]


def build_array_bvh(positions, indices, pos_stride=4, idx_stride=4, max_leaf=4, bins=16, max_depth=58):
    """buildArrayBvh (buildArrayBvh.ts:342) on float32 positions / uint32 indices."""
    positions = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1)
    indices = np.ascontiguousarray(indices, dtype=np.uint32).reshape(-1)
    ntri = indices.size // idx_stride
    cap = max(1, 2 * ntri)
    nodes = np.zeros((cap, 8), dtype=np.uint32)
    r2s = np.zeros(max(ntri, 1), dtype=np.uint32)
    n = lib().orc_build_array_bvh(_p(positions), positions.size, pos_stride, _p(indices), ntri, idx_stride,
                                  max_leaf, bins, max_depth, _p(nodes), _p(r2s))
    if n < 0:
        raise RuntimeError(lib().orc_last_error().decode())
    return BinaryBvh(nodes[:n].copy(), r2s[:ntri].copy(), indices, idx_stride)


class WideBvh:
    def __init__(self, binary, node_bounds, child_bounds, child_meta, child_count, wide_to_binary, status):
        self.binary = binary
        self.node_bounds = node_bounds      # (n, 6) float32
        self.child_bounds = child_bounds    # (n, 8, 6) uint16
        self.child_meta = child_meta        # (n, 8, 3) uint32
        self.child_count = child_count      # (n,) uint32
        self.wide_to_binary = wide_to_binary
        self.status = status                # 'wide' | 'empty' | 'binary-fallback'

    @property
    def node_count(self):
        return self.child_count.shape[0]


def collapse_wide(binary: BinaryBvh) -> WideBvh:
    """buildCompressedWideBvhFromArrayBvh (compressedWideBvh.ts:248)."""
    nb = binary.node_count
    ntri = binary.reordered_to_source.size
    cap = max(nb, 1)
    node_bounds = np.zeros((cap, 6), dtype=np.float32)
    child_bounds = np.zeros((cap, 8, 6), dtype=np.uint16)
    child_meta = np.zeros((cap, 8, 3), dtype=np.uint32)
    child_count = np.zeros(cap, dtype=np.uint32)
    w2b = np.zeros(cap, dtype=np.uint32)
    st = ctypes.c_int(0)
    n = lib().orc_collapse_wide(_p(binary.nodes), nb, ntri, cap, _p(node_bounds), _p(child_bounds),
                                _p(child_meta), _p(child_count), _p(w2b), ctypes.byref(st))
    if n < 0:
        raise RuntimeError(lib().orc_last_error().decode())
    status = {0: "wide", 1: "empty", 2: "binary-fallback"}[st.value]
    return WideBvh(binary, node_bounds[:n].copy(), child_bounds[:n].copy(), child_meta[:n].copy(),
                   child_count[:n].copy(), w2b[:n].copy(), status)


def build_tlas(aabbs, max_leaf=1, bins=16, max_depth=58):
    """buildTlas (tlas.ts:859) over (n, 6) instance AABBs (min xyz, max xyz) in double.

    Returns (nodes (m, 8) uint32, instanceIndices uint32)."""
    a = np.ascontiguousarray(aabbs, dtype=np.float64).reshape(-1, 6)
    n = a.shape[0]
    nodes = np.zeros((max(2 * n, 1), 8), np.uint32)
    perm = np.zeros(max(n, 1), np.uint32)
    m = lib().orc_build_tlas(_p(a), n, max_leaf, bins, max_depth, _p(nodes), _p(perm))
    if m < 0:
        raise RuntimeError(lib().orc_last_error().decode())
    return nodes[:m].copy(), perm[:n].copy()


def build_compressed_wide_bvh(positions, indices, **kw) -> WideBvh:
    """buildCompressedWideBvh (compressedWideBvh.ts:420)."""
    return collapse_wide(build_array_bvh(positions, indices, **kw))


def first_hit(wide: WideBvh, positions, rays, pos_stride=4, nthreads=0):
    """intersectCompressedWideBvhFirstHit (compressedWideBvh.ts:754) per ray.

    rays: (n, 8) float32 rows (ox, oy, oz, tmin, dx, dy, dz, tmax).
    Returns (prim int32 [-1 miss], t float64 [inf miss], bary float64 (n,2) = (u, v), bvh_tri int32).
    """
    positions = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1)
    rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
    n = rays.shape[0]
    prim = np.empty(n, dtype=np.int32)
    t = np.empty(n, dtype=np.float64)
    bary = np.empty((n, 2), dtype=np.float64)
    bt = np.empty(n, dtype=np.int32)
    b = wide.binary
    lib().orc_first_hit_batch(_p(wide.node_bounds), _p(wide.child_bounds), _p(wide.child_meta),
                              _p(wide.child_count), wide.node_count, _p(positions), pos_stride,
                              _p(b.reordered_indices), b.idx_stride, _p(b.reordered_to_source),
                              b.reordered_to_source.size, _p(rays), n, _p(prim), _p(t), _p(bary), _p(bt), nthreads)
    return prim, t, bary, bt


def first_hit_watertight(wide: WideBvh, positions, rays, pos_stride=4, nthreads=0):
    """First hit with the f32 watertight test (the device semantic), same tree.

    Returns (prim int32, t float32, bary float32 (n, 3) = weights of a, b, c).
    """
    positions = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1)
    rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
    n = rays.shape[0]
    prim = np.empty(n, dtype=np.int32)
    t = np.empty(n, dtype=np.float32)
    bary = np.empty((n, 3), dtype=np.float32)
    b = wide.binary
    lib().orc_first_hit_wt_batch(_p(wide.node_bounds), _p(wide.child_bounds), _p(wide.child_meta),
                                 _p(wide.child_count), wide.node_count, _p(positions), pos_stride,
                                 _p(b.reordered_indices), b.idx_stride, _p(b.reordered_to_source),
                                 b.reordered_to_source.size, _p(rays), n, _p(prim), _p(t), _p(bary), nthreads)
    return prim, t, bary


def count_visits(wide: WideBvh, positions, rays, pos_stride=4, nthreads=0, any_hit=False):
    """Near-first wide-node visits and triangle tests summed over the rays
    (any_hit: stop at the first accepted triangle, the shadow-ray query)."""
    positions = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1)
    rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
    nn = ctypes.c_long(0)
    nt = ctypes.c_long(0)
    b = wide.binary
    lib().orc_count_visits(_p(wide.node_bounds), _p(wide.child_bounds), _p(wide.child_meta),
                           _p(wide.child_count), wide.node_count, _p(positions), pos_stride,
                           _p(b.reordered_indices), b.idx_stride, _p(rays), rays.shape[0],
                           ctypes.byref(nn), ctypes.byref(nt), nthreads, 1 if any_hit else 0)
    return nn.value, nt.value


def brute_first_hit(positions, indices, rays, pos_stride=4, idx_stride=4):
    """Every triangle with the FP64 test; also returns the second-nearest t."""
    positions = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1)
    indices = np.ascontiguousarray(indices, dtype=np.uint32).reshape(-1)
    rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
    n = rays.shape[0]
    prim = np.empty(n, dtype=np.int32)
    t = np.empty(n, dtype=np.float64)
    bary = np.empty((n, 2), dtype=np.float64)
    second = np.empty(n, dtype=np.float64)
    lib().orc_brute_first_hit(_p(positions), pos_stride, _p(indices), idx_stride, indices.size // idx_stride,
                              _p(rays), n, _p(prim), _p(t), _p(bary), _p(second))
    return prim, t, bary, second


def triangle_fp64(o, d, a, b, c, tmin=0.0):
    f = lambda v: np.ascontiguousarray(v, dtype=np.float32)
    t = ctypes.c_double(0)
    bary = np.zeros(3, dtype=np.float64)
    hit = lib().orc_triangle_fp64(_p(f(o)), _p(f(d)), _p(f(a)), _p(f(b)), _p(f(c)), tmin, ctypes.byref(t), _p(bary))
    return bool(hit), t.value, bary


def watertight_f32(o, d, a, b, c, exclusive_min_t=0.0):
    """intersectOpticalTriangleWatertightF32 (opticalWatertightTriangle.ts:98)."""
    f = lambda v: np.ascontiguousarray(v, dtype=np.float32)
    t = ctypes.c_float(0)
    bary = np.zeros(3, dtype=np.float32)
    side = ctypes.c_int(0)
    mask = ctypes.c_int(0)
    hit = lib().orc_watertight_f32(_p(f(o)), _p(f(d)), _p(f(a)), _p(f(b)), _p(f(c)), exclusive_min_t,
                                   ctypes.byref(t), _p(bary), ctypes.byref(side), ctypes.byref(mask))
    return dict(hit=bool(hit), t=t.value, bary=bary, side=side.value, zero_edge_mask=mask.value)


# ---------------------------------------------------------------- path tracer
def _pt_lib():
    L = lib()
    if not getattr(L, "_pt_ready", False):
        P = ctypes.c_void_p
        L.orc_pt_render.restype = ctypes.c_int
        L.orc_pt_render.argtypes = [P, ctypes.c_long, P, ctypes.c_long, P, P, ctypes.c_int, P, ctypes.c_long, P,
                                    ctypes.c_long, P, ctypes.c_long, P,
                                    ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float, P, ctypes.c_int,
                                    ctypes.c_int,
                                    ctypes.c_int, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float,
                                    ctypes.c_int, P, P, P, P, ctypes.c_long, P, ctypes.c_int]
        L.orc_pt_scene_create.restype = ctypes.c_void_p
        L.orc_pt_scene_create.argtypes = [P, ctypes.c_long, P, ctypes.c_long, P, P, ctypes.c_int, P, ctypes.c_long,
                                          P, ctypes.c_long, P, ctypes.c_long, P, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_int]
        L.orc_pt_scene_render.restype = ctypes.c_int
        L.orc_pt_scene_render.argtypes = [P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int, P, P, P, P, ctypes.c_long,
                                          P]
        L.orc_pt_scene_free.restype = None
        L.orc_pt_scene_free.argtypes = [P]
        L._pt_ready = True
    return L


def flatten_scene(scene):
    """(positions (V,4) f32, indices (T,4) u32, tri_material u32, materials (M,12) f32,
    positional lights (P,16) f32, env (H,W,3) f32 or None, env_intensity) from an engine Scene."""
    pos, idx, tm = [], [], []
    base = 0
    for m in scene.meshes:
        p = np.asarray(m.positions, np.float32).reshape(-1, 3)
        i = np.asarray(m.indices, np.uint32).reshape(-1, 3)
        p4 = np.zeros((p.shape[0], 4), np.float32)
        p4[:, :3] = p
        i4 = np.zeros((i.shape[0], 4), np.uint32)
        i4[:, :3] = i + base
        pos.append(p4)
        idx.append(i4)
        tm.append(np.full(i.shape[0], m.material, np.uint32))
        base += p.shape[0]
    mats = np.zeros((len(scene.materials), 12), np.float32)
    for k, m in enumerate(scene.materials):
        mats[k, 0:3] = m.base_color
        mats[k, 3:7] = (m.roughness, m.metallic, m.transmission, m.ior)
        mats[k, 7:10] = m.emission
        mats[k, 10] = (0 if getattr(m, "double_sided", True) else 1) | (0 if getattr(m, "cast_shadow", True) else 2)
        mats[k, 11] = getattr(m, "specular_intensity", 1.0)
    pts = positional_lights(scene)
    env = None if scene.environment is None else np.ascontiguousarray(scene.environment.rgb, np.float32)
    ei = 1.0 if scene.environment is None else float(scene.environment.intensity)
    return np.concatenate(pos), np.concatenate(idx), np.concatenate(tm), mats, pts, env, ei


def positional_lights(scene):
    """(n, 16) float32, points then spots: position, 0, intensity, 0, axis, cos outer,
    cos inner, range, decay, spot flag (points: no cone, no range, decay 2)."""
    rows = []
    for l in scene.point_lights:
        rows.append([*l.position, 0, *l.intensity, 0, 0, 0, 0, -2, -1, 0, 2, 0])
    for l in getattr(scene, "spot_lights", []):
        d = np.asarray(l.direction, np.float32).astype(np.float64)
        d = d / np.sqrt((d * d).sum())
        outer = float(np.float32(l.angle))
        inner = outer * (1.0 - float(np.float32(l.penumbra)))
        rows.append([*l.position, 0, *l.intensity, 0, *d, math.cos(outer), math.cos(inner), l.distance, l.decay, 1])
    return np.array(rows, np.float32).reshape(-1, 16)


def area_lights(scene):
    """(n, 16) float32, rectangles then discs: centre, shape (0 / 1), u half axis,
    area, v half axis, 0, radiance, 0 (the emitting side is u x v)."""
    rows = []
    for r in getattr(scene, "rect_lights", []):
        u = np.float32(0.5) * np.asarray(r.edge_u, np.float32)
        v = np.float32(0.5) * np.asarray(r.edge_v, np.float32)
        c = (np.asarray(r.corner, np.float32) + u) + v
        cr = np.cross(u.astype(np.float64), v.astype(np.float64))
        rows.append([*c, 0, *u, 4.0 * math.sqrt((cr * cr).sum()), *v, 0, *r.radiance, 0])
    for dl in getattr(scene, "disc_lights", []):
        n = np.asarray(dl.normal, np.float32).astype(np.float64)
        n = n / math.sqrt((n * n).sum())
        t = np.array([-n[2], 0.0, n[0]]) if abs(n[0]) > 0.9 else np.array([0.0, n[2], -n[1]])
        t = t / math.sqrt((t * t).sum())
        b = np.array([n[1] * t[2] - n[2] * t[1], n[2] * t[0] - n[0] * t[2], n[0] * t[1] - n[1] * t[0]])
        rr = float(np.float32(dl.radius))
        rows.append([*dl.center, 1, *(t * rr), math.pi * rr * rr, *(b * rr), 0, *dl.radiance, 0])
    return np.array(rows, np.float32).reshape(-1, 16)


def present(rgb, tonemap=0, exposure=1.0, srgb=True):
    """The present pass on mean radiance `rgb` (..., 3), float64: exposure, then
    tonemap 0 ACES filmic (Narkowicz: x(2.51x + 0.03) / (x(2.43x + 0.59) + 0.14)),
    1 AgX (log2 range [-12.47393, 4.026069], sixth-order curve), 2 Reinhard
    x / (1 + x), 3 clamp to [0, 1], 4 none; then the sRGB OETF when `srgb`
    (shared-samplers/src/wgsl/tonemap.wgsl.ts:8-60, pt-webgpu/src/wgsl/present.wgsl.ts:59-80)."""
    x = np.asarray(rgb, np.float64)
    x = np.where(np.isnan(x) | (exposure <= 0), 0.0, np.sign(x) * np.minimum(np.abs(x) * exposure, 3.402823466e38))
    if tonemap == 1:
        lx = np.clip((np.log2(np.maximum(x, 1e-6)) + 12.47393) / (12.47393 + 4.026069), 0.0, 1.0)
        y = np.clip(15.5 * lx ** 6 - 40.14 * lx ** 5 + 31.96 * lx ** 4 - 6.868 * lx ** 3 + 0.4298 * lx ** 2
                    + 0.1191 * lx - 0.00232, 0.0, 1.0)
    elif tonemap == 2:
        v = np.maximum(x, 0.0)
        y = v / (1.0 + v)
    elif tonemap == 3:
        y = np.clip(x, 0.0, 1.0)
    elif tonemap == 4:
        y = x
    else:
        v = np.minimum(np.maximum(x, 0.0), 1e18)
        y = np.clip(v * (2.51 * v + 0.03) / (v * (2.43 * v + 0.59) + 0.14), 0.0, 1.0)
    if srgb:
        v = np.maximum(y, 0.0)
        y = np.where(v <= 0.0031308, v * 12.92, 1.055 * np.power(v, 1.0 / 2.4) - 0.055)
    return y


def directional_lights(scene):
    """(n, 8) float32: direction towards the light, cos(angular radius) (1 for a
    delta light), rgb (irradiance of a delta light, disc radiance otherwise), delta flag."""
    out = []
    for l in getattr(scene, "directional_lights", []):
        d = np.asarray(l.direction, np.float32).astype(np.float64)
        n = float(np.sqrt(d @ d))
        delta = float(l.angular_radius) == 0.0
        st = np.sin(np.float64(np.float32(l.angular_radius)))
        to_l = 1.0 if delta else 1.0 / (np.pi * st * st)
        E = np.asarray(l.irradiance, np.float32).astype(np.float64)
        out.append([*(-d / n), 1.0 if delta else np.cos(np.float64(np.float32(l.angular_radius))),
                    *(E * to_l), 1.0 if delta else 0.0])
    return np.array(out, np.float32).reshape(-1, 8)


def inverse_view_proj(camera, width, height):
    """Row-major float32 inverse of projection * view, as the engine computes it."""
    view, proj = camera.matrices(width / height)
    V = np.asarray(view, np.float64).reshape(4, 4).T
    Pm = np.asarray(proj, np.float64).reshape(4, 4).T
    return np.linalg.inv(Pm @ V).astype(np.float32)


class PtScene:
    """The CPU path tracer's scene, set up once (BVH build, material table,
    emitter and environment CDFs) and rendered any number of times."""

    def __init__(self, scene, bias=2e-5, light_selection="tree"):
        pos, idx, tm, mats, pts, env, ei = flatten_scene(scene)
        dls = directional_lights(scene)
        als = area_lights(scene)
        er = 0.0 if scene.environment is None else float(getattr(scene.environment, "rotation_y", 0.0))
        ew, eh = (0, 0) if env is None else (env.shape[1], env.shape[0])
        # the C side borrows these arrays: keep them alive with the handle
        self._keep = (pos, idx, tm, mats, pts, env, dls, als)
        self.triangles = int(idx.shape[0])
        self.handle = _pt_lib().orc_pt_scene_create(
            _p(pos), pos.shape[0], _p(idx), idx.shape[0], _p(tm), _p(mats), mats.shape[0],
            _p(pts) if pts.size else None, pts.shape[0], _p(als) if als.size else None, als.shape[0],
            _p(dls) if dls.size else None, dls.shape[0], _p(env) if env is not None else None, ew, eh, ei, er, bias,
            {"tree": 0, "uniform": 1}[light_selection])
        if not self.handle:
            raise RuntimeError("oracle path tracer: scene build failed")

    def render(self, camera, width, height, spp, max_bounces, seed=0, sample_base=0, nthreads=0, log_rays=0):
        """(sum, sum_sq) FP64 per pixel, shapes (H, W, 3); with log_rays > 0 also
        (closest_rays, shadow_rays, (n_closest, n_shadow)) as pt_render."""
        ivp = np.ascontiguousarray(inverse_view_proj(camera, width, height))
        s = np.zeros((height, width, 3), np.float64)
        q = np.zeros_like(s)
        lc = np.zeros((max(log_rays, 0), 8), np.float32)
        ls = np.zeros((max(log_rays, 0), 8), np.float32)
        totals = np.zeros(2, np.int64)
        _pt_lib().orc_pt_scene_render(self.handle, _p(ivp), width, height, spp, max_bounces, seed, sample_base,
                                      nthreads, _p(s), _p(q), _p(lc) if log_rays else None,
                                      _p(ls) if log_rays else None, max(log_rays, 0), _p(totals))
        self.last_totals = (int(totals[0]), int(totals[1]))
        if log_rays:
            nc, ns = self.last_totals
            return s, q, lc[:min(nc, log_rays)], ls[:min(ns, log_rays)], (nc, ns)
        return s, q

    def close(self):
        if self.handle:
            _pt_lib().orc_pt_scene_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pt_render(scene, camera, width, height, spp, max_bounces, seed=0, sample_base=0, bias=2e-5, nthreads=0,
              log_rays=0, light_selection="tree"):
    """CPU path tracer: (sum, sum_sq) FP64 per pixel, shapes (H, W, 3).

    With log_rays > 0 also returns (closest_rays, shadow_rays, totals): the
    first log_rays extension and shadow rays as (n, 8) float32 rows and the
    total number of each traced."""
    S = PtScene(scene, bias=bias, light_selection=light_selection)
    try:
        return S.render(camera, width, height, spp, max_bounces, seed=seed, sample_base=sample_base,
                        nthreads=nthreads, log_rays=log_rays)
    finally:
        S.close()


def pt_ray_totals(pt_scene, camera, width, height, spp, max_bounces, seed=0, nthreads=0):
    """Rays traced by one CPU render of a prepared PtScene, and its wall time:
    (closest, shadow, seconds).  The scene's BVH build is not in the time."""
    import time
    t0 = time.perf_counter()
    pt_scene.render(camera, width, height, spp, max_bounces, seed=seed, nthreads=nthreads)
    dt = time.perf_counter() - t0
    nc, ns = pt_scene.last_totals
    return nc, ns, dt


# ---------------------------------------------------------------- pick
def screen_to_world_ray(camera, px, py, width, height):
    """screenToWorldRay (shared-bvh/src/pickPrimitiveCpu.ts:68-108) in FP64 on
    the camera's float32 matrices: origin on the near plane, unit direction."""
    view, proj = camera.matrices(width / height)
    V = np.asarray(view, np.float64).reshape(4, 4).T
    Pm = np.asarray(proj, np.float64).reshape(4, 4).T
    inv = np.linalg.inv(Pm @ V)
    nx, ny = px / width * 2 - 1, 1 - py / height * 2
    far = inv @ np.array([nx, ny, 1.0, 1.0])
    near = inv @ np.array([nx, ny, -1.0, 1.0])
    far = far / np.abs(far).max()
    near = near / np.abs(near).max()
    o = near[:3] / near[3]
    orient = 1.0 if far[3] == 0 else np.sign(far[3] * near[3])
    d = (far[:3] * near[3] - near[:3] * far[3]) * orient
    return o, d / np.sqrt(d @ d)


def _ray_triangles(o, d, v0, v1, v2):
    """rayTriangle (pickPrimitiveCpu.ts:151-232) over arrays of triangles:
    hit distance (inf on a miss) and the signed barycentric margin min(u, v, w)."""
    e1r, e2r = v1 - v0, v2 - v0
    es = np.maximum(np.abs(e1r).max(1), np.abs(e2r).max(1))
    ds = np.abs(d).max()
    with np.errstate(divide="ignore", invalid="ignore"):
        e1, e2 = e1r / es[:, None], e2r / es[:, None]
        dr = d / ds
        ao = (o - v0) / es[:, None]
        n = np.cross(e1, e2)
        p = np.cross(dr, e2)
        det = np.einsum("ij,ij->i", e1, p)
        ok = (es > 0) & np.isfinite(es) & (np.abs(det) / (np.linalg.norm(n, axis=1) * np.linalg.norm(dr)) > 1e-7)
        inv = 1.0 / det
        u = np.einsum("ij,ij->i", ao, p) * inv
        q = np.cross(ao, e1)
        v = (q @ dr) * inv
        w = 1 - u - v
        t = np.einsum("ij,ij->i", e2, q) * inv * es / ds
        margin = np.minimum(np.minimum(u, v), w)
        ok &= np.isfinite(u) & np.isfinite(v) & np.isfinite(t) & (margin >= -1e-6) & (t > 0)
    return np.where(ok, t, np.inf), np.where(np.isfinite(margin), margin, -np.inf)


def pick_primitive(scene, camera, px, py, width, height):
    """pickPrimitiveCpu (pickPrimitiveCpu.ts:674-695) on an engine Scene:
    brute force over every triangle (placed in world space in FP64 for
    instances).  Returns None on a miss, else a dict with `mesh` (the scene
    primitive), `instance` (or -1), `triangle` (the source triangle index
    counted over all meshes in order, single-level scenes), `t` and `margin`
    (the barycentric distance of the hit to its triangle's nearest edge)."""
    if width <= 0 or height <= 0:
        return None
    o, d = screen_to_world_ray(camera, px, py, width, height)
    best = None
    items = ([(k, i.mesh, np.asarray(i.local_to_world, np.float64).reshape(4, 4)) for k, i in
              enumerate(scene.instances)] if scene.instances else
             [(-1, m, None) for m in range(len(scene.meshes))])
    tri_base = np.cumsum([0] + [m.indices.shape[0] for m in scene.meshes])
    for inst, mi, M in items:
        m = scene.meshes[mi]
        P = np.asarray(m.positions, np.float32).astype(np.float64).reshape(-1, 3)
        if M is not None:
            P = P @ M[:3, :3].T + M[:3, 3]
        I = np.asarray(m.indices, np.int64).reshape(-1, 3)
        t, margin = _ray_triangles(o, d, P[I[:, 0]], P[I[:, 1]], P[I[:, 2]])
        k = int(np.argmin(t))
        if np.isfinite(t[k]) and (best is None or t[k] < best["t"]):
            best = dict(mesh=int(mi), instance=int(inst), triangle=int(tri_base[mi] + k) if inst < 0 else -1,
                        t=float(t[k]), margin=float(margin[k]))
    return best


# ---------------------------------------------------------------- BSDF probes
def _f32(a, shape=None):
    a = np.ascontiguousarray(a, np.float32)
    return a if shape is None else a.reshape(shape)


def _bsdf_lib():
    L = _pt_lib()
    if not getattr(L, "_bsdf_ready", False):
        P = ctypes.c_void_p
        F = ctypes.c_float
        L.orc_smith_g1.restype = F
        L.orc_smith_g1.argtypes = [F, F]
        L.orc_ggx_d.restype = F
        L.orc_ggx_d.argtypes = [F, F]
        L.orc_ggx_vndf_batch.restype = None
        L.orc_ggx_vndf_batch.argtypes = [P, F, P, ctypes.c_long, P]
        L.orc_vndf_pdf_batch.restype = None
        L.orc_vndf_pdf_batch.argtypes = [P, P, P, ctypes.c_long, P]
        L.orc_diel_fresnel.restype = F
        L.orc_diel_fresnel.argtypes = [P, F, F]
        L.orc_diel_event_probs.restype = None
        L.orc_diel_event_probs.argtypes = [P, F, F, F, P]
        L.orc_bsdf_eval_batch.restype = None
        L.orc_bsdf_eval_batch.argtypes = [P, F, P, P, ctypes.c_long, P, P]
        L.orc_bsdf_sample_batch.restype = None
        L.orc_bsdf_sample_batch.argtypes = [P, F, P, ctypes.c_long, ctypes.c_uint32, P, P, P, P]
        L._bsdf_ready = True
    return L


def material12(base=(1, 1, 1), roughness=0.5, metallic=0.0, transmission=0.0, ior=1.5, specular=1.0):
    """The oracle's 12-float material record (layout at orc_pt_scene_create)."""
    return _f32([*base, roughness, metallic, transmission, ior, 0, 0, 0, 0, specular])


def smith_g1(c, alpha):
    return float(_bsdf_lib().orc_smith_g1(c, alpha))


def ggx_d(nh, alpha):
    return float(_bsdf_lib().orc_ggx_d(nh, alpha))


def ggx_vndf(wo, alpha, u):
    """Visible-normal samples (n, 3) for uniforms u (n, 2)."""
    u = _f32(u, (-1, 2))
    out = np.empty((u.shape[0], 3), np.float32)
    _bsdf_lib().orc_ggx_vndf_batch(_p(_f32(wo)), alpha, _p(u), u.shape[0], _p(out))
    return out


def vndf_pdf(mat, wo, wm):
    """Half-vector density D(wm) G1(wo) (wo.wm) / (n.wo) for directions wm (n, 3)."""
    wm = _f32(wm, (-1, 3))
    out = np.empty(wm.shape[0], np.float32)
    _bsdf_lib().orc_vndf_pdf_batch(_p(mat), _p(_f32(wo)), _p(wm), wm.shape[0], _p(out))
    return out


def diel_fresnel(mat, c, eta):
    return float(_bsdf_lib().orc_diel_fresnel(_p(mat), c, eta))


def diel_event_probs(mat, eta, cos_o, wo_wm):
    """(joint reflection, diffuse, transmission, P(reflection | not diffuse))."""
    out = np.empty(4, np.float32)
    _bsdf_lib().orc_diel_event_probs(_p(mat), eta, cos_o, wo_wm, _p(out))
    return out


def bsdf_eval(mat, eta, wo, wi):
    """(f |cos wi| rgb (n, 3), sampling density (n,)) for directions wi (n, 3)."""
    wi = _f32(wi, (-1, 3))
    fc = np.empty((wi.shape[0], 3), np.float32)
    pdf = np.empty(wi.shape[0], np.float32)
    _bsdf_lib().orc_bsdf_eval_batch(_p(mat), eta, _p(_f32(wo)), _p(wi), wi.shape[0], _p(fc), _p(pdf))
    return fc, pdf


def bsdf_sample(mat, eta, wo, n, seed=1):
    """n BSDF samples: (wi (n, 3), weight (n, 3), pdf (n,), flags (n,): bit 0 valid, bit 1 delta)."""
    wi = np.empty((n, 3), np.float32)
    w = np.empty((n, 3), np.float32)
    pdf = np.empty(n, np.float32)
    fl = np.empty(n, np.int32)
    _bsdf_lib().orc_bsdf_sample_batch(_p(mat), eta, _p(_f32(wo)), n, seed, _p(wi), _p(w), _p(pdf), _p(fl))
    return wi, w, pdf, fl


# ---------------------------------------------------------------- light tree
def _lt_lib():
    L = lib()
    if not getattr(L, "_lt_ready", False):
        P = ctypes.c_void_p
        L.orc_lt_build.restype = ctypes.c_long
        L.orc_lt_build.argtypes = [P, P, P, P, ctypes.c_long, P, ctypes.c_long]
        L.orc_lt_sample.restype = ctypes.c_float
        L.orc_lt_sample.argtypes = [P, ctypes.c_long, P, ctypes.c_float, ctypes.c_uint32, P]
        L.orc_lt_select.restype = ctypes.c_float
        L.orc_lt_select.argtypes = [P, ctypes.c_long, ctypes.c_uint32, ctypes.c_uint32, P, P, ctypes.c_float,
                                    ctypes.c_uint32, P]
        L.orc_lt_pdf.restype = ctypes.c_float
        L.orc_lt_pdf.argtypes = [P, ctypes.c_long, P, ctypes.c_float, ctypes.c_int]
        L.orc_lt_importance.restype = ctypes.c_float
        L.orc_lt_importance.argtypes = [P, ctypes.c_long, P, ctypes.c_float]
        L.orc_lt_importance_direct.restype = ctypes.c_float
        L.orc_lt_importance_direct.argtypes = [P, ctypes.c_long, P, P, ctypes.c_float]
        L._lt_ready = True
    return L


LT_BUCKETS = 1 << 24
LT_FLOOR = 1e-3


def light_tree_build(powers, centroids, aabbs, cones=None):
    """buildLightTree + packLightTreeForGPU (shared-samplers/src/lightTree.ts:492, 611):
    (nodes, 16) float32.  aabbs (n, 6) min|max; cones (n, 6) axis, thetaO, thetaE,
    oriented flag (None: every emitter full-sphere)."""
    pw = np.ascontiguousarray(powers, np.float64)
    n = pw.size
    c = np.ascontiguousarray(centroids, np.float64).reshape(n, 3)
    b = np.ascontiguousarray(aabbs, np.float64).reshape(n, 6)
    k = np.zeros((n, 6)) if cones is None else np.ascontiguousarray(cones, np.float64).reshape(n, 6)
    out = np.zeros((2 * n, 16), np.float32)
    m = _lt_lib().orc_lt_build(_p(pw), _p(c), _p(b), _p(k), n, _p(out), 2 * n)
    if m < 0:
        raise RuntimeError("light tree build failed")
    return out[:m].copy()


def light_tree_sample(tree, p, bucket, floor=LT_FLOOR):
    """samplePackedLightTreeCPU with the 24-bit draw `bucket`: (emitter, pmf)."""
    t = np.ascontiguousarray(tree, np.float32)
    e = ctypes.c_int(-1)
    pmf = _lt_lib().orc_lt_sample(_p(t), t.shape[0], _p(_f32(p)), floor, int(bucket), ctypes.byref(e))
    return e.value, float(pmf)


def light_tree_pdf(tree, p, emitter, floor=LT_FLOOR):
    """packedLightTreePdfCPU: the PMF of `emitter` at point p."""
    t = np.ascontiguousarray(tree, np.float32)
    return float(_lt_lib().orc_lt_pdf(_p(t), t.shape[0], _p(_f32(p)), floor, int(emitter)))


def light_tree_importance(tree, node, p, floor=LT_FLOOR):
    t = np.ascontiguousarray(tree, np.float32)
    return float(_lt_lib().orc_lt_importance(_p(t), int(node), _p(_f32(p)), floor))


def light_tree_importance_direct(tree, node, p, normal=None, floor=LT_FLOOR):
    """The integrator's importance of `node` at p (receiver term for `normal`,
    None: none), evaluated directly rather than in the reference's log form."""
    t = np.ascontiguousarray(tree, np.float32)
    nrm = None if normal is None else _p(_f32(normal))
    return float(_lt_lib().orc_lt_importance_direct(_p(t), int(node), _p(_f32(p)), nrm, floor))


def light_select(tree, n_pos, n_dist, p, bucket, normal=None, floor=LT_FLOOR):
    """The integrator's selection: tree over n_pos positional entries (tree None
    for one), n_dist distant entries evenly within n_dist / (n_dist + 1), the
    receiver term for `normal` (None: none): (entry, pmf)."""
    t = np.zeros((0, 16), np.float32) if tree is None else np.ascontiguousarray(tree, np.float32)
    e = ctypes.c_int(-1)
    nrm = None if normal is None else _p(_f32(normal))
    pmf = _lt_lib().orc_lt_select(_p(t) if t.size else None, t.shape[0], int(n_pos), int(n_dist), _p(_f32(p)), nrm,
                                  floor, int(bucket), ctypes.byref(e))
    return e.value, float(pmf)
