"""Seeded synthetic workloads (the reference publishes no datasets for this path).

All randomness comes from one counter-based splitmix64 stream family, so the
same seed yields the same geometry and rays in every process, in the tests,
the bench and the oracle checks.  Uniforms are the top 53 bits scaled to
[0, 1); normals come from Box-Muller on pairs of uniforms.
"""
from __future__ import annotations

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_C1 = np.uint64(0xBF58476D1CE4E5B9)
_C2 = np.uint64(0x94D049BB133111EB)


def _mix(z: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * _C1
        z = (z ^ (z >> np.uint64(27))) * _C2
    return z ^ (z >> np.uint64(31))


def splitmix64(seed: int, stream: int, n: int) -> np.ndarray:
    """n raw 64-bit outputs of stream `stream` of generator `seed`."""
    base = _mix(np.array([(seed * 0x100000001B3 + stream * 0x2545F4914F6CDD1D) & 0xFFFFFFFFFFFFFFFF],
                         dtype=np.uint64))[0]
    i = np.arange(1, n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = base + i * _GOLDEN
    return _mix(z)


def uniform(seed: int, stream: int, n: int) -> np.ndarray:
    return (splitmix64(seed, stream, n) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def normal(seed: int, stream: int, n: int) -> np.ndarray:
    m = (n + 1) // 2
    u = uniform(seed, stream, 2 * m)
    u1 = np.maximum(u[0::2], 1e-300)
    u2 = u[1::2]
    r = np.sqrt(-2.0 * np.log(u1))
    z = np.concatenate([r * np.cos(2 * np.pi * u2), r * np.sin(2 * np.pi * u2)])
    return z[:n]


class TriangleSoup:
    """positions (V, 4) float32 (w = 0), indices (T, 4) uint32 (.w = 0)."""

    def __init__(self, positions: np.ndarray, indices: np.ndarray):
        self.positions = np.ascontiguousarray(positions, dtype=np.float32)
        self.indices = np.ascontiguousarray(indices, dtype=np.uint32)

    @property
    def triangle_count(self) -> int:
        return self.indices.shape[0]


def random_triangles(n: int, seed: int = 1, sigma: float = 0.02) -> TriangleSoup:
    """n triangles: centroid ~ U[-1,1]^3, each vertex = centroid + N(0, sigma^2)^3."""
    cen = uniform(seed, 0, 3 * n).reshape(n, 3) * 2.0 - 1.0
    off = normal(seed, 1, 9 * n).reshape(n, 3, 3) * sigma
    v = (cen[:, None, :] + off).reshape(3 * n, 3)
    pos = np.zeros((3 * n, 4), dtype=np.float32)
    pos[:, :3] = v.astype(np.float32)
    idx = np.zeros((n, 4), dtype=np.uint32)
    idx[:, :3] = np.arange(3 * n, dtype=np.uint32).reshape(n, 3)
    return TriangleSoup(pos, idx)


def sphere_rays(n: int, seed: int = 2, radius: float = 3.0, target_half: float = 0.5, tmin: float = 1e-4,
                tmax: float = np.inf) -> np.ndarray:
    """(n, 8) float32 rays: origin uniform on the sphere of `radius`, direction
    normalised toward a uniform point of [-target_half, target_half]^3."""
    g = normal(seed, 0, 3 * n).reshape(n, 3)
    g /= np.linalg.norm(g, axis=1, keepdims=True)
    o = g * radius
    tgt = (uniform(seed, 1, 3 * n).reshape(n, 3) * 2.0 - 1.0) * target_half
    d = tgt - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.empty((n, 8), dtype=np.float32)
    rays[:, 0:3] = o.astype(np.float32)
    rays[:, 3] = tmin
    rays[:, 4:7] = d.astype(np.float32)
    rays[:, 7] = tmax
    return rays


def config1(n_tris: int = 65536, n_rays: int = 1 << 20, seed: int = 2024):
    """Plain BVH build + closest-hit query workload: 65,536 float32 triangles,
    1,048,576 rays, tmin 1e-4, tmax +inf."""
    return random_triangles(n_tris, seed=seed), sphere_rays(n_rays, seed=seed + 1)


# ---------------------------------------------------------------- box room
def grid_quad(origin, edge_u, edge_v, n: int):
    """n x n cells over the parallelogram origin + [0,1] edge_u + [0,1] edge_v, two
    triangles per cell, winding so the normal is edge_u x edge_v."""
    o = np.asarray(origin, np.float64)
    eu = np.asarray(edge_u, np.float64)
    ev = np.asarray(edge_v, np.float64)
    s = np.linspace(0.0, 1.0, n + 1)
    uu, vv = np.meshgrid(s, s, indexing="ij")
    pos = o + uu[..., None] * eu + vv[..., None] * ev
    pos = pos.reshape(-1, 3).astype(np.float32)
    i = np.arange(n)
    a = (i[:, None] * (n + 1) + i[None, :]).reshape(-1)
    b = a + (n + 1)
    c = b + 1
    d = a + 1
    tris = np.stack([np.stack([a, b, c], 1), np.stack([a, c, d], 1)], 1).reshape(-1, 3).astype(np.uint32)
    return pos, tris


def box_mesh(lo, hi, n: int):
    """Axis-aligned box [lo, hi], each face n x n cells, outward winding."""
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    dx, dy, dz = hi - lo
    X, Y, Z = np.array([dx, 0, 0]), np.array([0, dy, 0]), np.array([0, 0, dz])
    faces = [
        (lo, Y, X),                     # z = lo.z, normal -z
        (lo + Z, X, Y),                 # z = hi.z, normal +z
        (lo, Z, Y),                     # x = lo.x, normal -x
        (lo + X, Y, Z),                 # x = hi.x, normal +x
        (lo, X, Z),                     # y = lo.y, normal -y
        (lo + Y, Z, X),                 # y = hi.y, normal +y
    ]
    ps, ts, off = [], [], 0
    for o, eu, ev in faces:
        p, t = grid_quad(o, eu, ev, n)
        ps.append(p)
        ts.append(t + off)
        off += p.shape[0]
    return np.concatenate(ps), np.concatenate(ts)


def box_room(wall_cells: int = 128, box_cells: int = 64):
    """Procedural box room: five unit walls (open at z = 1), a 0.3 box
    (smooth dielectric, IOR 1.5) and a 0.3 x 0.6 x 0.3 box (GGX conductor,
    roughness 0.2), a 0.25 x 0.25 emitter under the ceiling (radiance 15).

    With the defaults: 5 x 128^2 x 2 + 2 x 6 x 64^2 x 2 + 2 = 262,146 triangles.
    Returns (engine.Scene, engine.Camera) for a 40 degree pinhole camera."""
    from .engine import Camera, Material, Mesh, Scene
    mats = [
        Material(base_color=(0.75, 0.75, 0.75), specular_intensity=0.0),        # 0 grey walls (Lambertian)
        Material(base_color=(0.63, 0.06, 0.05), specular_intensity=0.0),        # 1 left wall
        Material(base_color=(0.14, 0.45, 0.09), specular_intensity=0.0),        # 2 right wall
        Material(base_color=(0.9, 0.85, 0.6), roughness=0.2, metallic=1.0),    # 3 GGX conductor
        Material(base_color=(1.0, 1.0, 1.0), roughness=0.0, transmission=1.0, ior=1.5),  # 4 smooth dielectric
        Material(base_color=(0.0, 0.0, 0.0), emission=(15.0, 15.0, 15.0), specular_intensity=0.0),  # 5 emitter
    ]
    n = wall_cells
    meshes = []
    walls = [
        ((0, 0, 0), (0, 0, 1), (1, 0, 0), 0),   # floor y=0, normal +y
        ((0, 1, 0), (1, 0, 0), (0, 0, 1), 0),   # ceiling y=1, normal -y
        ((0, 0, 0), (1, 0, 0), (0, 1, 0), 0),   # back z=0, normal +z
        ((0, 0, 0), (0, 1, 0), (0, 0, 1), 1),   # left x=0, normal +x
        ((1, 0, 0), (0, 0, 1), (0, 1, 0), 2),   # right x=1, normal -x
    ]
    for o, eu, ev, m in walls:
        p, t = grid_quad(o, eu, ev, n)
        meshes.append(Mesh(p, t, m))
    p, t = box_mesh((0.55, 0.001, 0.15), (0.85, 0.601, 0.45), box_cells)  # lifted: no face coplanar with the floor
    meshes.append(Mesh(p, t, 3))
    p, t = box_mesh((0.15, 0.001, 0.5), (0.45, 0.301, 0.8), box_cells)
    meshes.append(Mesh(p, t, 4))
    h = 0.125
    p, t = grid_quad((0.5 - h, 0.999, 0.5 - h), (2 * h, 0, 0), (0, 0, 2 * h), 1)  # normal -y (down)
    meshes.append(Mesh(p, t, 5))
    cam = Camera(eye=(0.5, 0.5, 1.94), target=(0.5, 0.5, 0.0), fov_y_deg=40.0)
    return Scene(meshes=meshes, materials=mats), cam


# ---------------------------------------------------------------- instanced cloud
def icosphere(level: int):
    """Unit icosphere: the icosahedron with each face split into 4, `level`
    times, new vertices projected to the sphere.  20 * 4**level triangles,
    outward winding; shared edges produce bit-identical midpoints."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t],
                  [0, -1, -t], [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4],
                  [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8],
                  [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], np.int64)
    for _ in range(level):
        a, b, c = f[:, 0], f[:, 1], f[:, 2]
        edges = np.concatenate([np.stack([a, b], 1), np.stack([b, c], 1), np.stack([c, a], 1)])
        key = np.sort(edges, axis=1)
        uniq, inv = np.unique(key, axis=0, return_inverse=True)
        mid = v[uniq[:, 0]] + v[uniq[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        m = inv.reshape(3, -1) + v.shape[0]
        ab, bc, ca = m[0], m[1], m[2]
        v = np.concatenate([v, mid])
        f = np.concatenate([np.stack([a, ab, ca], 1), np.stack([b, bc, ab], 1), np.stack([c, ca, bc], 1),
                            np.stack([ab, bc, ca], 1)])
    return v.astype(np.float32), f.astype(np.uint32)


def torus(major: int = 256, minor: int = 64, R: float = 0.7, r: float = 0.3):
    """Torus around +y with `major` x `minor` segments (2 triangles each), outward winding."""
    u = 2 * np.pi * np.arange(major) / major
    w = 2 * np.pi * np.arange(minor) / minor
    U, W = np.meshgrid(u, w, indexing="ij")
    ring = R + r * np.cos(W)
    pos = np.stack([ring * np.cos(U), r * np.sin(W), ring * np.sin(U)], -1).reshape(-1, 3).astype(np.float32)
    i = np.arange(major)[:, None]
    j = np.arange(minor)[None, :]
    a = i * minor + j
    b = ((i + 1) % major) * minor + j
    c = ((i + 1) % major) * minor + (j + 1) % minor
    d = i * minor + (j + 1) % minor
    tris = np.stack([np.stack([a, d, c], -1), np.stack([a, c, b], -1)], -2).reshape(-1, 3).astype(np.uint32)
    return pos, tris


def random_rotations(u: np.ndarray) -> np.ndarray:
    """Uniform rotations from (n, 3) uniforms (Shoemake's unit-quaternion method)."""
    u1, u2, u3 = u[:, 0], u[:, 1], u[:, 2]
    q = np.stack([np.sqrt(1 - u1) * np.sin(2 * np.pi * u2), np.sqrt(1 - u1) * np.cos(2 * np.pi * u2),
                  np.sqrt(u1) * np.sin(2 * np.pi * u3), np.sqrt(u1) * np.cos(2 * np.pi * u3)], 1)
    x, y, z, w = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1)], 1)


def gradient_sky(width: int = 256, height: int = 128, horizon=(0.9, 0.9, 1.0), zenith=(0.25, 0.45, 0.9),
                 ground=(0.18, 0.16, 0.14)):
    """Analytic gradient sky baked to an equirectangular image (row 0 at +y):
    zenith-to-horizon blend by elevation above the horizon, flat ground below."""
    theta = np.pi * (np.arange(height) + 0.5) / height
    el = np.cos(theta)  # +1 at the zenith
    t = np.clip(el, 0.0, 1.0) ** 0.5
    sky = (1 - t)[:, None] * np.asarray(horizon) + t[:, None] * np.asarray(zenith)
    rows = np.where(el[:, None] >= 0, sky, np.asarray(ground))
    return np.ascontiguousarray(np.broadcast_to(rows[:, None, :], (height, width, 3)), np.float32)


def preetham_sky(sun_direction=(0.3, 0.8, 0.2), turbidity: float = 2.0, rayleigh: float = 1.0,
                 mie_coefficient: float = 0.005, mie_directional_g: float = 0.8, intensity: float = 1.0,
                 width: int = 256, height: int = 128):
    """Procedural daylight (core ProceduralSkyEnvironment): the Preetham 1999 sky
    baked by vt_bake_preetham_sky into a width x height equirectangular map,
    returned as an engine Environment (the reference bakes 256 x 128)."""
    import ctypes
    from . import _native as N
    from .engine import Environment

    class _Sky(ctypes.Structure):
        _fields_ = [("sun_direction", ctypes.c_float * 3), ("turbidity", ctypes.c_float),
                    ("rayleigh", ctypes.c_float), ("mie_coefficient", ctypes.c_float),
                    ("mie_directional_g", ctypes.c_float), ("intensity", ctypes.c_float)]

    d = _Sky((ctypes.c_float * 3)(*sun_direction), turbidity, rayleigh, mie_coefficient, mie_directional_g, intensity)
    rgb = np.empty((height, width, 3), np.float32)
    N.call("vt_bake_preetham_sky", ctypes.byref(d), width, height, ctypes.c_void_p(rgb.ctypes.data), rgb.size)
    return Environment(rgb)


def instanced_cloud(n_instances: int = 1024, seed: int = 3, n_points: int = 32, sphere_levels=(3, 4, 5, 6),
                    torus_segments=(256, 64), cube_cells=(32, 64, 128), extent: float = 20.0):
    """Two-level instanced workload: 8 prototype meshes (icospheres at levels
    3-6, a 256 x 64 torus, cubes with 32/64/128 cells per edge), `n_instances`
    placements with a uniform random rotation, scale U[0.2, 1] and translation
    U[-extent, extent]^3; one material per instance (50% Lambert albedo
    U[0.1, 0.9]^3, 30% GGX conductor roughness U[0.05, 0.6], 20% dielectric IOR
    U[1.3, 1.7]); a gradient sky and `n_points` point lights of intensity
    U[5, 50].  Returns (engine.Scene, engine.Camera)."""
    from .engine import Camera, Environment, Instance, Material, Mesh, PointLight, Scene
    meshes = []
    for lv in sphere_levels:
        p, t = icosphere(lv)
        meshes.append(Mesh(p, t, 0))
    p, t = torus(*torus_segments)
    meshes.append(Mesh(p, t, 0))
    for n in cube_cells:
        p, t = box_mesh((-0.6, -0.6, -0.6), (0.6, 0.6, 0.6), n)
        meshes.append(Mesh(p, t, 0))
    n = n_instances
    u = uniform(seed, 10, 16 * n).reshape(n, 16)
    rot = random_rotations(u[:, 0:3])
    scale = 0.2 + 0.8 * u[:, 3]
    trans = (u[:, 4:7] * 2 - 1) * extent
    which = np.minimum((u[:, 7] * len(meshes)).astype(np.int64), len(meshes) - 1)
    kind = u[:, 8]
    mats, insts = [], []
    for i in range(n):
        if kind[i] < 0.5:
            mats.append(Material(base_color=tuple(0.1 + 0.8 * u[i, 9:12]), specular_intensity=0.0))
        elif kind[i] < 0.8:
            mats.append(Material(base_color=tuple(0.5 + 0.45 * u[i, 9:12]), roughness=0.05 + 0.55 * u[i, 12],
                                 metallic=1.0))
        else:
            mats.append(Material(base_color=(1.0, 1.0, 1.0), roughness=0.0, transmission=1.0, ior=1.3 + 0.4 * u[i, 12]))
        M = np.eye(4)
        M[:3, :3] = rot[i] * scale[i]
        M[:3, 3] = trans[i]
        insts.append(Instance(mesh=int(which[i]), local_to_world=M.astype(np.float32), material=i))
    lp = uniform(seed, 11, 4 * n_points).reshape(n_points, 4)
    lights = [PointLight(tuple((lp[k, :3] * 2 - 1) * extent), (5 + 45 * lp[k, 3],) * 3) for k in range(n_points)]
    env = Environment(gradient_sky(), 1.0)
    cam = Camera(eye=(0.0, 6.0, 3.2 * extent), target=(0.0, 0.0, 0.0), fov_y_deg=45.0, near=0.01,
                 far=20.0 * extent)
    return Scene(meshes=meshes, materials=mats, instances=insts, point_lights=lights, environment=env), cam


# ---------------------------------------------------------------- batch of box rooms
def box_room_sized(triangles: int):
    """Box room with wall and box subdivisions chosen so that its triangle
    count (10 w^2 + 24 b^2 + 2 with b = w / 2) is close to `triangles`."""
    w = max(2, int(round((max(triangles, 64) / 16.0) ** 0.5)))
    return box_room(wall_cells=w, box_cells=max(1, w // 2))


def box_room_batch(n: int = 64, seed: int = 4):
    """Batched-launch workload: n box rooms with triangle counts log-uniform in
    [2^12, 2^21], resolution from {256^2, 512^2, 768^2, 1024^2}, 2-8 bounces,
    4-32 spp.  Returns a list of (scene, camera, width, height, bounces, spp)."""
    u = uniform(seed, 30, 4 * n).reshape(n, 4)
    out = []
    for i in range(n):
        tris = int(round(2 ** (12 + 9 * u[i, 0])))
        res = (256, 512, 768, 1024)[min(3, int(u[i, 1] * 4))]
        bounces = 2 + min(6, int(u[i, 2] * 7))
        spp = 4 + min(28, int(u[i, 3] * 29))
        sc, cam = box_room_sized(tris)
        out.append((sc, cam, res, res, bounces, spp))
    return out
