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
