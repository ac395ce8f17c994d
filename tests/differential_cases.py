"""Inputs of the reference's CWBVH differential gate
(shared-bvh/src/__tests__/compressedWideBvhDifferential.test.ts:150-279),
regenerated here: a 128-triangle random mesh (centres uniform in
[-100, 100]^3, edges uniform in [-4, 4]^3 with |e1 x e2|^2 >= 0.25, xorshift32
seeded 0x51a7c0de) and 512 rays (xorshift32 seeded 0xc001d00d): even rays come
down a random triangle's normal from 2..302 away, odd rays start uniformly in
[-250, 250]^3 with a uniform direction; tMin 0.001 + U*0.05, tMax 20 + U*400.
The gate: leaf-size-1 wide traversal equals a canonical traversal on every
ray, with more than 100 hits and more than 100 misses."""
import numpy as np

from vitrum_b200 import scenes


def xorshift32(seed):
    state = seed & 0xFFFFFFFF

    def random():
        nonlocal state
        state ^= (state << 13) & 0xFFFFFFFF
        state ^= state >> 17
        state ^= (state << 5) & 0xFFFFFFFF
        return state / 4294967296.0

    return random


def _normalize(v):
    v = np.asarray(v, np.float64)
    return v / np.sqrt(max(float(v @ v), 1e-30))


def random_mesh(n=128):
    rnd = xorshift32(0x51A7C0DE)
    pos, idx, centers, normals = [], [], [], []
    for tri in range(n):
        c = np.array([rnd() * 200 - 100, rnd() * 200 - 100, rnd() * 200 - 100])
        while True:
            e1 = np.array([rnd() * 8 - 4, rnd() * 8 - 4, rnd() * 8 - 4])
            e2 = np.array([rnd() * 8 - 4, rnd() * 8 - 4, rnd() * 8 - 4])
            nrm = np.cross(e1, e2)
            if nrm @ nrm >= 0.25:
                break
        v0 = c - (e1 + e2) / 3
        pos += [[*v0, 0], [*(v0 + e1), 0], [*(v0 + e2), 0]]
        idx.append([3 * tri, 3 * tri + 1, 3 * tri + 2, 0])
        centers.append(c)
        normals.append(_normalize(nrm))
    return scenes.TriangleSoup(np.array(pos, np.float32), np.array(idx, np.uint32)), centers, normals


def differential_rays(centers, normals, n=512):
    rnd = xorshift32(0xC001D00D)
    rays = np.zeros((n, 8), np.float32)
    for i in range(n):
        if i % 2 == 0:
            tri = int(rnd() * len(centers))
            dist = 2 + rnd() * 300
            o = centers[tri] + normals[tri] * dist
            d = -normals[tri]
        else:
            o = np.array([rnd() * 500 - 250, rnd() * 500 - 250, rnd() * 500 - 250])
            d = _normalize([rnd() * 2 - 1, rnd() * 2 - 1, rnd() * 2 - 1])
        tmin = 0.001 + rnd() * 0.05
        tmax = 20 + rnd() * 400
        rays[i, 0:3] = o
        rays[i, 3] = tmin
        rays[i, 4:7] = d
        rays[i, 7] = tmax
    return rays
