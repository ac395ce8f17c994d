"""Pins the CPU oracle against the reference's own golden vectors and known answers.

Golden: tests/golden/scenepack_golden.json, extracted by tests/golden/make_golden.py
from the reference fixture packages/shared-bvh/src/__tests__/scenePack.golden.json
(captured by scenePackGolden.test.ts).  The box / triangle scenes below restate
that test's scene builders (boxMesh, unitTriMesh, multiMeshScene).
"""
import json
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "scenepack_golden.json")
BOX_IDX = [0, 1, 2, 4, 1, 2, 1, 5, 6, 5, 4, 6, 0, 2, 3, 2, 6, 7,
           0, 1, 3, 1, 5, 3, 3, 5, 7, 5, 6, 7, 0, 4, 3, 4, 6, 7]


def box(mn, mx):
    x0, y0, z0 = mn
    x1, y1, z1 = mx
    return np.array([x0, y0, z0, x1, y0, z0, x0, y1, z0, x0, y0, z1,
                     x1, y1, z1, x1, y0, z1, x0, y1, z1, x1, y1, z1], np.float32).reshape(-1, 3)


def unit_tri():
    return np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)


SCENES = {
    "multiMesh": [box([0, 0, 0], [1, 1, 1]), box([0, 0, 0], [1, 1, 1]), unit_tri(), box([10, 0, 0], [11, 1, 1])],
    "resizeSplice": [box([0, 0, 0], [1, 1, 1]), box([5, 0, 0], [6, 1, 1])],
}


def pack(P):
    pos = np.zeros((P.shape[0], 4), np.float32)
    pos[:, :3] = P
    idx3 = np.array(BOX_IDX if P.shape[0] == 8 else [0, 1, 2], np.uint32).reshape(-1, 3)
    idx = np.zeros((idx3.shape[0], 4), np.uint32)
    idx[:, :3] = idx3
    return pos, idx


def golden_blas():
    g = json.load(open(GOLDEN))
    for name, prims in SCENES.items():
        pk = g[name]
        nodes = np.array(pk["bvhNodes"], np.uint32).reshape(-1, 8)
        idx_g = np.array(pk["indices"], np.uint32).reshape(-1, 4)
        b = pk["primitiveTlasBindings"]
        for i, (bd, P) in enumerate(zip(b, prims)):
            end = b[i + 1]["blasRoot"] if i + 1 < len(b) else nodes.shape[0]
            gn = nodes[bd["blasRoot"]:end].copy()
            leaf = (gn[:, 7] >> 16) == 0xFFFF
            gn[leaf, 6] -= bd["triStart"]          # scenePack rebases leaf offsets by triStart
            gi = idx_g[bd["triStart"]:bd["triStart"] + bd["triCount"]].copy()
            gi[:, :3] -= bd["vertexStart"]          # and index words by vertexStart
            yield f"{name}/{bd['primitiveId']}", P, gn, gi


@pytest.mark.parametrize("case", list(golden_blas()), ids=lambda c: c[0])
def test_build_matches_reference_golden_bytes(case):
    _, P, gold_nodes, gold_idx = case
    pos, idx = pack(P)
    b = oracle.build_array_bvh(pos, idx)
    assert np.array_equal(b.nodes, gold_nodes)
    assert np.array_equal(b.reordered_indices.reshape(-1, 4), gold_idx)


def golden_tlas():
    g = json.load(open(GOLDEN))
    for name in SCENES:
        pk = g[name]
        by_root = {}
        for bd in pk["primitiveTlasBindings"]:
            by_root.setdefault(bd["blasRoot"], bd)
        l2w = np.array(pk["tlasInstanceLocalToWorld"], np.float32).reshape(-1, 4, 4)
        aabbs = []
        for i, root in enumerate(pk["tlasBlasRoots"]):
            bd = by_root[root]
            lo, hi = np.array(bd["localAabbMin"], np.float64), np.array(bd["localAabbMax"], np.float64)
            M = l2w[i].astype(np.float64).T  # column-major storage
            corners = np.array([[(hi if c & 1 else lo)[0], (hi if c & 2 else lo)[1], (hi if c & 4 else lo)[2]]
                                for c in range(8)])
            w = corners @ M[:3, :3].T + M[:3, 3]  # transformAabb (scenePack.ts:197-223)
            aabbs.append(np.r_[w.min(0), w.max(0)])
        yield name, np.array(aabbs), np.array(pk["tlasNodes"], np.uint32).reshape(-1, 8), \
            np.array(pk["tlasInstanceIndices"], np.uint32), pk["tlasNodeCount"]


@pytest.mark.parametrize("case", list(golden_tlas()), ids=lambda c: c[0])
def test_tlas_matches_reference_golden_bytes(case):
    """buildTlas (tlas.ts:859) over the instances' world AABBs: node words and instance order."""
    _, aabbs, gold_nodes, gold_perm, count = case
    nodes, perm = oracle.build_tlas(aabbs)
    assert nodes.shape[0] == count
    assert np.array_equal(nodes, gold_nodes)
    assert np.array_equal(perm, gold_perm)


def test_tlas_balanced_fallback_on_coincident_instances():
    # every instance on the same AABB: SAH finds no split, the balanced median
    # fallback still gives one instance per leaf (maxLeafSize 1)
    aabbs = np.tile([0.0, 0.0, 0.0, 1.0, 1.0, 1.0], (37, 1))
    nodes, perm = oracle.build_tlas(aabbs)
    leaf = (nodes[:, 7] >> 16) == 0xFFFF
    assert (nodes[leaf, 7] & 0xFFFF).max() == 1 and leaf.sum() == 37
    assert sorted(perm.tolist()) == list(range(37))


def test_empty_and_single():
    # buildArrayBvh.test.ts:44-72
    b = oracle.build_array_bvh(np.zeros((0, 4), np.float32), np.zeros((0, 4), np.uint32))
    assert b.node_count == 1 and b.nodes[0, 7] == oracle.LEAF_FLAG and b.nodes[0, 6] == 0
    pos, idx = pack(unit_tri())
    b = oracle.build_array_bvh(pos, idx)
    assert b.node_count == 1 and b.nodes[0, 7] == (oracle.LEAF_FLAG | 1)


def test_planar_floor_is_balanced():
    # buildArrayBvh.test.ts:142-184 (B7 planar SAH): 1000 quads on y=0, depth <= 16, leaves <= 4
    side = 32
    pos, idx = [], []
    v = q = 0
    for i in range(side):
        for j in range(side):
            if q >= 1000:
                break
            pos += [i, 0, j, 0, i + 1, 0, j, 0, i + 1, 0, j + 1, 0, i, 0, j + 1, 0]
            idx += [v, v + 1, v + 2, 0, v, v + 2, v + 3, 0]
            v += 4
            q += 1
    b = oracle.build_array_bvh(np.array(pos, np.float32), np.array(idx, np.uint32))
    n = b.nodes
    depth, leaf_tris, max_leaf = 0, 0, 0
    stack = [(0, 0)]
    while stack:
        i, d = stack.pop()
        depth = max(depth, d)
        if (n[i, 7] >> 16) == 0xFFFF:
            c = int(n[i, 7] & 0xFFFF)
            leaf_tris += c
            max_leaf = max(max_leaf, c)
            continue
        stack += [(i + 1, d + 1), (i + int(n[i, 6]), d + 1)]
    assert leaf_tris == 2000 and max_leaf <= 4 and depth <= 16


def test_coincident_centroids_median_split():
    # buildArrayBvh.test.ts:208-238
    pos = np.array([0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0], np.float32)
    idx = np.tile(np.array([0, 1, 2, 0], np.uint32), 17)
    b = oracle.build_array_bvh(pos, idx, max_leaf=3)
    leaf = (b.nodes[:, 7] >> 16) == 0xFFFF
    counts = b.nodes[leaf, 7] & 0xFFFF
    assert counts.max() <= 3 and counts.sum() == 17
    assert list(b.reordered_to_source) == list(range(17))


def test_depth_cap_fails_instead_of_violating_leaf_cap():
    # buildArrayBvh.test.ts:240-256
    pos = np.zeros((24, 4), np.float32)
    pos[:, 0] = np.arange(24)
    idx = np.zeros((8, 4), np.uint32)
    idx[:, :3] = np.arange(24).reshape(8, 3)
    with pytest.raises(RuntimeError, match="maxDepth"):
        oracle.build_array_bvh(pos, idx, max_leaf=1, max_depth=1)


def random_mesh(n, seed):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-10, 10, (n, 3))
    v = (c[:, None, :] + rng.normal(0, 1.0, (n, 3, 3))).reshape(-1, 3)
    pos = np.zeros((3 * n, 4), np.float32)
    pos[:, :3] = v
    idx = np.zeros((n, 4), np.uint32)
    idx[:, :3] = np.arange(3 * n).reshape(n, 3)
    return pos, idx


def random_rays(n, seed, spread=15.0):
    rng = np.random.default_rng(seed)
    o = rng.uniform(-spread, spread, (n, 3)) * 2
    d = rng.uniform(-spread, spread, (n, 3)) - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = o
    r[:, 3] = 1e-4
    r[:, 4:7] = d
    r[:, 7] = np.inf
    return r


def test_wide_collapse_is_conservative_and_stack_safe():
    # compressedWideBvh.test.ts: stack proof and conservative quantisation
    pos, idx = random_mesh(3000, 3)
    w = oracle.build_compressed_wide_bvh(pos, idx)
    assert w.status == "wide"
    assert (w.child_count >= 1).all() and (w.child_count <= 8).all()
    nb = w.node_bounds.astype(np.float64)
    for node in range(w.node_count):
        for s in range(int(w.child_count[node])):
            kind, ref, cnt = w.child_meta[node, s]
            q = w.child_bounds[node, s].astype(np.float64)
            mn, mx = nb[node, :3], nb[node, 3:]
            ext = np.where(mx > mn, mx - mn, 0)
            lo = np.where(q[:3] <= 0, mn, np.where(q[:3] >= 65535, mx, mn + ext * q[:3] / 65535))
            hi = np.where(q[3:] <= 0, mn, np.where(q[3:] >= 65535, mx, mn + ext * q[3:] / 65535))
            if kind == 1:
                cb = w.node_bounds[ref].astype(np.float64)
                assert (lo <= cb[:3] + 1e-12).all() and (hi >= cb[3:] - 1e-12).all()


def test_first_hit_equals_brute_force():
    # compressedWideBvh.test.ts:395-433 (first hit vs brute force)
    pos, idx = random_mesh(500, 5)
    w = oracle.build_compressed_wide_bvh(pos, idx)
    rays = random_rays(400, 6)
    p, t, b, _ = oracle.first_hit(w, pos, rays)
    bp, bt, bb, _ = oracle.brute_first_hit(pos, idx, rays)
    assert (p >= 0).sum() > 50 and (p < 0).sum() > 50
    assert np.array_equal(p, bp)
    h = p >= 0
    assert np.allclose(t[h], bt[h], rtol=0, atol=0)


def test_tmin_tmax_exclusive():
    # cwbvhTMinParity.test.ts:31-67: a hit exactly at tMin or tMax is rejected
    pos = np.array([-1, -1, 5, 0, 1, -1, 5, 0, 0, 1, 5, 0], np.float32)
    idx = np.array([0, 1, 2, 0], np.uint32)
    w = oracle.build_compressed_wide_bvh(pos, idx)
    def ray(tmin, tmax):
        return np.array([[0, 0, 0, tmin, 0, 0, 1, tmax]], np.float32)
    assert oracle.first_hit(w, pos, ray(5, np.inf))[0][0] == -1
    p, t, _, _ = oracle.first_hit(w, pos, ray(5 - 1e-4, np.inf))
    assert p[0] == 0 and abs(t[0] - 5) < 1e-6
    assert oracle.first_hit(w, pos, ray(1e-5, 5))[0][0] == -1
    # watertight semantic agrees
    assert oracle.first_hit_watertight(w, pos, ray(5, np.inf))[0][0] == -1
    assert oracle.first_hit_watertight(w, pos, ray(1e-5, 5))[0][0] == -1
    assert oracle.first_hit_watertight(w, pos, ray(5 - 1e-4, np.inf))[0][0] == 0


# ---- watertight known answers: opticalWatertightTriangle.test.ts:35-140
WT = oracle.watertight_f32


def test_wt_planar_diagonal_exact_tie():
    a = WT([0, 0, 0], [0, 0, 1], [-1, -1, 1], [1, -1, 1], [1, 1, 1])
    b = WT([0, 0, 0], [0, 0, 1], [-1, -1, 1], [1, 1, 1], [-1, 1, 1])
    assert a["hit"] and b["hit"]
    assert np.float32(a["t"]).tobytes() == np.float32(b["t"]).tobytes() and a["t"] == 1.0
    assert a["zero_edge_mask"] != 0 and b["zero_edge_mask"] != 0
    assert a["side"] == -1 and b["side"] == -1


def test_wt_convex_edge_and_vertex_ties():
    ex = WT([2, 2, 0], [-1, -1, 0], [1, -1, -1], [1, 1, -1], [1, 1, 1])
    ey = WT([2, 2, 0], [-1, -1, 0], [-1, 1, -1], [1, 1, 1], [1, 1, -1])
    assert ex["hit"] and ey["hit"] and ex["t"] == ey["t"] == 1.0
    assert ex["side"] == 1 and ey["side"] == 1
    faces = [([1, -1, -1], [1, 1, -1], [1, 1, 1]), ([-1, 1, -1], [1, 1, 1], [1, 1, -1]),
             ([-1, -1, 1], [1, -1, 1], [1, 1, 1])]
    hits = [WT([2, 2, 2], [-1, -1, -1], *f) for f in faces]
    assert all(h["hit"] and h["zero_edge_mask"] >= 3 for h in hits)
    assert len({h["t"] for h in hits}) == 1 and {h["side"] for h in hits} == {1}


def test_wt_silhouette_tangency_sides():
    f = WT([2, 0, 0], [-1, 1, 0], [1, -1, -1], [1, 1, -1], [1, 1, 1])
    b = WT([2, 0, 0], [-1, 1, 0], [-1, 1, -1], [1, 1, 1], [1, 1, -1])
    assert (f["side"], b["side"]) == (1, -1) and f["t"] == b["t"] == 1.0


def test_wt_adjacent_f32_layers_are_distinct():
    outer_t = 1.0
    inner_t = float(np.nextafter(np.float32(1.0), np.float32(2.0)))
    o = WT([0, 0, 0], [0, 0, 1], [-1, -1, outer_t], [1, -1, outer_t], [0, 1, outer_t])
    i = WT([0, 0, 0], [0, 0, 1], [-1, -1, inner_t], [1, -1, inner_t], [0, 1, inner_t], o["t"])
    assert o["hit"] and i["hit"] and o["t"] == outer_t and i["t"] == inner_t


def test_wt_agrees_with_fp64_on_random_pairs():
    rng = np.random.default_rng(11)
    agree = hits = 0
    for _ in range(3000):
        o = rng.uniform(-3, 3, 3)
        tri = rng.uniform(-1, 1, (3, 3))
        d = tri.mean(0) + rng.normal(0, 0.3, 3) - o
        w = WT(o, d, *tri)
        h, t, _ = oracle.triangle_fp64(o, d, *tri)
        hits += h
        agree += (w["hit"] == h)
        if w["hit"] and h:
            assert abs(w["t"] - t) <= 1e-4 * t
    assert hits > 500 and agree == 3000


def test_differential_gate_leaf1_wide_equals_brute_force():
    # compressedWideBvhDifferential.test.ts:239-279 on the oracle: the leaf-1
    # 8-wide traversal answers exactly what brute force answers
    from differential_cases import differential_rays, random_mesh
    soup, centers, normals = random_mesh()
    rays = differential_rays(centers, normals)
    w = oracle.build_compressed_wide_bvh(soup.positions, soup.indices, max_leaf=1)
    prim, t, _ = oracle.first_hit(w, soup.positions, rays)[:3]
    bprim, bt = oracle.brute_first_hit(soup.positions, soup.indices, rays)[:2]
    assert np.array_equal(prim, bprim)
    assert np.allclose(t[prim >= 0], bt[prim >= 0], rtol=1e-12)
    hits = int((prim >= 0).sum())
    assert hits > 100 and len(rays) - hits > 100, hits
