"""Two-level (TLAS over instances of per-mesh BLAS) scenes on the GPU.

The two-level traversal must answer exactly what a single-level query over the
same scene baked into world space answers: hit ids equal up to FP64 near-ties
and edge/grazing cases (oracle/parity.py), t within 1e-5 relative and
barycentrics within 1e-5.  The truth is the CPU oracle's FP64 query
(intersectCompressedWideBvhFirstHit, shared-bvh/src/compressedWideBvh.ts:754)
on the flattened geometry; the instance world AABBs follow transformAabb
(scenePack.ts:197-223) and the top level buildTlas (tlas.ts:859), whose node
bytes the oracle matches against the reference's golden fixture.
"""
import numpy as np
import pytest

import oracle
from oracle import parity
from vitrum_b200 import _native as N
from vitrum_b200 import scenes
from vitrum_b200.engine import Camera, Engine, Instance, Material, Mesh, PointLight, Scene

pytestmark = pytest.mark.gpu


def small_cloud(n=48, seed=5):
    return scenes.instanced_cloud(n_instances=n, seed=seed, n_points=4, sphere_levels=(1, 2), torus_segments=(24, 8),
                                  cube_cells=(3, 5), extent=4.0)


def cloud_rays(n, seed, extent=4.0):
    # origins on a sphere around the cloud, aimed at points inside it
    u = scenes.uniform(seed, 20, 5 * n).reshape(n, 5)
    z = 2 * u[:, 0] - 1
    ph = 2 * np.pi * u[:, 1]
    r = np.sqrt(1 - z * z)
    o = 2.5 * extent * np.stack([r * np.cos(ph), r * np.sin(ph), z], 1)
    tgt = (np.stack([u[:, 2], u[:, 3], u[:, 4]], 1) * 2 - 1) * extent
    d = tgt - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 3] = 1e-4
    rays[:, 4:7] = d
    rays[:, 7] = np.inf
    return rays


def flattened_soup(sc):
    flat = sc.flattened()
    pos, idx, _, _, _, _, _ = oracle.flatten_scene(flat)
    offs = np.cumsum([0] + [sc.meshes[i.mesh].indices.shape[0] for i in sc.instances])
    return flat, pos, idx, offs


def placed_fp64(sc, rays, inst, prim):
    """FP64 Moller-Trumbore t, u, v of each ray against its placed triangle,
    vertices carried to world space in double (no f32 rounding)."""
    n = inst.size
    V = np.zeros((n, 3, 3))
    for k in range(n):
        I = sc.instances[inst[k]]
        m = sc.meshes[I.mesh]
        M = np.asarray(I.local_to_world, np.float32).astype(np.float64).reshape(4, 4)
        loc = np.asarray(m.positions, np.float32).astype(np.float64)[np.asarray(m.indices)[prim[k]]]
        V[k] = loc @ M[:3, :3].T + M[:3, 3]
    o = rays[:, 0:3].astype(np.float64)
    d = rays[:, 4:7].astype(np.float64)
    a, b, c = V[:, 0], V[:, 1], V[:, 2]
    e1, e2 = b - a, c - a
    nrm = np.cross(e1, e2)
    det = -np.einsum("ij,ij->i", d, nrm)
    ao = o - a
    dao = np.cross(ao, d)
    u = np.einsum("ij,ij->i", e2, dao) / det
    v = -np.einsum("ij,ij->i", e1, dao) / det
    t = np.einsum("ij,ij->i", ao, nrm) / det
    return t, u, v


def test_instanced_trace_matches_flattened_oracle(cuda):
    sc, _ = small_cloud()
    flat, pos, idx, offs = flattened_soup(sc)
    rays = cloud_rays(40000, 9)
    e = Engine()
    e.set_scene(sc)
    hits, inst = e.trace_rays(rays)
    assert ((hits["prim"] < 0) == (inst < 0)).all()
    g = hits.copy()
    g["prim"] = np.where(inst >= 0, offs[np.maximum(inst, 0)] + hits["prim"], -1)
    wide = oracle.build_compressed_wide_bvh(pos, idx)
    ref = oracle.first_hit(wide, pos, rays)
    res = parity.classify(pos, idx, rays, g, ref, placed=True)
    print({k: v for k, v in res.items() if k != "error_rays"})
    assert res["hits"] > 10000
    assert res["error"] == 0, res["error_rays"][:5]
    assert res["edge"] <= 8, res
    # t and barycentrics against the placed triangle in FP64 (the flattened f32
    # soup above is only an approximation of the placed geometry)
    hit = np.nonzero(inst >= 0)[0]
    t, u, v = placed_fp64(sc, rays[hit], inst[hit], hits["prim"][hit])
    dt = np.abs(hits["t"][hit] - t) / t
    du = np.maximum(np.abs(hits["u"][hit] - u), np.abs(hits["v"][hit] - v))
    print(f"placed-triangle FP64: max t rel {dt.max():.2e}, max bary {du.max():.2e}")
    assert dt.max() <= parity.T_REL and du.max() <= parity.BARY_ABS
    e.dispose()


def test_instanced_and_flattened_engines_agree(cuda):
    # the same scene as instances and as world-space meshes: identical ids
    # except where the instance-space ray transform moves a near-tie or an edge
    sc, _ = small_cloud(seed=7)
    flat, pos, idx, offs = flattened_soup(sc)
    rays = cloud_rays(20000, 10)
    a, b = Engine(), Engine()
    a.set_scene(sc)
    b.set_scene(flat)
    ha, ia = a.trace_rays(rays)
    hb, ib = b.trace_rays(rays)
    assert (ib == -1).all()
    ga = np.where(ia >= 0, offs[np.maximum(ia, 0)] + ha["prim"], -1)
    same = ga == hb["prim"]
    assert same.mean() > 0.999, same.mean()
    both = same & (ga >= 0)
    assert np.allclose(ha["t"][both], hb["t"][both], rtol=1e-5, atol=0)
    a.dispose()
    b.dispose()


def test_instanced_render_matches_cpu_oracle(cuda):
    sc, cam = small_cloud(n=24, seed=11)
    cam = Camera(eye=(0.0, 2.0, 11.0), target=(0.0, 0.0, 0.0), fov_y_deg=50.0, near=0.01, far=100.0)
    W = H = 24
    n, B = 256, 4
    e = Engine(max_bounces=B, oracle_accumulation=True)
    e.set_scene(sc)
    e.render_frame(cam, W, H, samples=n)
    gm, gv = e.capture_moments()
    s, q = oracle.pt_render(sc.flattened(), cam, W, H, n, B)
    cm = s / n
    cv = np.maximum(q / n - cm * cm, 0) * n / (n - 1)
    z = np.abs(gm - cm) / (np.sqrt((gv + cv) / n) + 1e-9)
    identical = np.isclose(gm, cm, rtol=1e-4, atol=1e-6).mean()
    print(f"instanced gpu vs flattened cpu oracle: {identical:.3f} agree to 1e-4, max z {z.max():.2f}")
    assert (z > 4).sum() <= 3
    assert abs(gm.mean() / cm.mean() - 1) < 1e-2
    e.dispose()


def test_pick_returns_instance_index(cuda):
    p, t = scenes.box_mesh((-0.5, -0.5, -0.5), (0.5, 0.5, 0.5), 2)
    insts = []
    for k, x in enumerate((-3.0, 0.0, 3.0)):
        M = np.eye(4, dtype=np.float32)
        M[0, 3] = x
        insts.append(Instance(0, M, k))
    sc = Scene(meshes=[Mesh(p, t, 0)], materials=[Material(), Material(), Material()], instances=insts,
               point_lights=[PointLight((0, 5, 5), (10, 10, 10))])
    cam = Camera(eye=(0.0, 0.0, 6.0), target=(0.0, 0.0, 0.0), fov_y_deg=60.0)
    e = Engine(max_bounces=1, debug=True)
    e.set_scene(sc)
    e.render_frame(cam, 64, 64, samples=1)
    assert e.debug.pick_triangle(32.0, 32.0) == 1      # the middle instance
    assert e.debug.pick_primitive(32.0, 32.0) == 0     # ... of the scene's one mesh primitive
    assert e.debug.pick_triangle(2.0, 2.0) is None and e.debug.pick_primitive(2.0, 2.0) is None
    e.dispose()


def test_instance_validation(cuda):
    p, t = scenes.box_mesh((0, 0, 0), (1, 1, 1), 1)
    e = Engine()
    bad = [
        Scene(meshes=[Mesh(p, t, 0)], materials=[Material()], instances=[Instance(1, np.eye(4), 0)]),
        Scene(meshes=[Mesh(p, t, 0)], materials=[Material()], instances=[Instance(0, np.eye(4), 3)]),
        Scene(meshes=[Mesh(p, t, 0)], materials=[Material()], instances=[Instance(0, np.zeros((4, 4)), 0)]),
        Scene(meshes=[Mesh(p, t, 0)], materials=[Material(emission=(1, 1, 1))],
              instances=[Instance(0, np.eye(4), 0)]),
    ]
    for sc in bad:
        with pytest.raises(N.VtError):
            e.set_scene(sc)
    e.dispose()


def test_full_instanced_cloud_renders(cuda):
    # the 1024-instance workload: 8 prototypes, 399,616 distinct and
    # 50,961,408 instanced triangles
    sc, cam = scenes.instanced_cloud()
    e = Engine(max_bounces=8)
    e.set_scene(sc)
    e.render_frame(cam, 192, 108, samples=2)
    img = e.capture_frame()
    assert np.isfinite(img).all() and img[..., :3].mean() > 0
    rays = cloud_rays(1 << 16, 12, extent=20.0)
    hits, inst = e.trace_rays(rays)
    assert (inst >= 0).sum() > 1000 and ((hits["prim"] < 0) == (inst < 0)).all()
    e.dispose()


def _golden_engine_scene(name):
    from test_oracle_golden import GOLDEN, SCENES
    import json
    from vitrum_b200.engine import Instance, Material, Mesh, Scene
    pk = json.load(open(GOLDEN))[name]
    prims = SCENES[name]
    roots = [bd["blasRoot"] for bd in pk["primitiveTlasBindings"]]
    meshes = []
    for P in prims:
        from test_oracle_golden import pack
        pos, idx = pack(P)
        meshes.append(Mesh(pos[:, :3].copy(), idx[:, :3].copy(), 0))
    l2w = np.array(pk["tlasInstanceLocalToWorld"], np.float32).reshape(-1, 4, 4)
    insts = [Instance(roots.index(r), l2w[i].T.copy(), 0) for i, r in enumerate(pk["tlasBlasRoots"])]
    return Scene(meshes=meshes, materials=[Material()], instances=insts), pk


@pytest.mark.parametrize("name", ["multiMesh", "resizeSplice"])
def test_engine_tlas_matches_reference_golden(cuda, name):
    """The engine's own top level (packSceneFromCore, scenePack.ts:1104-1310):
    node words and instance order byte-equal to the reference's golden pack."""
    sc, pk = _golden_engine_scene(name)
    e = Engine()
    e.set_scene(sc)
    nodes, perm = e.export_tlas()
    e.dispose()
    assert nodes.shape[0] == pk["tlasNodeCount"]
    assert np.array_equal(nodes, np.array(pk["tlasNodes"], np.uint32).reshape(-1, 8))
    assert np.array_equal(perm, np.array(pk["tlasInstanceIndices"], np.uint32))


def _world_aabbs(sc):
    """transformAabb (scenePack.ts:197-223) of each placed mesh's local box, in FP64."""
    out = []
    for inst in sc.instances:
        P = np.asarray(sc.meshes[inst.mesh].positions, np.float32).reshape(-1, 3).astype(np.float64)
        lo, hi = P.min(0), P.max(0)
        M = np.asarray(inst.local_to_world, np.float32).astype(np.float64).reshape(4, 4)
        mn, mx = np.full(3, np.inf), np.full(3, -np.inf)
        for c in range(8):
            q = [(hi if c & 1 else lo)[0], (hi if c & 2 else lo)[1], (hi if c & 4 else lo)[2]]
            for k in range(3):
                v = M[k, 0] * q[0] + M[k, 1] * q[1] + M[k, 2] * q[2] + M[k, 3]
                mn[k], mx[k] = min(mn[k], v), max(mx[k], v)
        out.append(np.r_[mn, mx])
    return np.array(out)


def test_engine_tlas_matches_oracle_on_cloud(cuda):
    """48- and 1024-instance clouds: the engine's top level byte-equal to the
    oracle's buildTlas over the same world boxes, before and after a rebuild
    over moved instances."""
    for sc in (small_cloud()[0], scenes.instanced_cloud()[0]):
        e = Engine()
        e.set_scene(sc)
        nodes, perm = e.export_tlas()
        on, op = oracle.build_tlas(_world_aabbs(sc))
        assert np.array_equal(nodes, on) and np.array_equal(perm, op)
        from test_gpu_instance_update import moved
        mv = moved(sc.instances, 3)
        e.update_instances(mv, rebuild=True)
        nodes, perm = e.export_tlas()
        e.dispose()
        import dataclasses
        on, op = oracle.build_tlas(_world_aabbs(dataclasses.replace(sc, instances=mv)))
        assert np.array_equal(nodes, on) and np.array_equal(perm, op)
