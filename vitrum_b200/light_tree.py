"""The light tree next-event estimation selects emitters with: the reference's
buildLightTree + packLightTreeForGPU (shared-samplers/src/lightTree.ts:492, 611)
through vt_light_tree_build, and the device selection (samplePackedLightTreeCPU,
:1237) through vt_light_tree_select_device.  The engine builds its own tree
over a scene's light entries; these calls expose the same code for tests and
for hosts that want the packed tree."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as N

FLOATS_PER_NODE = 16
BUCKETS = 1 << 24


def build_light_tree(powers, centroids, aabbs, cones=None) -> np.ndarray:
    """(nodes, 16) float32 packed tree.  aabbs (n, 6) min|max; cones (n, 6):
    axis xyz, thetaO, thetaE, oriented flag (None: every emitter full-sphere)."""
    pw = np.asarray(powers, np.float64).reshape(-1)
    n = pw.size
    c = np.asarray(centroids, np.float64).reshape(n, 3)
    b = np.asarray(aabbs, np.float64).reshape(n, 6)
    k = np.zeros((n, 6)) if cones is None else np.asarray(cones, np.float64).reshape(n, 6)
    em = (N.LightTreeEmitter * max(n, 1))()
    for i in range(n):
        e = em[i]
        e.power = float(pw[i])
        for j in range(3):
            e.centroid[j] = float(c[i, j])
            e.aabb_min[j] = float(b[i, j])
            e.aabb_max[j] = float(b[i, 3 + j])
            e.cone_axis[j] = float(k[i, j])
        e.cone_theta_o = float(k[i, 3])
        e.cone_theta_e = float(k[i, 4])
        e.oriented = int(k[i, 5] != 0)
    count = ctypes.c_size_t(0)
    N.call("vt_light_tree_build", ctypes.cast(em, ctypes.c_void_p), n, None, 0, ctypes.byref(count))
    out = np.zeros((count.value, FLOATS_PER_NODE), np.float32)
    N.call("vt_light_tree_build", ctypes.cast(em, ctypes.c_void_p), n, ctypes.c_void_p(out.ctypes.data), out.size,
           ctypes.byref(count))
    return out


def select_device(tree, points, buckets, n_distant=0, normals=None, device=0):
    """Device selection for each point (n, 3), receiver normal (n, 3; None:
    none) and 24-bit draw over the tree's leaves plus `n_distant` distant
    entries: (entry uint32, pmf float32) arrays."""
    import torch
    dev = torch.device("cuda", device)
    tree = np.zeros((0, FLOATS_PER_NODE), np.float32) if tree is None else tree
    t = torch.from_numpy(np.ascontiguousarray(tree, np.float32).reshape(-1, FLOATS_PER_NODE)).to(dev)
    p = torch.from_numpy(np.ascontiguousarray(points, np.float32).reshape(-1, 3)).to(dev)
    b = torch.from_numpy(np.ascontiguousarray(buckets, np.uint32).view(np.int32)).to(dev)
    n = p.shape[0]
    nr = None
    if normals is not None:
        nr = torch.from_numpy(np.ascontiguousarray(normals, np.float32).reshape(-1, 3)).to(dev)
        if nr.shape[0] != n:
            raise ValueError("normals and points differ in length")
    e = torch.empty(n, dtype=torch.int32, device=dev)
    pmf = torch.empty(n, dtype=torch.float32, device=dev)
    s = torch.cuda.current_stream(dev)
    N.call("vt_light_tree_select_device", ctypes.c_void_p(t.data_ptr()) if t.shape[0] else None, t.shape[0],
           int(n_distant), ctypes.c_void_p(p.data_ptr()),
           ctypes.c_void_p(nr.data_ptr()) if nr is not None else None, ctypes.c_void_p(b.data_ptr()), n, ctypes.c_void_p(e.data_ptr()), ctypes.c_void_p(pmf.data_ptr()),
           ctypes.c_void_p(s.cuda_stream))
    torch.cuda.synchronize(dev)
    return e.cpu().numpy().view(np.uint32), pmf.cpu().numpy()
