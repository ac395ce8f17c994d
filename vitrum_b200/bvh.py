"""Mesh acceleration structure: the shared-bvh API surface on the B200 path.

Mirrors the reference's shared-bvh entry points (packages/shared-bvh/src):

    buildArrayBvh / buildCompressedWideBvh   -> build_compressed_wide_bvh()
    intersectCompressedWideBvhFirstHit       -> Bvh.intersect_first_hit()
    intersectCompressedWideBvhAnyHit         -> Bvh.intersect_any_hit()
    buildTlas (tlas.ts:859)                  -> build_tlas()
    validateBvhEncoding                      -> validate_bvh_encoding()

Options keep the reference names and defaults (BuildArrayBvhOpts,
buildArrayBvh.ts:277-318).  Invalid options raise ValueError (RangeError /
TypeError in the reference).  Everything runs through libvitrum_pt.so.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as N

# the reference's BuildArrayBvhOpts keys, plus traversalTree: the tree the queries traverse
# ("reference": the built tree, reference 8-wide grouping; "sah": the built tree, SAH-optimal
# grouping; "fast", the default: a second tree with <= 2 triangles per leaf, 32 bins, SAH-optimal
# grouping).  The exported binary tree and every hit are the same whichever is chosen.
_OPTION_KEYS = ("positionStride", "indexStride", "maxLeafTriangles", "binCount", "maxDepth", "traversalTree")
_TRAVERSAL = {None: 0, "reference": 1, "sah": 2, "fast": 3}


def _options(opts: dict) -> N.BuildOptions:
    for k in opts:
        if k not in _OPTION_KEYS:
            raise ValueError(f"unknown option {k!r}")
    if opts.get("traversalTree") not in _TRAVERSAL:
        raise ValueError("traversalTree must be 'reference', 'sah' or 'fast'")
    return N.BuildOptions(int(opts.get("positionStride", 4)), int(opts.get("indexStride", 4)),
                          int(opts.get("maxLeafTriangles", 4)), int(opts.get("binCount", 16)),
                          int(opts.get("maxDepth", 58)), _TRAVERSAL[opts.get("traversalTree")])


def _ptr(a) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


class Bvh:
    """Owning handle of a vt_bvh (device-resident 8-wide BVH)."""

    def __init__(self, handle: ctypes.c_void_p, device: int):
        self._h = handle
        self.device = device

    # ------------------------------------------------------------ lifecycle
    def close(self) -> None:
        if self._h:
            N.call("vt_bvh_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        if not self._h:
            raise RuntimeError("Bvh is disposed")
        return self._h

    # ---------------------------------------------------------------- info
    def info(self) -> dict:
        i = N.BvhInfo()
        N.call("vt_bvh_get_info", self.handle, ctypes.byref(i))
        return {f: getattr(i, f) for f, _ in N.BvhInfo._fields_}

    def validate(self) -> dict:
        """Structural proof of the device-resident 8-wide tree (vt_bvh_validate);
        raises VtError(VT_ERR_BUILD) on a violation."""
        p = N.WideProof()
        N.call("vt_bvh_validate", self.handle, ctypes.byref(p))
        return {f: getattr(p, f) for f, _ in N.WideProof._fields_}

    def export_binary(self):
        """(nodes (n, 8) uint32 in the reference layout, reordered_to_source uint32)."""
        inf = self.info()
        nodes = np.zeros((inf["binary_node_count"], 8), dtype=np.uint32)
        r2s = np.zeros(max(inf["triangle_count"], 1), dtype=np.uint32)
        N.call("vt_bvh_export_binary", self.handle, _ptr(nodes), nodes.size, _ptr(r2s), r2s.size)
        return nodes, r2s[: inf["triangle_count"]]

    def export_wide(self):
        """(node words uint32, 20 per 8-wide node; records float32, 16 per
        triangle record) of this backend's published encoding."""
        nw, nf = ctypes.c_size_t(), ctypes.c_size_t()
        N.call("vt_bvh_export_wide", self.handle, None, 0, None, 0, ctypes.byref(nw), ctypes.byref(nf))
        words = np.empty(nw.value, np.uint32)
        recs = np.empty(nf.value, np.float32)
        N.call("vt_bvh_export_wide", self.handle, _ptr(words), words.size, _ptr(recs), recs.size, ctypes.byref(nw),
               ctypes.byref(nf))
        return words, recs

    # ------------------------------------------------------------- queries
    def intersect_first_hit(self, rays: np.ndarray) -> np.ndarray:
        """Closest hit for host rays (n, 8) float32 -> structured (prim, t, u, v)."""
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        out = np.empty(rays.shape[0], dtype=HIT_DTYPE)
        N.call("vt_bvh_trace_closest", self.handle, _ptr(rays), rays.shape[0], _ptr(out))
        return out

    def intersect_any_hit(self, rays: np.ndarray) -> np.ndarray:
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        out = np.empty(rays.shape[0], dtype=np.uint8)
        N.call("vt_bvh_trace_any", self.handle, _ptr(rays), rays.shape[0], _ptr(out))
        return out.astype(bool)

    def set_trace_order(self, cell_bits: int) -> None:
        """Spatial trace order of batches of >= 65,536 rays: 2^cell_bits cells per
        axis (1..6), 0 = input order.  Results do not depend on it."""
        N.call("vt_bvh_set_trace_order", self.handle, int(cell_bits))

    def trace_closest_device(self, rays_ptr: int, n: int, hits_ptr: int, stream: int = 0) -> None:
        """Enqueue closest hit on device buffers (32-byte rays, 16-byte hits)."""
        N.call("vt_bvh_trace_closest_device", self.handle, ctypes.c_void_p(rays_ptr), n,
               ctypes.c_void_p(hits_ptr), ctypes.c_void_p(stream))

    def trace_any_device(self, rays_ptr: int, n: int, occluded_ptr: int, stream: int = 0) -> None:
        N.call("vt_bvh_trace_any_device", self.handle, ctypes.c_void_p(rays_ptr), n,
               ctypes.c_void_p(occluded_ptr), ctypes.c_void_p(stream))


HIT_DTYPE = np.dtype([("prim", np.int32), ("t", np.float32), ("u", np.float32), ("v", np.float32)])


def build_compressed_wide_bvh(positions, indices, device: int = 0, **opts) -> Bvh:
    """buildCompressedWideBvh(positions, indices, triMaterialIds, opts) on the GPU path.

    positions: float32 array (stride positionStride), indices: uint32 array
    (stride indexStride).  Host arrays are copied; the caller keeps them.
    """
    o = _options(opts)
    pos = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1)
    idx = np.ascontiguousarray(indices, dtype=np.uint32).reshape(-1)
    h = ctypes.c_void_p()
    N.call("vt_bvh_build", device, _ptr(pos), pos.size, _ptr(idx), idx.size, ctypes.byref(o), ctypes.byref(h))
    return Bvh(h, device)


def build_compressed_wide_bvh_device(positions_ptr: int, position_words: int, indices_ptr: int, index_words: int,
                                     device: int = 0, stream: int = 0, **opts) -> Bvh:
    o = _options(opts)
    h = ctypes.c_void_p()
    N.call("vt_bvh_build_device", device, ctypes.c_void_p(positions_ptr), position_words,
           ctypes.c_void_p(indices_ptr), index_words, ctypes.byref(o), ctypes.c_void_p(stream), ctypes.byref(h))
    return Bvh(h, device)


def watertight_eval_device(cases_ptr: int, n: int, out_ptr: int, device: int = 0, stream: int = 0) -> None:
    N.call("vt_watertight_eval_device", device, ctypes.c_void_p(cases_ptr), n, ctypes.c_void_p(out_ptr),
           ctypes.c_void_p(stream))


_TLAS_KEYS = ("maxLeafSize", "binCount", "maxDepth")


def build_tlas(aabbs, **opts):
    """buildTlas (shared-bvh/src/tlas.ts:859) over (n, 6) instance world AABBs
    (min xyz, max xyz; doubles).  Options keep the reference names
    (maxLeafSize 1, binCount 16, maxDepth 58).  Returns (nodes (m, 8) uint32 in
    the reference's 32-byte layout, instanceIndices uint32)."""
    for k in opts:
        if k not in _TLAS_KEYS:
            raise ValueError(f"unknown option {k!r}")
    a = np.ascontiguousarray(aabbs, dtype=np.float64).reshape(-1, 6)
    n = a.shape[0]
    count = ctypes.c_size_t(0)
    args = (int(opts.get("maxLeafSize", 1)), int(opts.get("binCount", 16)), int(opts.get("maxDepth", 58)))
    N.call("vt_tlas_build", _ptr(a), n, *args, None, 0, None, 0, ctypes.byref(count))
    nodes = np.zeros((count.value, 8), np.uint32)
    perm = np.zeros(n, np.uint32)
    N.call("vt_tlas_build", _ptr(a), n, *args, _ptr(nodes), nodes.size, _ptr(perm), n, ctypes.byref(count))
    return nodes, perm


def validate_bvh_encoding(node_words, total_nodes, roots=None, triangle_count=None, traversal_stack_capacity=None):
    """validateBvhEncoding (shared-bvh/src/validateBvhEncoding.ts:55): structural
    proof of a packed binary BVH (8 u32 words per node).  Returns the proof as
    a dict with the reference's keys; raises VtError(VT_ERR_BUILD) carrying the
    reference's message on a violation."""
    w = np.ascontiguousarray(np.asarray(node_words).view(np.uint32) if np.asarray(node_words).dtype == np.float32
                             else np.asarray(node_words, np.uint32)).reshape(-1)
    r = None if roots is None else np.ascontiguousarray(roots, np.uint32)
    p = N.BvhProof()
    N.call("vt_validate_bvh_encoding", _ptr(w) if w.size else None, w.size, int(total_nodes),
           _ptr(r) if r is not None and r.size else (ctypes.c_void_p(1) if r is not None else None),
           0 if r is None else r.size, -1 if triangle_count is None else int(triangle_count),
           0 if traversal_stack_capacity is None else int(traversal_stack_capacity), ctypes.byref(p))
    out = {"nodeCount": p.node_count, "rootCount": p.root_count, "interiorNodeCount": p.interior_node_count,
           "leafNodeCount": p.leaf_node_count, "maxDepth": p.max_depth,
           "maxTraversalStackEntries": p.max_traversal_stack_entries,
           "traversalStackCapacity": p.traversal_stack_capacity}
    if triangle_count is not None:
        out["triangleCount"] = p.triangle_count
    return out
