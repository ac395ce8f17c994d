"""Closest-hit parity classification -- TEST INFRASTRUCTURE ONLY.

Compares device closest-hit records with the oracle's FP64 query
(intersectCompressedWideBvhFirstHit, shared-bvh/src/compressedWideBvh.ts:754)
and sorts every disagreement into:

  tie      the two nearest FP64 hits of the ray (over ALL triangles) lie within
           `tie_rel` relative t of each other: either answer is correct
           (the exemption the acceptance criterion states);
  edge     the ray passes within the derived edge bound of an edge of one of
           the two triangles in dispute, or meets it at or below the
           reference's grazing cut-off: the reference's FP64 test accepts
           barycentrics down to -1e-6 and rejects |det| / (|n||d|) <= 1e-7
           (compressedWideBvh.ts:600-612), while the device decides with the
           watertight f32 test (opticalWatertightTriangle.ts:98), whose edge
           functions carry f32 rounding.  The bound per ray/triangle pair is
               1e-6 + 8 * 2^-24 / g            (single-level trees)
           with g = |det| / (|n||d|) the pair's conditioning: the reference's
           signed tolerance plus eight f32 ulps of the unit barycentric,
           amplified by 1/g as the shear divides by the ray-normal cosine.
           Instanced scenes add the f32 rounding of the placement,
               16 * 2^-24 * R / h,
           R the largest world coordinate of the triangle, h its smallest
           altitude (the flattened soup and the instance-space ray each round
           world coordinates once).  Counted, reported, and bounded by the
           tests that call this;
  error    anything else -- must be zero.

Agreement of t and barycentrics is checked on rays whose ids match:
|dt| <= t_rel * t and |du|, |dv| <= bary_abs (barycentrics sum to one, so the
tolerance is relative to that sum).
"""
from __future__ import annotations

import numpy as np

from . import brute_first_hit, triangle_fp64

T_REL = 1e-5
BARY_ABS = 1e-5
TIE_REL = 1e-6
REF_BARY_TOL = 1e-6      # compressedWideBvh.ts:600-612, signed
REF_GRAZE = 1e-7         # compressedWideBvh.ts:590, |det| / (|n||d|) <= 1e-7 rejects
F32_ULP = 2.0 ** -24


def edge_bound(g, placed=None):
    """Derived edge margin of one ray/triangle pair (module docstring)."""
    eps = REF_BARY_TOL + 8 * F32_ULP / max(g, REF_GRAZE)
    if placed is not None:
        eps += 16 * F32_ULP * placed
    return eps


def placement_ratio(a, b, c):
    """R / h of a placed triangle: largest |world coordinate| over its smallest altitude."""
    a = np.asarray(a, np.float64); b = np.asarray(b, np.float64); c = np.asarray(c, np.float64)
    area2 = np.linalg.norm(np.cross(b - a, c - a))
    longest = max(np.linalg.norm(b - a), np.linalg.norm(c - b), np.linalg.norm(a - c))
    if not (area2 > 0):
        return np.inf
    return float(max(np.abs(a).max(), np.abs(b).max(), np.abs(c).max()) / (area2 / longest))


def _tri(soup_pos, soup_idx, prim):
    iv = soup_idx[prim, :3]
    return soup_pos[iv[0], :3], soup_pos[iv[1], :3], soup_pos[iv[2], :3]


def _fp64_margin(o, d, a, b, c):
    """Signed FP64 barycentric margin min(w, u, v) and the grazing ratio."""
    o = np.asarray(o, np.float64); d = np.asarray(d, np.float64)
    a = np.asarray(a, np.float64); b = np.asarray(b, np.float64); c = np.asarray(c, np.float64)
    e1, e2 = b - a, c - a
    n = np.cross(e1, e2)
    det = -np.dot(d, n)
    if det == 0 or not np.isfinite(det):
        return -np.inf, 0.0
    ao = o - a
    dao = np.cross(ao, d)
    u = np.dot(e2, dao) / det
    v = -np.dot(e1, dao) / det
    w = 1 - u - v
    graze = abs(det) / (np.linalg.norm(n) * np.linalg.norm(d))
    return min(u, v, w), graze


def classify(positions, indices, rays, gpu, ref, tie_rel=TIE_REL, placed=False, t_rel=T_REL,
             bary_abs=BARY_ABS, max_detail=20):
    """gpu: structured array (prim, t, u, v); ref: (prim, t, bary(n,2)) from oracle.first_hit.
    placed: the soup is a flattened instanced scene (adds the placement term to the edge bound)."""
    pos = np.asarray(positions, np.float32).reshape(-1, 4)
    idx = np.asarray(indices, np.uint32).reshape(-1, 4)
    rays = np.asarray(rays, np.float32).reshape(-1, 8)
    rp, rt, rb = ref[0], ref[1], ref[2]
    gp = gpu["prim"]
    mism = np.nonzero(gp != rp)[0]
    out = dict(n=int(rays.shape[0]), hits=int((rp >= 0).sum()), mismatches=int(mism.size), tie=0, edge=0,
               error=0, error_rays=[], edge_margin_max=0.0)
    for i in mism:
        ray = rays[i:i + 1]
        _, t1, _, t2 = brute_first_hit(pos, idx, ray)
        t1, t2 = float(t1[0]), float(t2[0])
        if np.isfinite(t1) and np.isfinite(t2) and (t2 - t1) <= tie_rel * t1:
            out["tie"] += 1
            continue
        o, d = ray[0, 0:3], ray[0, 4:7]
        edge = False
        for p in (int(gp[i]), int(rp[i])):
            if p < 0:
                continue
            tri = _tri(pos, idx, p)
            m, g = _fp64_margin(o, d, *tri)
            bound = edge_bound(g, placement_ratio(*tri) if placed else None)
            if g <= REF_GRAZE * (1 + 1e-9) or abs(m) <= bound:
                edge = True
                if np.isfinite(m):
                    out["edge_margin_max"] = max(out["edge_margin_max"], float(abs(m)))
        if edge:
            out["edge"] += 1
        else:
            out["error"] += 1
            if len(out["error_rays"]) < max_detail:
                out["error_rays"].append(int(i))
    same = (gp == rp) & (rp >= 0)
    if same.any():
        dt = np.abs(gpu["t"][same].astype(np.float64) - rt[same]) / np.abs(rt[same])
        du = np.abs(gpu["u"][same].astype(np.float64) - rb[same, 0])
        dv = np.abs(gpu["v"][same].astype(np.float64) - rb[same, 1])
        out["t_max_rel"] = float(dt.max())
        out["bary_max_abs"] = float(max(du.max(), dv.max()))
        out["t_bad"] = int((dt > t_rel).sum())
        out["bary_bad"] = int(((du > bary_abs) | (dv > bary_abs)).sum())
    else:
        out["t_max_rel"] = 0.0
        out["bary_max_abs"] = 0.0
        out["t_bad"] = 0
        out["bary_bad"] = 0
    miss_ok = (gp < 0) & (rp < 0)
    out["miss_both"] = int(miss_ok.sum())
    return out


def triangle_check(o, d, a, b, c, tmin=0.0):
    """FP64 reference test of one ray/triangle pair (compressedWideBvh.ts:551)."""
    return triangle_fp64(o, d, a, b, c, tmin)


def watertight_disagreements(positions, indices, rays, gpu_prim, wt_prim):
    """Rays where the device and the f32 watertight oracle chose different
    triangles, split into exact f32 t ties (either order is correct) and
    real disagreements.  Returns (ties, errors) as lists of ray indices."""
    from . import watertight_f32
    pos = np.asarray(positions, np.float32).reshape(-1, 4)
    idx = np.asarray(indices, np.uint32).reshape(-1, 4)
    rays = np.asarray(rays, np.float32).reshape(-1, 8)
    ties, errors = [], []
    for i in np.nonzero(gpu_prim != wt_prim)[0]:
        r = rays[i]
        res = []
        for p in (int(gpu_prim[i]), int(wt_prim[i])):
            if p < 0:
                res.append(None)
                continue
            res.append(watertight_f32(r[0:3], r[4:7], *_tri(pos, idx, p), float(r[3])))
        if all(x is not None and x["hit"] for x in res) and \
                np.float32(res[0]["t"]).tobytes() == np.float32(res[1]["t"]).tobytes():
            ties.append(int(i))
        else:
            errors.append(int(i))
    return ties, errors
