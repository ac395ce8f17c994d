"""Closest-hit parity classification -- TEST INFRASTRUCTURE ONLY.

Compares device closest-hit records with the oracle's FP64 query
(intersectCompressedWideBvhFirstHit, shared-bvh/src/compressedWideBvh.ts:754)
and sorts every disagreement into:

  tie      the two nearest FP64 hits of the ray (over ALL triangles) lie within
           `tie_rel` relative t of each other: either answer is correct
           (the exemption the acceptance criterion states);
  edge     the ray passes within `edge_eps` barycentric units of an edge of
           one of the two triangles in dispute, or hits it at a grazing angle
           (|det| / (|n||d|) below 1e-6): the reference FP64 test (with its
           signed 1e-6 tolerance) and the watertight f32 test may legitimately
           decide differently there; counted and reported separately;
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
EDGE_EPS = 1e-3


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


def classify(positions, indices, rays, gpu, ref, tie_rel=TIE_REL, edge_eps=EDGE_EPS, t_rel=T_REL,
             bary_abs=BARY_ABS, max_detail=20):
    """gpu: structured array (prim, t, u, v); ref: (prim, t, bary(n,2)) from oracle.first_hit."""
    pos = np.asarray(positions, np.float32).reshape(-1, 4)
    idx = np.asarray(indices, np.uint32).reshape(-1, 4)
    rays = np.asarray(rays, np.float32).reshape(-1, 8)
    rp, rt, rb = ref[0], ref[1], ref[2]
    gp = gpu["prim"]
    mism = np.nonzero(gp != rp)[0]
    out = dict(n=int(rays.shape[0]), hits=int((rp >= 0).sum()), mismatches=int(mism.size), tie=0, edge=0,
               error=0, error_rays=[])
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
            m, g = _fp64_margin(o, d, *_tri(pos, idx, p))
            if abs(m) <= edge_eps or g <= 1e-6:
                edge = True
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
