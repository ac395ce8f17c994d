"""Neural radiance cache restated in numpy -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's baseline leg use this
module, as the checker of the CUDA kernels in vitrum_b200/csrc/nrc_kernels.cu;
nothing in the product imports it.

Follows the reference NRC of packages/walkaround-hybrid/src/neural/nrc/:
  spatial hash            nrcEncoding.ts:107-115 (primes 1, 2654435761, 805459861)
  level resolution        nrcEncoding.ts:117-119 (floor(Nmin * b^l))
  trilinear corners       nrcEncoding.ts:132-160
  normalise to the AABB   nrcEncoding.ts:163-178
  hash-grid forward       nrcEncoding.ts:185-203
  hash-grid backward      nrcEncoding.ts:214-236 (collisions accumulate)
  relative-L2 luminance   wgsl/fusedMlp.wgsl.ts:62-125 (stop-gradient denominator,
                          epsilon 1e-2, delta clamp 65504, NaN -> 0)
  Adam                    fusedMlpTrainer.ts:30-80 (non-finite guards, +-65504 clamp)
The network layout (64 inputs: 32 hash features, degree-4 real SH of the
direction, normal, roughness, diffuse and specular albedo, a constant 1; five
64-wide ReLU layers; 3 linear outputs) is the one the CUDA path implements.
With ``fp16=True`` the activations, inputs and backward deltas are rounded to
binary16 where the device stores them in fp16; products are summed in float64
(the device sums in fp32), so agreement is to fp16 rounding, not bit-exact.
"""
from __future__ import annotations

import numpy as np

P2 = 2654435761
P3 = 805459861
LUM = (0.299, 0.587, 0.114)
EPS = 1e-2
MAX_DELTA = 65504.0
WIDTH = 64
LAYERS = 6


def spatial_hash(ix, iy, iz, table_size):
    """(ix * 1) ^ (iy * P2) ^ (iz * P3) in uint32 arithmetic, modulo table_size."""
    m = np.uint64(0xFFFFFFFF)
    ix = np.asarray(ix, np.int64).astype(np.uint64) & m
    iy = np.asarray(iy, np.int64).astype(np.uint64) & m
    iz = np.asarray(iz, np.int64).astype(np.uint64) & m
    h = ix ^ ((iy * np.uint64(P2)) & m) ^ ((iz * np.uint64(P3)) & m)
    return (h % np.uint64(table_size)).astype(np.int64)


def level_resolutions(base, growth, levels):
    return np.array([np.floor(base * growth ** l) for l in range(levels)], np.float64)


def normalise(pos, aabb_min, aabb_max):
    """The device's f32 form of normalizeToAabb: clamp((p - min) * (1 / ext), 0, 1)."""
    pos = np.asarray(pos, np.float32)
    mn = np.asarray(aabb_min, np.float32)
    ext = np.asarray(aabb_max, np.float32) - mn
    inv = np.where(ext > 1e-20, np.float32(1.0) / np.where(ext > 1e-20, ext, 1), 0).astype(np.float32)
    return np.clip((pos - mn) * inv, 0, 1).astype(np.float32)


def trilinear(n01, resolution, table_size):
    """Rows (n, 8) and weights (n, 8) of the 8 corners (corner c: bit0 x, bit1 y, bit2 z)."""
    p = (n01.astype(np.float32) * np.float32(resolution)).astype(np.float32)
    x0 = np.floor(p)
    f = (p - x0).astype(np.float32)
    i0 = x0.astype(np.int64)
    rows = np.empty((n01.shape[0], 8), np.int64)
    wts = np.empty((n01.shape[0], 8), np.float64)
    for c in range(8):
        cx, cy, cz = c & 1, (c >> 1) & 1, (c >> 2) & 1
        wx = f[:, 0] if cx else 1 - f[:, 0]
        wy = f[:, 1] if cy else 1 - f[:, 1]
        wz = f[:, 2] if cz else 1 - f[:, 2]
        wts[:, c] = wx.astype(np.float64) * wy * wz
        rows[:, c] = spatial_hash(i0[:, 0] + cx, i0[:, 1] + cy, i0[:, 2] + cz, table_size)
    return rows, wts


def hash_grid_forward(table, n01, res):
    """table (levels, T, 2) -> features (n, 2 * levels)."""
    levels, T, _ = table.shape
    out = np.zeros((n01.shape[0], 2 * levels))
    for l in range(levels):
        rows, w = trilinear(n01, res[l], T)
        out[:, 2 * l:2 * l + 2] = np.einsum("nc,ncf->nf", w, table[l][rows].astype(np.float64))
    return out


def hash_grid_backward(dfeat, n01, res, table_shape):
    """Scatter d(loss)/d(features) (n, 2 * levels) into a table-shaped gradient."""
    levels, T, F = table_shape
    g = np.zeros(table_shape)
    for l in range(levels):
        rows, w = trilinear(n01, res[l], T)
        for c in range(8):
            np.add.at(g[l], rows[:, c], w[:, c:c + 1] * dfeat[:, 2 * l:2 * l + 2])
    return g


def sh4(d):
    """Real spherical harmonics, bands 0..3 (16 values), of unit directions (n, 3)."""
    x, y, z = d[:, 0].astype(np.float64), d[:, 1].astype(np.float64), d[:, 2].astype(np.float64)
    xx, yy, zz = x * x, y * y, z * z
    return np.stack([
        np.full_like(x, 0.28209479177387814),
        -0.48860251190291987 * y, 0.48860251190291987 * z, -0.48860251190291987 * x,
        1.0925484305920792 * x * y, -1.0925484305920792 * y * z, 0.94617469575755997 * zz - 0.31539156525251999,
        -1.0925484305920792 * x * z, 0.54627421529603959 * (xx - yy),
        -0.59004358992664352 * y * (3 * xx - yy), 2.8906114426405538 * x * y * z,
        0.45704579946446572 * y * (1 - 5 * zz), 0.3731763325901154 * z * (5 * zz - 3),
        0.45704579946446572 * x * (1 - 5 * zz), 1.4453057213202769 * z * (xx - yy),
        0.59004358992664352 * x * (3 * yy - xx)], 1)


def f16(a):
    return np.asarray(a, np.float64).astype(np.float16).astype(np.float64)


def encode(records, table, res, aabb_min, aabb_max, fp16=True):
    """records (n, 16) -> (inputs (n, 64), normalised positions (n, 3))."""
    r = np.asarray(records, np.float32).reshape(-1, 16)
    n01 = normalise(r[:, 0:3], aabb_min, aabb_max)
    levels = table.shape[0]
    X = np.zeros((r.shape[0], WIDTH))
    X[:, 0:2 * levels] = hash_grid_forward(table, n01, res)
    X[:, 32:48] = sh4(r[:, 3:6])
    X[:, 48:58] = r[:, 6:16]
    X[:, 58] = 1.0
    return (f16(X) if fp16 else X), n01


def forward(W, X, fp16=True):
    """W (6, 64 out, 64 in) -> (layer inputs [X, H1..H5], prediction (n, 3))."""
    Wd = f16(W) if fp16 else np.asarray(W, np.float64)
    acts = [X]
    h = X
    for l in range(LAYERS - 1):
        h = np.maximum(h @ Wd[l].T, 0.0)
        if fp16:
            h = f16(h)
        acts.append(h)
    pred = h @ Wd[LAYERS - 1][:3].T
    return acts, pred


def rel_l2_luminance(pred):
    s = np.max(np.abs(pred), axis=1)
    nl = (LUM[0] * pred[:, 0] + LUM[1] * pred[:, 1] + LUM[2] * pred[:, 2]) / np.where(s > 0, s, 1)
    return np.where(s > 0, np.clip(nl, -1, 1) * s, 0.0)


def output_gradient(pred, target, num_samples):
    """nrcRelativeL2OutputGradient: d(mean loss)/d(pred), (n, 3); and the mean loss."""
    pred = np.asarray(pred, np.float64)
    target = np.asarray(target, np.float64)
    ok = np.isfinite(pred).all(1) & np.isfinite(target).all(1)
    lum = np.minimum(np.abs(rel_l2_luminance(np.where(ok[:, None], pred, 0))), 1e19)
    den = lum * lum + EPS
    with np.errstate(over="ignore", invalid="ignore"):
        raw = (pred - target) * (2.0 / num_samples / 3.0 / den)[:, None]
    raw = np.where(np.isnan(raw), 0.0, raw)
    g = np.where(ok[:, None], np.clip(raw, -MAX_DELTA, MAX_DELTA), 0.0)
    with np.errstate(over="ignore", invalid="ignore"):
        loss = np.where(ok, ((pred - target) ** 2).sum(1) / den / 3.0, 0.0).sum() / num_samples
    return g, loss


def backward(W, acts, gout, fp16=True):
    """Gradients of the mean loss: dW (6, 64, 64) and d(inputs) (n, 64).

    gout = d(mean loss)/d(pred).  With fp16 the per-sample deltas are carried
    as N * delta rounded to binary16 (the device's loss scaling by the batch
    size), and unscaled in float64."""
    n = gout.shape[0]
    Wd = f16(W) if fp16 else np.asarray(W, np.float64)
    scale = float(n) if fp16 else 1.0
    G = np.zeros((n, WIDTH))
    G[:, :3] = gout * scale
    if fp16:
        G = f16(np.clip(G, -MAX_DELTA, MAX_DELTA))
    dW = np.zeros((LAYERS, WIDTH, WIDTH))
    for l in range(LAYERS - 1, -1, -1):
        dW[l] = G.T @ acts[l] / scale
        dX = G @ Wd[l]
        if l == 0:
            return dW, dX / scale
        G = np.where(acts[l] > 0, dX, 0.0)
        if fp16:
            G = f16(np.clip(G, -MAX_DELTA, MAX_DELTA))
    raise AssertionError("unreachable")


def gradients(W, table, samples, res, aabb_min, aabb_max, fp16=True):
    """(dW, d_table, loss) of the mean relative-L2 loss over samples (n, 20)."""
    s = np.asarray(samples, np.float32).reshape(-1, 20)
    X, n01 = encode(s[:, :16], table, res, aabb_min, aabb_max, fp16)
    acts, pred = forward(W, X, fp16)
    g, loss = output_gradient(pred, s[:, 16:19], s.shape[0])
    dW, dX = backward(W, acts, g, fp16)
    dT = hash_grid_backward(dX[:, :2 * table.shape[0]], n01, res, table.shape)
    return dW, dT, loss


def adam(param, m, v, g, lr, t, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam step with the reference's guards (returns new param, m, v)."""
    param, m, v, g = (np.asarray(a, np.float64) for a in (param, m, v, g))
    mi = beta1 * m + (1 - beta1) * g
    vi = beta2 * v + (1 - beta2) * g * g
    up = param - lr * (mi / (1 - beta1 ** t)) / (np.sqrt(vi / (1 - beta2 ** t)) + eps)
    ok = np.isfinite(g) & np.isfinite(up)
    return (np.where(ok, np.clip(up, -65504, 65504), param), np.where(ok, mi, m), np.where(ok, vi, v))
