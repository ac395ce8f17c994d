"""Neural radiance cache kernels (tcgen05 MLP, hash grid, Adam) against the
numpy oracle (oracle/nrc.py): forward, gradients, optimiser step, learning.

Tolerances: the device stores inputs, activations and backward deltas in fp16
and accumulates in fp32; the oracle rounds at the same places and sums in
float64.  Predictions agree to 1e-2 of their scale; gradients to 3e-2 in
relative Frobenius norm per layer and over the table.
"""
import dataclasses

import numpy as np
import pytest

from oracle import nrc as O
from vitrum_b200 import _native as N
from vitrum_b200.nrc import NrcConfig, RadianceCache

pytestmark = pytest.mark.gpu


def random_records(n, seed, box=((0, 0, 0), (1, 1, 1))):
    rng = np.random.default_rng(seed)
    mn, mx = np.array(box[0], np.float64), np.array(box[1], np.float64)
    r = np.zeros((n, 16), np.float32)
    r[:, 0:3] = mn + rng.random((n, 3)) * (mx - mn)
    d = rng.standard_normal((n, 3))
    r[:, 3:6] = d / np.linalg.norm(d, axis=1, keepdims=True)
    nn = rng.standard_normal((n, 3))
    r[:, 6:9] = nn / np.linalg.norm(nn, axis=1, keepdims=True)
    r[:, 9] = rng.random(n)
    r[:, 10:16] = rng.random((n, 6))
    return r


def randomise(cache, seed, w_scale=0.25, t_scale=0.5):
    rng = np.random.default_rng(seed)
    cfg = cache.config
    W = (rng.standard_normal((6, 64, 64)) * w_scale).astype(np.float32)
    W[5, 3:] = 0
    T = (rng.standard_normal((cfg.levels, 1 << cfg.log2_table_size, 2)) * t_scale).astype(np.float32)
    cache.set_params(W, T)
    return W, T


def oracle_pred(cfg, W, T, recs):
    res = O.level_resolutions(cfg.base_resolution, cfg.growth, cfg.levels)
    X, _ = O.encode(recs, O.f16(T), res, cfg.aabb_min, cfg.aabb_max)
    _, pred = O.forward(W, X)
    return pred


@pytest.mark.parametrize("n", [1, 127, 128, 1000, 40000])
def test_query_matches_oracle(cuda, n):
    cfg = NrcConfig(levels=8, log2_table_size=12, base_resolution=4, growth=1.6)
    c = RadianceCache(cfg)
    W, T = randomise(c, 7)
    recs = random_records(n, 11)
    got = c.query(recs)
    want = oracle_pred(cfg, W, T, recs)
    scale = np.abs(want).max() + 1e-3
    err = np.abs(got - want).max() / scale
    print(f"n={n}: max |gpu - oracle| / scale = {err:.2e}")
    assert err < 1e-2
    c.close()


@pytest.mark.parametrize("n", [1, 129, 385, 40000, 300000])
def test_query_tiles_per_cta_agree(cuda, n):
    """The MLP tile knob (query tiles of 128 in flight per inference CTA, one per
    warpgroup, 1..4) changes only the launch shape: every query's prediction is
    the same bit for bit, and matches the oracle, at tile counts that leave
    warpgroups without a tile."""
    cfg = NrcConfig(levels=8, log2_table_size=12, base_resolution=4, growth=1.6)
    recs = random_records(n, 21)
    outs = []
    for tiles in (1, 2, 3, 4):
        c = RadianceCache(dataclasses.replace(cfg, infer_tiles=tiles))
        W, T = randomise(c, 7)
        outs.append(c.query(recs))
        c.close()
    assert all(np.array_equal(outs[0], o) for o in outs[1:])
    want = oracle_pred(cfg, W, T, recs[:2000])
    assert np.abs(outs[2][:2000] - want).max() / (np.abs(want).max() + 1e-3) < 1e-2
    with pytest.raises(Exception):
        RadianceCache(dataclasses.replace(cfg, infer_tiles=5))


def test_query_full_size_grid(cuda):
    # 16 levels x 2^19 entries x 2 features, base 16, growth 1.5
    cfg = NrcConfig(aabb_min=(-2, -1, -3), aabb_max=(2, 3, 1))
    c = RadianceCache(cfg)
    W, T = randomise(c, 8)
    recs = random_records(3000, 12, box=((-2, -1, -3), (2, 3, 1)))
    got = c.query(recs)
    want = oracle_pred(cfg, W, T, recs)
    assert np.abs(got - want).max() / (np.abs(want).max() + 1e-3) < 1e-2
    c.close()


def training_samples(n, seed):
    r = random_records(n, seed)
    s = np.zeros((n, 20), np.float32)
    s[:, :16] = r
    p, d = r[:, 0:3].astype(np.float64), r[:, 3:6].astype(np.float64)
    s[:, 16] = 0.5 + 0.4 * np.sin(6 * p[:, 0]) * np.cos(4 * p[:, 1]) + 0.2 * d[:, 1]
    s[:, 17] = 0.3 + 0.3 * p[:, 2] ** 2 + 0.1 * d[:, 0]
    s[:, 18] = 0.8 * np.exp(-4 * ((p[:, 0] - 0.5) ** 2 + (p[:, 1] - 0.5) ** 2))
    return s


@pytest.mark.parametrize("n", [128, 3000])
def test_gradients_match_oracle(cuda, n):
    cfg = NrcConfig(levels=6, log2_table_size=10, base_resolution=4, growth=1.8)
    c = RadianceCache(cfg)
    W, T = randomise(c, 3, w_scale=0.2, t_scale=0.3)
    s = training_samples(n, 5)
    gw, gt, loss = c.gradients(s)
    res = O.level_resolutions(cfg.base_resolution, cfg.growth, cfg.levels)
    dW, dT, oloss = O.gradients(W, O.f16(T), s, res, cfg.aabb_min, cfg.aabb_max)
    for l in range(6):
        rel = np.linalg.norm(gw[l] - dW[l]) / (np.linalg.norm(dW[l]) + 1e-30)
        print(f"layer {l}: |dW| {np.linalg.norm(dW[l]):.3e} rel err {rel:.2e}")
        assert rel < 3e-2, (l, rel)
    relt = np.linalg.norm(gt - dT) / (np.linalg.norm(dT) + 1e-30)
    print(f"table: rel err {relt:.2e}; loss gpu {loss:.5f} oracle {oloss:.5f}")
    assert relt < 3e-2
    assert abs(loss - oloss) <= 1e-2 * abs(oloss)
    assert not gw[5, 3:].any()
    c.close()


def test_adam_step_matches_oracle(cuda):
    cfg = NrcConfig(levels=4, log2_table_size=8, base_resolution=4, growth=2.0)
    c = RadianceCache(cfg)
    W, T = randomise(c, 4, w_scale=0.2, t_scale=0.3)
    s = training_samples(512, 9)
    gw, gt, _ = c.gradients(s)
    c.train_step(s)
    W1, T1 = c.get_params()
    w_want, _, _ = O.adam(W, 0, 0, gw, cfg.learning_rate, 1)
    t_want, _, _ = O.adam(T, 0, 0, gt, cfg.table_learning_rate, 1)
    assert np.abs(W1 - w_want).max() < 1e-6
    assert np.abs(T1 - t_want).max() < 1e-6
    c.close()


def test_training_reduces_loss_and_generalises(cuda):
    """300 Adam steps at learning rate 1e-2 on a smooth target.  The held-out
    error is typically 1e-3 to 2e-3; an occasional late loss spike (Adam's
    step at a high learning rate) lifts a single checkpoint about tenfold, so
    the bar is on the median of the last three checkpoints."""
    cfg = NrcConfig(levels=8, log2_table_size=14, base_resolution=4, growth=1.5)
    c = RadianceCache(cfg)
    held = training_samples(8192, 77)
    first, rels, losses = None, [], []
    for step in range(300):
        loss = c.train_step(training_samples(4096, 1000 + step))
        first = loss if first is None else first
        if step in (279, 289, 299):
            pred = c.query(held[:, :16])
            rels.append(float(np.mean((pred - held[:, 16:19]) ** 2) / np.mean(held[:, 16:19] ** 2)))
            losses.append(loss)
    rel = float(np.median(rels))
    print(f"loss {first:.4f} -> {losses}; held-out relative MSE at steps 280/290/300 {rels}")
    assert np.median(losses) < 0.1 * first
    assert rel < 0.01
    c.close()


def test_config_validation(cuda):
    for bad in (NrcConfig(levels=0), NrcConfig(levels=17), NrcConfig(log2_table_size=3),
                NrcConfig(growth=0.5), NrcConfig(learning_rate=0.0), NrcConfig(aabb_min=(1, 0, 0), aabb_max=(0, 1, 1))):
        with pytest.raises(N.VtError):
            RadianceCache(bad)
