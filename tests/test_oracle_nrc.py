"""Pins the numpy NRC oracle (oracle/nrc.py) against the reference's known
answers (walkaround-hybrid/src/neural/nrc/__tests__/nrcEncoding.test.ts,
fusedMlp.test.ts) and against finite differences."""
import math

import numpy as np
import pytest

from oracle import nrc as O


def test_spatial_hash_formula():
    # nrcEncoding.test.ts:54-64: (ix*1) ^ (iy*2654435761) ^ (iz*805459861) in u32
    expected = (5 ^ ((9 * 2654435761) & 0xFFFFFFFF) ^ ((2 * 805459861) & 0xFFFFFFFF)) % 1000
    assert O.spatial_hash(5, 9, 2, 1000) == expected
    h = O.spatial_hash(np.arange(50) * 13, np.arange(50) * 7 + 1, np.arange(50) * 101 + 3, 97)
    assert (h >= 0).all() and (h < 97).all()


def test_level_resolution_is_floor_of_geometric_growth():
    r = O.level_resolutions(16, 1.5, 16)
    assert r[0] == 16 and r[1] == 24 and r[2] == 36 and r[15] == math.floor(16 * 1.5 ** 15)


@pytest.mark.parametrize("p", [(0.13, 0.77, 0.41), (0.5, 0.5, 0.5), (0.999, 0.001, 0.333)])
def test_trilinear_weights_partition_of_unity(p):
    # nrcEncoding.test.ts:70-76
    rows, w = O.trilinear(np.array([p], np.float32), 8, 97)
    assert abs(w.sum() - 1) < 1e-6 and (rows >= 0).all() and (rows < 97).all()


def test_normalise_clamps_to_unit_box():
    # nrcEncoding.test.ts:104-110
    n = O.normalise(np.array([[2.0, -3.0, 0.0]]), (-1, -1, -1), (1, 1, 1))
    assert n[0, 0] == 1 and n[0, 1] == 0 and abs(n[0, 2] - 0.5) < 1e-7


def test_hash_grid_backward_is_the_weighted_scatter():
    # nrcEncoding.test.ts:250-285: each corner row receives weight * dOut, and
    # per level the scattered gradient sums back to dOut
    rng = np.random.default_rng(3)
    n01 = rng.random((1, 3)).astype(np.float32)
    res = O.level_resolutions(4, 2.0, 3)
    dout = rng.standard_normal((1, 6))
    g = O.hash_grid_backward(dout, n01, res, (3, 61, 2))
    for l in range(3):
        assert np.allclose(g[l].sum(0), dout[0, 2 * l:2 * l + 2], atol=1e-12)
        rows, w = O.trilinear(n01, res[l], 61)
        want = np.zeros((61, 2))
        for c in range(8):
            want[rows[0, c]] += w[0, c] * dout[0, 2 * l:2 * l + 2]
        assert np.allclose(g[l], want, atol=1e-12)


def test_relative_l2_known_answers():
    # fusedMlp.test.ts:176-211
    g, _ = O.output_gradient(np.array([[0.0, 0.0, 0.0]]), np.array([[1.0, 2.0, 3.0]]), 1)
    assert np.allclose(g[0], [-2 / 3 / 0.01, -4 / 3 / 0.01, -6 / 3 / 0.01], rtol=1e-12)
    pred = np.array([[4.0, 2.0, 1.0]])
    g, _ = O.output_gradient(pred, np.array([[1.0, 1.0, 1.0]]), 2)
    lum = 0.299 * 4 + 0.587 * 2 + 0.114 * 1
    scale = 2 / 2 / 3 / (lum * lum + 0.01)
    assert np.allclose(g[0], [3 * scale, 1 * scale, 0.0], rtol=1e-12)
    big = np.finfo(np.float64).max
    g, _ = O.output_gradient(np.array([[big, -big, big]]), np.zeros((1, 3)), 1)
    assert np.isfinite(g).all() and (np.abs(g) <= 65504).all()
    g, _ = O.output_gradient(np.array([[np.nan, 0.0, 0.0]]), np.zeros((1, 3)), 1)
    assert (g == 0).all()


def test_sh4_is_orthonormal():
    # Fibonacci-sphere quadrature of the 16x16 Gram matrix
    n = 200000
    i = np.arange(n) + 0.5
    z = 1 - 2 * i / n
    r = np.sqrt(1 - z * z)
    phi = math.pi * (1 + 5 ** 0.5) * i
    d = np.stack([r * np.cos(phi), r * np.sin(phi), z], 1)
    Y = O.sh4(d)
    G = Y.T @ Y * (4 * math.pi / n)
    assert np.abs(G - np.eye(16)).max() < 1e-3


def _small_problem(seed=0, n=64, levels=3, T=64):
    rng = np.random.default_rng(seed)
    W = rng.standard_normal((6, 64, 64)) * 0.2
    W[5, 3:] = 0
    table = rng.standard_normal((levels, T, 2)) * 0.5
    s = np.zeros((n, 20))
    s[:, 0:3] = rng.random((n, 3))
    d = rng.standard_normal((n, 3))
    s[:, 3:6] = d / np.linalg.norm(d, axis=1, keepdims=True)
    s[:, 6:16] = rng.random((n, 10))
    s[:, 16:19] = rng.random((n, 3)) * 2
    res = O.level_resolutions(4, 2.0, levels)
    return W, table, s, res


def _loss(W, table, s, res):
    X, _ = O.encode(s[:, :16], table, res, (0, 0, 0), (1, 1, 1), fp16=False)
    _, pred = O.forward(W, X, fp16=False)
    # the relative-L2 denominator is a stop-gradient: hold it at the base point
    return pred


def test_oracle_backward_matches_finite_differences():
    W, table, s, res = _small_problem()
    dW, dT, _ = O.gradients(W, table, s, res, (0, 0, 0), (1, 1, 1), fp16=False)
    X, _ = O.encode(s[:, :16], table, res, (0, 0, 0), (1, 1, 1), fp16=False)
    _, p0 = O.forward(W, X, fp16=False)
    lum = np.minimum(np.abs(O.rel_l2_luminance(p0)), 1e19)
    den = lum * lum + O.EPS

    def frozen_loss(Wx, Tx):
        pred = _loss(Wx, Tx, s, res)
        return (((pred - s[:, 16:19]) ** 2).sum(1) / den / 3).mean()

    rng = np.random.default_rng(1)
    h = 1e-6
    for _ in range(12):
        l, o, i = rng.integers(0, 6), rng.integers(0, 3), rng.integers(0, 64)
        if l < 5:
            o = rng.integers(0, 64)
        Wp, Wm = W.copy(), W.copy()
        Wp[l, o, i] += h
        Wm[l, o, i] -= h
        fd = (frozen_loss(Wp, table) - frozen_loss(Wm, table)) / (2 * h)
        assert abs(fd - dW[l, o, i]) <= 1e-6 * max(1.0, abs(fd)), (l, o, i, fd, dW[l, o, i])
    touched = np.argwhere(np.abs(dT) > 1e-8)
    for idx in touched[rng.choice(len(touched), 8, replace=False)]:
        Tp, Tm = table.copy(), table.copy()
        Tp[tuple(idx)] += h
        Tm[tuple(idx)] -= h
        fd = (frozen_loss(W, Tp) - frozen_loss(W, Tm)) / (2 * h)
        assert abs(fd - dT[tuple(idx)]) <= 1e-6 * max(1.0, abs(fd))


def test_adam_first_step_moves_by_learning_rate():
    p, m, v = O.adam(np.array([1.0, -2.0, 0.5]), np.zeros(3), np.zeros(3), np.array([0.3, -4.0, 0.0]), 1e-2, 1)
    assert np.allclose(p, [1.0 - 1e-2, -2.0 + 1e-2, 0.5], atol=1e-9)
    p2, _, _ = O.adam(np.array([1.0]), np.zeros(1), np.zeros(1), np.array([np.nan]), 1e-2, 1)
    assert p2[0] == 1.0
