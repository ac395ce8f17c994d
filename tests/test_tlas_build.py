"""The product's top-level build (vt_tlas_build, host C++) byte for byte
against the reference's golden TLAS and against the oracle's restatement of
buildTlas (shared-bvh/src/tlas.ts:859-989).  No GPU needed."""
import numpy as np
import pytest

import oracle
from vitrum_b200 import _native as N
from vitrum_b200 import bvh as vb

from test_oracle_golden import golden_tlas


@pytest.mark.parametrize("case", list(golden_tlas()), ids=lambda c: c[0])
def test_tlas_build_matches_reference_golden_bytes(case):
    _, aabbs, gold_nodes, gold_perm, count = case
    nodes, perm = vb.build_tlas(aabbs)
    assert nodes.shape[0] == count
    assert np.array_equal(nodes, gold_nodes)
    assert np.array_equal(perm, gold_perm)


def _random_aabbs(n, seed, spread=20.0, size=(0.05, 2.0)):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-spread, spread, (n, 3))
    h = rng.uniform(*size, (n, 3))
    return np.concatenate([c - h, c + h], axis=1)


@pytest.mark.parametrize("n,leaf,bins", [(1, 1, 16), (2, 1, 16), (7, 1, 16), (64, 1, 16), (1024, 1, 16),
                                         (1000, 4, 16), (333, 2, 8), (500, 1, 32)])
def test_tlas_build_matches_oracle(n, leaf, bins):
    a = _random_aabbs(n, seed=n * 31 + leaf)
    nodes, perm = vb.build_tlas(a, maxLeafSize=leaf, binCount=bins)
    on, op = oracle.build_tlas(a, max_leaf=leaf, bins=bins)
    assert np.array_equal(nodes, on) and np.array_equal(perm, op)


def test_tlas_build_degenerate_inputs_match_oracle():
    cases = [
        np.tile([0.0, 0.0, 0.0, 1.0, 1.0, 1.0], (37, 1)),                       # coincident: balanced fallback
        np.concatenate([np.tile([0.0, 0.0, 0.0, 0.0, 0.0, 0.0], (9, 1)),        # points and slabs
                        _random_aabbs(20, 3, size=(0.0, 0.0))]),
        _random_aabbs(300, 4, spread=1e-9),                                     # centroid span ~ 1e-9
        np.array([[i, 0, 0, i + 1, 1, 1] for i in range(200)], np.float64),     # a line of boxes
    ]
    for a in cases:
        nodes, perm = vb.build_tlas(a)
        on, op = oracle.build_tlas(a)
        assert np.array_equal(nodes, on) and np.array_equal(perm, op)


def test_tlas_build_rejects_bad_input():
    with pytest.raises(N.VtError):
        vb.build_tlas(np.zeros((0, 6)))
    with pytest.raises(N.VtError) as e:
        vb.build_tlas(np.array([[0, 0, 0, -1, 1, 1]], np.float64))
    assert e.value.status == 2
    with pytest.raises(N.VtError):
        vb.build_tlas(np.array([[0, 0, 0, np.inf, 1, 1]], np.float64))
    with pytest.raises(ValueError):
        vb.build_tlas(np.zeros((1, 6)), leafSize=2)
