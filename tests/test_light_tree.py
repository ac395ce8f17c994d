"""The light tree (shared-samplers/src/lightTree.ts): the product's builder
(vt_light_tree_build) byte-equal to the oracle's restatement, and the oracle
pinned by the known answers of the reference's own tests
(shared-samplers/__tests__/lightTree.test.ts, lightTreeTraversal.test.ts).
No GPU needed."""
import math

import numpy as np
import pytest

import oracle
from vitrum_b200.light_tree import BUCKETS, build_light_tree


def line_input(powers):
    """makeInput of lightTree.test.ts:44-52: emitters at (2i, 0, 0), unit boxes."""
    n = len(powers)
    c = np.array([[2.0 * i, 0, 0] for i in range(n)])
    return np.asarray(powers, float), c, np.concatenate([c - 0.5, c + 0.5], 1)


def random_input(n, seed, cones=False, spread=10.0):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-spread, spread, (n, 3))
    h = rng.uniform(0.0, 1.0, (n, 3)) * (rng.random((n, 1)) < 0.7)
    p = rng.uniform(0.0, 5.0, n) * (rng.random(n) < 0.95)
    k = None
    if cones:
        ax = rng.normal(size=(n, 3))
        k = np.concatenate([ax, np.zeros((n, 1)), rng.uniform(0.2, math.pi, (n, 1)),
                            (rng.random((n, 1)) < 0.6).astype(float)], 1)
    return p, c, np.concatenate([c - h, c + h], 1), k


@pytest.mark.parametrize("n,cones", [(1, False), (2, False), (3, True), (17, True), (64, False), (257, True),
                                     (1000, True)])
def test_product_tree_equals_oracle_bytes(n, cones):
    p, c, b, k = random_input(n, seed=n, cones=cones)
    a = build_light_tree(p, c, b, k)
    o = oracle.light_tree_build(p, c, b, k)
    assert a.shape == o.shape and a.tobytes() == o.tobytes()


def test_product_tree_equals_oracle_degenerate():
    # co-located centroids: the descending-power split (lightTree.ts:393-402)
    n = 9
    c = np.zeros((n, 3))
    p = np.array([3, 1, 4, 1, 5, 9, 2, 6, 5], float)
    b = np.zeros((n, 6))
    a = build_light_tree(p, c, b)
    o = oracle.light_tree_build(p, c, b)
    assert a.tobytes() == o.tobytes()
    # balanced: depth ceil(log2 9) + 1 levels at most
    depth = {0: 0}
    for i in range(a.shape[0]):
        if a[i, 2] >= 0:
            depth[int(a[i, 2])] = depth[i] + 1
            depth[int(a[i, 3])] = depth[i] + 1
    assert max(depth.values()) <= math.ceil(math.log2(n))


def pmfs(tree, p, n):
    return np.array([oracle.light_tree_pdf(tree, p, e) for e in range(n)])


def test_single_and_pair_layout():
    # lightTree.test.ts:56-101: one emitter -> one leaf; two -> internal + two leaves
    t = oracle.light_tree_build(*line_input([42.0]))
    assert t.shape[0] == 1 and t[0, 0] == 0 and t[0, 1] == 1 and t[0, 15] == 1
    assert oracle.light_tree_pdf(t, [0, 0, 0], 0) == 1.0
    t = oracle.light_tree_build(*line_input([3.0, 7.0]))
    assert t.shape[0] == 3 and t[0, 0] == -1 and t[0, 15] == 2
    assert t[0, 1] == 1.0 and abs(t[1, 1] - 0.3) < 1e-7 and abs(t[2, 1] - 0.7) < 1e-7
    # represented powers are scale-free: doubling every power leaves the packed tree unchanged
    p, c, b = line_input([1.0, 2.0, 4.0, 8.0])
    assert oracle.light_tree_build(p, c, b).tobytes() == oracle.light_tree_build(2 * p, c, b).tobytes()


@pytest.mark.parametrize("n", [3, 4, 16, 64, 1000])
def test_pmf_partitions_to_exactly_one(n):
    # lightTreeTraversal.test.ts:106-155, :168-220: bucket-multiple PMFs summing to 1
    p, c, b, k = random_input(n, seed=7 * n, cones=True)
    t = oracle.light_tree_build(p, c, b, k)
    rng = np.random.default_rng(n)
    for x in rng.uniform(-12, 12, (3, 3)):
        f = pmfs(t, x, n)
        assert (f >= 1.0 / BUCKETS).all()                      # every leaf keeps its reserved bucket
        assert np.all(np.round(f * BUCKETS) == f * BUCKETS)
        assert f.sum() == 1.0
    assert oracle.light_tree_pdf(t, [0, 0, 0], n + 5) == 0.0   # an emitter not in the tree


def test_draws_agree_with_the_pmf():
    # lightTreeTraversal.test.ts:273-310: each draw's PMF is the deterministic PMF,
    # and the frequencies over every bucket reproduce it exactly
    p, c, b, k = random_input(12, seed=3, cones=True)
    t = oracle.light_tree_build(p, c, b, k)
    x = [1.0, -2.0, 0.5]
    f = pmfs(t, x, 12)
    rng = np.random.default_rng(1)
    for u in rng.integers(0, BUCKETS, 2000):
        e, pmf = oracle.light_tree_sample(t, x, int(u))
        assert pmf == f[e]
    # boundary of a represented interval: both sides land in the intended leaves
    t2 = oracle.light_tree_build(*line_input([1e-300, 1e300]))
    left = round(oracle.light_tree_pdf(t2, [0, 0, 0], 0) * BUCKETS)
    assert left >= 1
    assert oracle.light_tree_sample(t2, [0, 0, 0], left - 1)[0] == 0
    assert oracle.light_tree_sample(t2, [0, 0, 0], left)[0] == 1


def test_near_light_dominates_and_cones_cull():
    # lightTreeTraversal.test.ts:316-345: equal power, near vs far
    p = np.array([1.0, 1.0])
    c = np.array([[0.0, 0, 0], [100.0, 0, 0]])
    b = np.concatenate([c, c], 1)
    t = oracle.light_tree_build(p, c, b)
    f = pmfs(t, [1.0, 0, 0], 2)
    assert f[0] > 0.99
    # :403-413: a one-sided emitter facing away gets (almost) nothing
    k = np.array([[1.0, 0, 0, 0.0, math.pi / 2, 1.0], [0, 0, 0, 0, 0, 0.0]])
    c = np.array([[0.0, 0, 0], [3.0, 0, 0]])
    b = np.concatenate([c, c], 1)
    t = oracle.light_tree_build(np.array([1.0, 1.0]), c, b, k)
    behind = pmfs(t, [-2.0, 0, 0], 2)
    in_front = pmfs(t, [2.0, 0, 0], 2)
    assert behind[0] < 1e-3 and in_front[0] > 0.2
    # full-sphere packing: axis 0 and both cosines -1
    assert (t[0, 10:13] == 0).all() and t[0, 13] == -1 and t[0, 14] == -1


def test_distant_entries_share_their_buckets_evenly():
    p, c, b, k = random_input(5, seed=2)
    t = oracle.light_tree_build(p, c, b, k)
    for n_dist in (1, 2, 3):
        d = (BUCKETS * n_dist) // (n_dist + 1)
        tot = {}
        for bucket in np.linspace(0, BUCKETS - 1, 4001).astype(np.int64):
            e, pmf = oracle.light_select(t, 5, n_dist, [0.5, 0.5, 0.5], int(bucket))
            assert (e >= 5) == (bucket < d)
            tot[e] = pmf
        dist = [tot[5 + j] for j in range(n_dist)]
        assert abs(sum(dist) - d / BUCKETS) < 1e-12 and max(dist) - min(dist) <= 1.0 / BUCKETS
    # one positional entry: it takes the rest; none: the distant ones take all
    assert oracle.light_select(None, 1, 1, [0, 0, 0], BUCKETS - 1) == (0, 0.5)
    assert oracle.light_select(None, 0, 2, [0, 0, 0], BUCKETS - 1) == (1, 0.5)


def test_receiver_term_favours_lights_above_the_surface():
    """Two equal point lights above and below a receiver: with the normal up,
    the one below the horizon keeps only its defensive share (half the
    buckets over two leaves), the one above takes the rest; without a normal,
    or with a zero one (transmissive surfaces), they split evenly."""
    k = np.zeros((2, 6))
    k[:, 3], k[:, 4] = 0.0, math.pi
    c = np.array([[0.0, 1.0, 0.0], [0.0, -1.0, 0.0]])
    t = oracle.light_tree_build(np.array([1.0, 1.0]), c, np.concatenate([c, c], 1), k)
    up = dict(oracle.light_select(t, 2, 0, [0, 0, 0], b, [0, 1, 0]) for b in (0, BUCKETS - 1))
    assert up == {0: 0.75, 1: 0.25}  # entry 0 is the light above
    for nrm in (None, [0, 0, 0]):
        assert oracle.light_select(t, 2, 0, [0, 0, 0], 0, nrm)[1] == 0.5


def test_direct_importance_matches_the_reference_form():
    """The integrator's importance (direct f32 form, no receiver term) and the
    reference's scale-safe log form compute the same quantity: they agree to
    a few f32 ulps on every node of random trees, for points inside and
    outside the nodes' boxes and cones, except where the orientation taper
    (cos - cos_e) / (cos_o - cos_e) subtracts nearly equal cosines and
    magnifies their last-place differences (at most about 1e-4 here)."""
    worst, errs = 0.0, []
    for seed in range(4):
        p, c, b, k = random_input(40, seed=seed, cones=seed % 2 == 1, spread=3.0)
        t = oracle.light_tree_build(p, c, b, k)
        rng = np.random.default_rng(seed)
        for q in rng.uniform(-3, 4, (60, 3)):
            for node in range(t.shape[0]):
                ref = oracle.light_tree_importance(t, node, q)
                got = oracle.light_tree_importance_direct(t, node, q)
                if ref == 0.0 or got == 0.0:
                    assert ref == got or max(ref, got) < 1e-30
                    continue
                worst = max(worst, abs(got / ref - 1))
                errs.append(abs(got / ref - 1))
    assert worst < 2e-4 and np.median(errs) < 1e-6 and np.quantile(errs, 0.99) < 2e-6, (worst, np.quantile(errs, 0.99))
