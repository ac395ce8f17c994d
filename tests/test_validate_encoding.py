"""validateBvhEncoding (shared-bvh/src/validateBvhEncoding.ts:55) through the
C ABI (vt_validate_bvh_encoding), with the cases of the reference's own test
(shared-bvh/src/__tests__/validateBvhEncoding.test.ts), and the proof on every
tree the builder and the oracle produce.  No GPU needed."""
import numpy as np
import pytest

import oracle
from vitrum_b200 import _native as N
from vitrum_b200 import scenes
from vitrum_b200.bvh import validate_bvh_encoding as validate

W = 8
LEAF = 0xFFFF0000


def three_node_tree():
    nodes = np.zeros(3 * W, np.float32)
    words = nodes.view(np.uint32)
    nodes[0:6] = [0, 0, 0, 2, 1, 1]
    words[6], words[7] = 2, 0
    nodes[W:W + 6] = [0, 0, 0, 1, 1, 1]
    words[W + 6], words[W + 7] = 0, LEAF | 1
    nodes[2 * W:2 * W + 6] = [1, 0, 0, 2, 1, 1]
    words[2 * W + 6], words[2 * W + 7] = 1, LEAF | 1
    return nodes


def rejects(pattern, *args, **kw):
    with pytest.raises(N.VtError) as e:
        validate(*args, **kw)
    assert e.value.status == 6 and pattern in str(e.value), str(e.value)


def test_exact_proof_for_a_valid_tree():
    assert validate(three_node_tree(), 3, triangle_count=2) == {
        "nodeCount": 3, "rootCount": 1, "interiorNodeCount": 1, "leafNodeCount": 2, "maxDepth": 1,
        "maxTraversalStackEntries": 2, "traversalStackCapacity": 60, "triangleCount": 2}


def test_disjoint_forest_needs_every_root():
    nodes = np.zeros(2 * W, np.float32)
    words = nodes.view(np.uint32)
    nodes[0:6] = [0, 0, 0, 1, 1, 1]
    words[6], words[7] = 0, LEAF | 1
    nodes[W:W + 6] = [2, 0, 0, 3, 1, 1]
    words[W + 6], words[W + 7] = 1, LEAF | 1
    assert validate(nodes, 2, roots=[0, 1], triangle_count=2)["rootCount"] == 2
    rejects("unreachable", nodes, 2, roots=[0], triangle_count=2)


def test_rejects_malformed_extent_roots_topology_axes_bounds():
    rejects("expected exactly 8", np.zeros(7, np.float32), 1)
    rejects("declared more than once", three_node_tree(), 3, roots=[0, 0])
    t = three_node_tree(); t.view(np.uint32)[6] = 1
    rejects("invalid relative right-child offset", t, 3)
    t = three_node_tree(); t.view(np.uint32)[7] = 3
    rejects("invalid split axis", t, 3)
    t = three_node_tree(); t[W] = np.nan
    rejects("non-finite bounds", t, 3)
    t = three_node_tree(); t[W] = 2; t[W + 3] = 1
    rejects("inverted bounds", t, 3)
    t = three_node_tree(); t[2 * W + 3] = 3
    rejects("do not enclose child", t, 3)


def test_rejects_shared_children_and_small_stacks():
    nodes = np.zeros(5 * W, np.float32)
    words = nodes.view(np.uint32)
    for n in range(5):
        nodes[n * W:n * W + 6] = [0, 0, 0, 1, 1, 1]
    words[6], words[7] = 4, 0
    words[W + 6], words[W + 7] = 3, 0
    for n in (2, 3, 4):
        words[n * W + 7] = LEAF
    rejects("reachable more than once", nodes, 5)
    rejects("exceeding shader capacity 1", three_node_tree(), 3, traversal_stack_capacity=1)


def test_arbitrary_child_order_stack_bound():
    nodes = np.zeros(9 * W, np.float32)
    words = nodes.view(np.uint32)
    for n in range(9):
        nodes[n * W:n * W + 6] = [0, 0, 0, 1, 1, 1]
        words[n * W + 7] = LEAF
    for n in (0, 2, 4, 6):
        words[n * W + 6], words[n * W + 7] = 2, 0
    p = validate(nodes, 9, triangle_count=0, traversal_stack_capacity=5)
    assert p["maxDepth"] == 4 and p["maxTraversalStackEntries"] == 5
    rejects("requires 5 live stack entries", nodes, 9, triangle_count=0, traversal_stack_capacity=4)


def test_rejects_leaf_ranges_that_escape_overlap_or_gap():
    t = three_node_tree(); t.view(np.uint32)[2 * W + 6] = 2
    rejects("exceeds triangle capacity", t, 3, triangle_count=2)
    t = three_node_tree(); t.view(np.uint32)[2 * W + 6] = 0
    rejects("overlaps", t, 3, triangle_count=2)
    t = three_node_tree(); t.view(np.uint32)[W + 6] = 1
    rejects("leaves a gap", t, 3, triangle_count=3)


def test_empty_buffer():
    assert validate(np.zeros(0, np.uint32), 0, triangle_count=0)["nodeCount"] == 0


@pytest.mark.parametrize("n", [1, 2, 100, 65536])
def test_every_built_tree_passes(n):
    soup = scenes.random_triangles(n, seed=n)
    b = oracle.build_array_bvh(soup.positions, soup.indices)
    p = validate(b.nodes, b.node_count, triangle_count=n)
    assert p["leafNodeCount"] + p["interiorNodeCount"] == b.node_count
    nodes, perm = oracle.build_tlas(np.concatenate([soup.positions.reshape(-1, 4)[:min(n, 64), :3],
                                                    soup.positions.reshape(-1, 4)[:min(n, 64), :3] + 0.1], 1))
    validate(nodes, nodes.shape[0], triangle_count=perm.size)
