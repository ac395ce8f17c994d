"""The C-ABI library loads and exports every entry point include/*.h declares (no GPU needed)."""
import glob
import os
import re

import numpy as np
import pytest

from vitrum_b200 import _native as N
from vitrum_b200 import bvh, scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(vt_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "vt_bvh_build" in names and "vt_bvh_trace_closest_device" in names


@pytest.mark.parametrize("name", declared_functions())
def test_symbol_exported(name):
    lib = N.lib()
    assert hasattr(lib, name), f"{name} declared in include/ but not exported"


def test_binding_table_matches_header():
    assert set(N.SIGNATURES) == set(declared_functions())


def test_version_and_error_strings():
    assert b"sm_100a" in N.lib().vt_version()
    assert N.lib().vt_last_error() is not None


def test_null_arguments_are_rejected_without_device():
    # argument validation happens before any CUDA call
    with pytest.raises(N.VtError) as e:
        N.call("vt_bvh_build", 0, None, 0, None, 0, None, None)
    assert e.value.status == 1
    with pytest.raises(N.VtError):
        N.call("vt_bvh_trace_closest", None, None, 1, None)


def test_unknown_build_option_raises():
    with pytest.raises(ValueError):
        bvh.build_compressed_wide_bvh(np.zeros(12, np.float32), np.zeros(4, np.uint32), leafSize=2)


def test_traversal_tree_option_maps_to_the_abi():
    # the reference's option keys plus traversalTree; names map to the C enum (0 = default)
    o = bvh._options({"maxLeafTriangles": 2, "traversalTree": "sah"})
    assert (o.max_leaf_triangles, o.traversal_tree) == (2, 2)
    assert bvh._options({}).traversal_tree == 0
    assert bvh._options({"traversalTree": "fast"}).traversal_tree == 3
    with pytest.raises(ValueError):
        bvh._options({"traversalTree": "binary"})
    with pytest.raises(N.VtError):  # set before any device work: a null handle is rejected
        N.call("vt_bvh_set_trace_order", None, 5)


def test_tuning_and_option_structs_match_the_header():
    # every vt_tuning / vt_engine_options / vt_nrc_config field the header declares, in order
    import re
    from vitrum_b200.batch import _Tuning
    from vitrum_b200.engine import _EngineOptions
    from vitrum_b200.nrc import _Config
    hdr = open(__import__("os").path.join(__import__("os").path.dirname(__file__), "..", "include",
                                          "vitrum_pt.h")).read()
    for cname, py in (("vt_tuning", _Tuning), ("vt_engine_options", _EngineOptions), ("vt_nrc_config", _Config)):
        body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (cname, cname), hdr, re.S).group(1)
        body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
        fields = re.findall(r"(\w+)(?:\[\d+\])?;", body)
        assert fields == [f for f, _ in py._fields_], cname


def test_generators_are_deterministic():
    a, ra = scenes.config1(256, 64, seed=7)
    b, rb = scenes.config1(256, 64, seed=7)
    c, _ = scenes.config1(256, 64, seed=8)
    assert np.array_equal(a.positions, b.positions) and np.array_equal(ra, rb)
    assert not np.array_equal(a.positions, c.positions)
    d = ra[:, 4:7].astype(np.float64)
    assert np.allclose(np.linalg.norm(d, axis=1), 1, atol=1e-6)
    assert np.allclose(np.linalg.norm(ra[:, 0:3].astype(np.float64), axis=1), 3, atol=1e-5)
