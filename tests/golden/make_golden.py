"""Extract the reference's byte golden for the BVH/TLAS pack into a small fixture.

Source (read from the reference checkout, never at test time):
  packages/shared-bvh/src/__tests__/scenePack.golden.json
captured by the reference's own test packages/shared-bvh/src/__tests__/scenePackGolden.test.ts.

The fixture keeps, for the `multiMesh` and `resizeSplice` packs, exactly the
buffers the BVH tests need: packed positions, BVH-order indices, BLAS node
words, per-primitive bindings and the TLAS buffers.  Run:

    python tests/golden/make_golden.py <reference checkout root>
"""
import json
import os
import sys


def main(ref_root: str) -> None:
    src = os.path.join(ref_root, "packages/shared-bvh/src/__tests__/scenePack.golden.json")
    with open(src) as f:
        g = json.load(f)
    keep = ("positions", "indices", "bvhNodes", "triangleCount", "tlasNodes", "tlasInstanceIndices",
            "tlasBlasRoots", "tlasInstanceWorldToLocal", "tlasInstanceLocalToWorld", "tlasNodeCount",
            "primitiveTlasBindings")
    out = {name: {k: g[name][k] for k in keep} for name in ("multiMesh", "resizeSplice")}
    out["_source"] = "packages/shared-bvh/src/__tests__/scenePack.golden.json"
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "scenepack_golden.json")
    with open(dst, "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print("wrote", dst, os.path.getsize(dst), "bytes")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <reference checkout root>")
    main(sys.argv[1])
