"""Per-ray node-visit and triangle-test counts for the algorithmic-bytes model.

The bench reports roofline.achieved = algorithmic bytes per launch / kernel
time with, per ray, B = 32 (ray in) + 16 (hit out) + 80 * V_node + 48 * V_tri.
V_node and V_tri are counted here by the CPU oracle's near-first traversal of
the reference-algorithm BVH (binned SAH + 8-wide collapse) for the exact
seeded workload, so the model does not depend on the device layout.

    python tests/golden/make_visit_counts.py
"""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from vitrum_b200 import scenes  # noqa: E402


def main():
    out = {}
    soup, rays = scenes.config1()
    w = oracle.build_compressed_wide_bvh(soup.positions, soup.indices)
    nn, nt = oracle.count_visits(w, soup.positions, rays)
    n = rays.shape[0]
    out["closest_hit_65536_tris_1048576_rays_seed2024"] = {
        "rays": n, "node_visits": nn, "triangle_tests": nt,
        "v_node": nn / n, "v_tri": nt / n,
        "bytes_per_ray": 32 + 16 + 80 * nn / n + 48 * nt / n,
    }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "visit_counts.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
