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
    # path-tracing rays of the box room (512^2 / 64 spp / 5 bounces workload):
    # rays logged by the CPU path tracer at 128 x 128, 4 spp, same camera
    sc, cam = scenes.box_room()
    _, _, lc, ls, (nc, ns) = oracle.pt_render(sc, cam, 128, 128, 4, 5, log_rays=1 << 20)
    pos, idx, _, _, _, _, _ = oracle.flatten_scene(sc)
    wb = oracle.build_compressed_wide_bvh(pos, idx)
    cn, ct = oracle.count_visits(wb, pos, lc)
    sn, st = oracle.count_visits(wb, pos, ls, any_hit=True)
    out["box_room_pt_512_64spp_5b"] = {
        "sample": "128x128 pixels, 4 spp, 5 bounces (CPU path tracer, same estimator and camera)",
        "paths": 128 * 128 * 4, "closest_rays": nc, "shadow_rays": ns,
        "closest_per_path": nc / (128 * 128 * 4), "shadow_per_path": ns / (128 * 128 * 4),
        "closest_v_node": cn / len(lc), "closest_v_tri": ct / len(lc),
        "shadow_v_node": sn / len(ls), "shadow_v_tri": st / len(ls),
        "closest_bytes_per_ray": 32 + 16 + 80 * cn / len(lc) + 48 * ct / len(lc),
        "shadow_bytes_per_ray": 32 + 16 + 80 * sn / len(ls) + 48 * st / len(ls),
    }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "visit_counts.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
