"""Render one of the named workloads once, for profilers and quick checks.

    python -m vitrum_b200.workloads box_room  [--width 512 --height 512 --spp 64 --bounces 5]
    python -m vitrum_b200.workloads instanced [--width 1920 --height 1080 --spp 16 --bounces 8]
    python -m vitrum_b200.workloads query     [--rays 1048576]

Prints the frame's stage times (or the query's hit count) as one JSON line.
"""
from __future__ import annotations

import argparse
import json


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("workload", choices=["box_room", "instanced", "query"])
    ap.add_argument("--width", type=int, default=0)
    ap.add_argument("--height", type=int, default=0)
    ap.add_argument("--spp", type=int, default=0)
    ap.add_argument("--bounces", type=int, default=0)
    ap.add_argument("--frames", type=int, default=1)
    ap.add_argument("--rays", type=int, default=1 << 20)
    ap.add_argument("--instances", type=int, default=1024)
    a = ap.parse_args(argv)
    from . import scenes
    if a.workload == "query":
        from .bvh import build_compressed_wide_bvh
        soup, rays = scenes.config1(65536, a.rays, seed=2024)
        with build_compressed_wide_bvh(soup.positions, soup.indices) as g:
            hits = g.intersect_first_hit(rays)
        print(json.dumps({"workload": "query", "rays": a.rays, "hits": int((hits["prim"] >= 0).sum())}))
        return
    from .engine import Engine
    if a.workload == "box_room":
        sc, cam = scenes.box_room()
        W, H, spp, B = a.width or 512, a.height or 512, a.spp or 64, a.bounces or 5
    else:
        sc, cam = scenes.instanced_cloud(n_instances=a.instances)
        W, H, spp, B = a.width or 1920, a.height or 1080, a.spp or 16, a.bounces or 8
    e = Engine(max_bounces=B)
    e.set_scene(sc)
    out = {}
    for f in range(a.frames):
        e.reset()
        out = e.profile_frame(cam, W, H, samples=spp, frame_seed=f)
    st = e.stats()
    e.dispose()
    print(json.dumps({"workload": a.workload, "resolution": [W, H], "spp": spp, "bounces": B,
                      "stages": out, "closest_rays": st["closest_rays"], "shadow_rays": st["shadow_rays"]}))


if __name__ == "__main__":
    main()
