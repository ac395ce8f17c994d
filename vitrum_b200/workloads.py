"""Render one of the named workloads once, for profilers and quick checks.

    python -m vitrum_b200.workloads box_room  [--width 512 --height 512 --spp 64 --bounces 5]
    python -m vitrum_b200.workloads instanced [--width 1920 --height 1080 --spp 16 --bounces 8]
    python -m vitrum_b200.workloads query     [--rays 1048576 --trace-order 0]
    python -m vitrum_b200.workloads nrc       [--rays 1048576 --frames 10 --tiles 1]
    (--nrc: path tracing with the neural radiance cache, 4 x 65,536 training samples per frame)

Prints the frame's stage times (or the query's hit count) as one JSON line.
"""
from __future__ import annotations

import argparse
import json


def nrc_timing(n, reps, tiles=0):
    """Cache query and training throughput on device arrays (default cache
    config: 16 x 2^19 x 2 hash grid, 5 x 64 MLP; `tiles` query tiles per
    inference CTA, 0 = the default), CUDA-event timed."""
    import numpy as np
    import torch
    from .nrc import NrcConfig, RadianceCache
    dev = torch.device("cuda", 0)
    c = RadianceCache(NrcConfig(aabb_min=(-1, -1, -1), aabb_max=(1, 1, 1), infer_tiles=tiles))
    g = torch.Generator(device=dev).manual_seed(1)
    rec = torch.rand((n, 16), device=dev, generator=g) * 2 - 1
    d = rec[:, 3:6] / rec[:, 3:6].norm(dim=1, keepdim=True)
    rec[:, 3:6] = d
    rgb = torch.empty((n, 3), device=dev)
    smp = torch.rand((65536, 20), device=dev, generator=g)
    s = torch.cuda.current_stream(dev).cuda_stream
    reps = max(reps, 3)
    for _ in range(2):
        c.query_device(rec.data_ptr(), n, rgb.data_ptr(), s)
        c.train_step_device(smp.data_ptr(), 65536, s)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ev[0].record()
    for _ in range(reps):
        c.query_device(rec.data_ptr(), n, rgb.data_ptr(), s)
    ev[1].record()
    for _ in range(reps):
        c.train_step_device(smp.data_ptr(), 65536, s)
    ev[2].record()
    torch.cuda.synchronize()
    q_ms = ev[0].elapsed_time(ev[1]) / reps
    t_ms = ev[1].elapsed_time(ev[2]) / reps
    c.close()
    flop = 2 * 64 * 64 * 6  # padded MMA work per query (algorithmic 2 * 20,672)
    return {"workload": "nrc", "queries": n, "infer_tiles": tiles, "query_ms": q_ms, "queries_per_s": n / q_ms * 1e3,
            "mma_tflops": n * flop / q_ms / 1e9, "train_step_ms_65536": t_ms}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("workload", choices=["box_room", "instanced", "query", "nrc"])
    ap.add_argument("--width", type=int, default=0)
    ap.add_argument("--height", type=int, default=0)
    ap.add_argument("--spp", type=int, default=0)
    ap.add_argument("--bounces", type=int, default=0)
    ap.add_argument("--frames", type=int, default=1)
    ap.add_argument("--rays", type=int, default=1 << 20)
    ap.add_argument("--instances", type=int, default=1024)
    ap.add_argument("--nrc", action="store_true", help="path tracing with the neural radiance cache")
    ap.add_argument("--tiles", type=int, default=0, help="nrc: query tiles per inference CTA (1..4)")
    ap.add_argument("--trace-order", type=int, default=0,
                    help="query: spatial trace order, Morton bits per axis (0: input order)")
    a = ap.parse_args(argv)
    from . import scenes
    if a.workload == "nrc":
        print(json.dumps(nrc_timing(a.rays, a.frames, a.tiles)))
        return
    if a.workload == "query":
        from .bvh import build_compressed_wide_bvh
        soup, rays = scenes.config1(65536, a.rays, seed=2024)
        with build_compressed_wide_bvh(soup.positions, soup.indices) as g:
            g.set_trace_order(a.trace_order)
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
    if a.nrc:
        e.set_nrc(prefix_bounces=1)
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
