"""Benchmark of the B200 ray-tracing hot path (one JSON line on rank 0).

Headline workload (per GPU, N=1): unidirectional path tracing of the
procedural box room -- 262,146 triangles, 512 x 512, 64 spp, at most 5
bounces, NEE + MIS, Russian roulette after bounce 3, FP32 accumulation.  One
step = one frame rendered from a cleared accumulation.  Metric: Mrays/s
(extension + shadow rays traced, whole job); samples/s and ms/frame beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

* value: device time of K frames (CUDA events on the engine's stream around
  each frame's graph replays; barrier + synchronize around the loop; max
  over ranks).  Each frame streams ~400 MB of wave state (> 126 MB L2).
* e2e: the same frames through the public Engine calls with the image read
  back to host memory each step (vt_render_frame + vt_capture).
* roofline: the traversal kernel (extension + shadow launches) -- algorithmic
  bytes 32 + 16 + 80 V_node + 48 V_tri per ray with V counted by the CPU
  oracle on this scene's path-tracing rays (tests/golden/visit_counts.json),
  divided by the traversal stages' device time from a profiled frame, against
  the measured HBM copy bandwidth.
* query: the closest-hit query workload (65,536 triangles, 1,048,576 rays)
  with its own roofline, reported in the same line.
* instanced: the two-level workload (1024 instances, 1920x1080, 16 spp, 8
  bounces) in the same line: Mrays/s, ms/frame, stage times.
* nrc: equal-time relMSE of the neural-radiance-cache path tracer against
  plain path tracing on the instanced scene at 1920x1080 x 16 spp per frame:
  64 frames from a cold start (training and warm-up charged), five seeds,
  against a 16,384-spp FP64 oracle; accumulated and per-frame results.
* light_tree: light-tree against uniform NEE selection at equal time on the
  instanced scene; build: GPU scene builds against the host pipeline.
* batch: 64 box rooms of uneven size rendered as one batch (autotuned launch
  shape, one CUDA graph per batch frame) against the same frames one scene at
  a time: aggregate Mrays/s of both.
* Launch shapes and tree shapes come from the project's autotuners, run
  outside the timed regions.
* cpu_baseline / --impl reference: the C restatement (oracle) of the same
  estimator on all host cores, full 512x512 frame at a few spp per step, the
  scene and BVH built before the clock starts (no reference CPU integrator
  exists at this scale; the reference's own CPU tracer is a Lambert-only
  brute-force test helper); the query line carries the config-1 build time
  and query rate of the C restatement of shared-bvh at 1 thread and all cores.
* N > 1: independent replicas (pixels/frames are independent, the scene is
  replicated, no data-path collective): weak scaling.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W = H = 512
SPP = 64
BOUNCES = 5
Q_TRIS = 65536
Q_RAYS = 1 << 20
Q_SEED = 2024
Q_BATCHES = 4
WORKLOAD = ("box-room path tracing: 262,146 triangles, 512x512, 64 spp, max 5 bounces, NEE+MIS on the area "
            "light, RR after bounce 3, FP32 accumulation")
METRIC = "Mrays/s (box-room path tracing 512x512, 64 spp, 5 bounces; extension + shadow rays)"


def _env_rank():
    from vitrum_b200.replicas import env_rank
    return env_rank()


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _profile_value(name, key):
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith(key + ":"):
            return float(line.split(":")[1].split()[0])
    return None


def _scaled_traffic(rays_per_frame):
    """DRAM bytes of the traversal launches per frame: the ncu-measured bytes per
    extension ray of a bounce-0 launch (profiles/path_trace_box_room.txt) times
    the frame's traced rays (an estimate: shadow rays are assumed to cost the same)."""
    b = _profile_value("path_trace_box_room.txt", "dram_bytes_per_extension_ray")
    return None if b is None else b * rays_per_frame


def _visits():
    with open(os.path.join(ROOT, "tests", "golden", "visit_counts.json")) as f:
        return json.load(f)


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", f"vt_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        self.proc.wait()
        self.f.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ CPU baseline
REF_SPP = 32  # samples per pixel of each reference-arm step (full 512x512 frame, about 5 s on 16 host cores)


def _cpu_pt_scene():
    import oracle
    from vitrum_b200 import scenes
    sc, cam = scenes.box_room()
    t0 = time.perf_counter()
    S = oracle.PtScene(sc)
    return S, cam, time.perf_counter() - t0


def cpu_pt_baseline(S, cam, spp=REF_SPP):
    """The path-tracing estimator restated in C (oracle) on the full 512x512
    frame of the same scene and camera at `spp` samples per pixel, on all host
    cores, plus the single-thread rate on a 64x64 frame of the same
    camera (the scene and its BVH are built before either clock starts)."""
    import oracle
    threads = oracle.hw_threads()
    nc, ns, dt = oracle.pt_ray_totals(S, cam, W, H, spp, BOUNCES, seed=31, nthreads=threads)
    nc1, ns1, dt1 = oracle.pt_ray_totals(S, cam, 64, 64, 4, BOUNCES, seed=32, nthreads=1)
    return {"value": (nc + ns) / dt / 1e6, "unit": "Mrays/s", "cores": threads, "kind": "port",
            "sample": f"full {W}x{H} frame of the same scene and camera, {spp} spp, {BOUNCES} bounces "
                      f"({nc + ns} rays, {dt:.2f} s); C restatement of the estimator (FP64 visibility through the "
                      f"reference binned-SAH BVH), scene and BVH built before the clock starts",
            "single_thread": {"value": (nc1 + ns1) / dt1 / 1e6, "unit": "Mrays/s", "cores": 1,
                              "sample": f"64x64 frame of the same camera, 4 spp ({nc1 + ns1} rays)"}}


_QUERY_HITS = {}


def cpu_query_baseline():
    """Config-1 closest-hit workload through the C restatement of shared-bvh
    (buildArrayBvh + 8-wide collapse, then the reference's FP64 LIFO first-hit
    query): build ms, and query Mrays/s on 1 thread and on all host cores, each
    on a bounded slice of the 1,048,576 bench rays.  The FP64 hits of that
    slice also check the device's hits of the same rays (tie / edge / error
    counts, as the parity tests classify them)."""
    import oracle
    from oracle import parity
    from vitrum_b200 import scenes
    soup, _ = scenes.config1(Q_TRIS, 16, seed=Q_SEED)
    t0 = time.perf_counter()
    b = oracle.build_array_bvh(soup.positions, soup.indices)
    t1 = time.perf_counter()
    w = oracle.collapse_wide(b)
    t2 = time.perf_counter()
    rays = scenes.sphere_rays(Q_RAYS, seed=Q_SEED + 1)
    threads = oracle.hw_threads()
    n1, nall = 16384, 131072
    t3 = time.perf_counter()
    oracle.first_hit(w, soup.positions, rays[:n1], nthreads=1)
    t4 = time.perf_counter()
    ref = oracle.first_hit(w, soup.positions, rays[:nall], nthreads=threads)
    t5 = time.perf_counter()
    check = None
    if "hits" in _QUERY_HITS:
        from vitrum_b200.bvh import HIT_DTYPE
        dev_hits = _QUERY_HITS["hits"][:nall].view(HIT_DTYPE).reshape(-1)
        rep = parity.classify(soup.positions, soup.indices, rays[:nall], dev_hits, ref[:3])
        check = {k: rep[k] for k in ("n", "hits", "mismatches", "tie", "edge", "error")}
        check["edge_margin_max"] = rep["edge_margin_max"]
    return {"value": nall / (t5 - t4) / 1e6, "unit": "Mrays/s", "cores": threads, "kind": "port",
            "parity_vs_fp64": check,
            "sample": f"first {nall} of the 1,048,576 bench rays on all cores; C restatement of shared-bvh "
                      "(binned SAH, greedy 8-wide collapse, FP64 LIFO first-hit query)",
            "single_thread": {"value": n1 / (t4 - t3) / 1e6, "unit": "Mrays/s", "cores": 1,
                              "sample": f"first {n1} bench rays"},
            "build_ms": {"binary_sah": round((t1 - t0) * 1e3, 1), "wide_collapse": round((t2 - t1) * 1e3, 1),
                         "cores": 1}}


def run_reference(args, rank, world):
    """The reference's estimator on the host cores (C restatement; the
    reference ships no production CPU integrator and no JS runtime exists on
    this image): every step renders the full 512x512 frame of the headline
    scene and camera at REF_SPP samples per pixel with all host threads.  The
    scene set-up and BVH build happen once, before the warm-up."""
    if rank != 0:
        return
    import oracle
    S, cam, build_s = _cpu_pt_scene()
    threads = oracle.hw_threads()
    for i in range(args.warmup):
        oracle.pt_ray_totals(S, cam, W, H, REF_SPP, BOUNCES, seed=1000 + i, nthreads=threads)
    rays, secs = 0, 0.0
    for i in range(args.steps):
        nc, ns, dt = oracle.pt_ray_totals(S, cam, W, H, REF_SPP, BOUNCES, seed=i, nthreads=threads)
        rays += nc + ns
        secs += dt
    S.close()
    value = rays / secs / 1e6
    sample = (f"each step the full {W}x{H} frame of the same scene and camera at {REF_SPP} spp, {BOUNCES} bounces, "
              f"all {threads} host threads; C restatement of the path-tracing estimator (the reference ships no "
              f"production CPU integrator); scene + BVH built once before the warm-up ({build_s:.2f} s)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (procedural box room)",
        "config": {"workload": WORKLOAD, "resolution": [W, H], "spp_per_step": REF_SPP, "max_bounces": BOUNCES,
                   "scene_build_s": round(build_s, 3)},
        "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ query workload
def run_query(args, dev, local, rank, world, barrier):
    import torch
    from vitrum_b200 import _native as N
    from vitrum_b200 import bvh as vb
    from vitrum_b200 import scenes
    soup, _ = scenes.config1(Q_TRIS, 16, seed=Q_SEED)
    g = vb.build_compressed_wide_bvh(soup.positions, soup.indices, device=local)
    host = [scenes.sphere_rays(Q_RAYS, seed=Q_SEED + 1 + 1000 * rank + b) for b in range(Q_BATCHES)]
    d_rays = [torch.from_numpy(r).to(dev) for r in host]
    d_hits = [torch.empty((Q_RAYS, 4), dtype=torch.int32, device=dev) for _ in range(Q_BATCHES)]
    stream = torch.cuda.current_stream(dev)

    def step(i):
        b = i % Q_BATCHES
        g.trace_closest_device(d_rays[b].data_ptr(), Q_RAYS, d_hits[b].data_ptr(), stream.cuda_stream)

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize(dev)
    barrier()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    ev[0].record(stream)
    for i in range(args.steps):
        step(i)
        ev[i + 1].record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    per = [ev[i].elapsed_time(ev[i + 1]) for i in range(args.steps)]
    total_ms = ev[0].elapsed_time(ev[-1])
    if rank == 0:
        _QUERY_HITS["hits"] = d_hits[0].cpu().numpy()  # batch 0: the rays the CPU baseline re-traces
    # the same launches in spatial trace order (entry cell and octant, 2^5 cells per axis), sort included
    g.set_trace_order(5)
    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize(dev)
    ev[0].record(stream)
    for i in range(args.steps):
        step(i)
    ev[1].record(stream)
    torch.cuda.synchronize(dev)
    spatial_ms = ev[0].elapsed_time(ev[1]) / args.steps
    g.set_trace_order(0)
    pin = [torch.from_numpy(r).pin_memory() for r in host]
    pin_hits = torch.empty((Q_RAYS, 4), dtype=torch.int32).pin_memory()
    N.call("vt_bvh_trace_closest", g.handle, ctypes.c_void_p(pin[0].data_ptr()), Q_RAYS,
           ctypes.c_void_p(pin_hits.data_ptr()))
    t0 = time.perf_counter()
    for i in range(args.steps):
        N.call("vt_bvh_trace_closest", g.handle, ctypes.c_void_p(pin[i % Q_BATCHES].data_ptr()), Q_RAYS,
               ctypes.c_void_p(pin_hits.data_ptr()))
    e2e_s = time.perf_counter() - t0
    model = _visits()["closest_hit_65536_tris_1048576_rays_seed2024"]
    peak, peak_kind = _peaks()
    avg_s = statistics.mean(per) / 1e3
    achieved = model["bytes_per_ray"] * Q_RAYS / avg_s / 1e9
    g.close()
    return {
        "workload": "closest-hit query: 65,536 float32 triangles, 1,048,576 rays/launch (tmin 1e-4, tmax inf); "
                    "4 rotating ray batches (192 MB rays+hits) > 126 MB L2",
        "value": Q_RAYS * args.steps / (total_ms / 1e3) / 1e6, "unit": "Mrays/s",
        "ms_per_launch": total_ms / args.steps,
        "spatial_order_ms_per_launch": spatial_ms,
        "e2e": {"value": Q_RAYS * args.steps / e2e_s / 1e6, "unit": "Mrays/s", "h2d_bytes_per_step": Q_RAYS * 32,
                "d2h_bytes_per_step": Q_RAYS * 16},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": _profile_value("traverse_closest_config1.txt", "dram_bytes_per_launch"),
                     "peak_kind": peak_kind,
                     "model": f"{model['bytes_per_ray']:.1f} B/ray (48 + 80*{model['v_node']:.3f} + "
                              f"48*{model['v_tri']:.3f})"},
    }


# ------------------------------------------------------------------ instanced workload
I_W, I_H, I_SPP, I_BOUNCES = 1920, 1080, 16, 8


def run_instanced(args, dev, local, barrier):
    """1024-instance two-level scene (8 prototypes, 399,616 distinct / 50,961,408
    instanced triangles), gradient sky + 32 point lights, 1920x1080, 16 spp, 8 bounces."""
    import torch
    from vitrum_b200 import scenes
    from vitrum_b200.engine import Engine
    sc, cam = scenes.instanced_cloud()
    e = Engine(device=local, max_bounces=I_BOUNCES)
    t0 = time.perf_counter()
    e.set_scene(sc)
    build_s = time.perf_counter() - t0
    steps = max(1, min(args.steps, 3))

    def frame(seed):
        e.reset()
        e.render_frame(cam, I_W, I_H, samples=I_SPP, frame_seed=seed)

    # tree shape and launch shape from the project's autotuners (outside the timed
    # region): on this scene, with lambertian, metal and glass instances and sky
    # misses in one queue, the launch-shape tuner turns the material sort on
    shape_trials = e.autotune_bvh(sc, cam, I_W, I_H, samples=I_SPP, frame_seed=555) if not args.no_autotune else []
    trials = e.autotune(cam, I_W, I_H, samples=I_SPP, frame_seed=555) if not args.no_autotune else []
    tuning = dict(e.tuning, trials=len(trials), bvh_shape_trials=shape_trials)
    frame(7)
    e.reset()
    stages = e.profile_frame(cam, I_W, I_H, samples=I_SPP, frame_seed=8)
    torch.cuda.synchronize(dev)
    barrier()
    r0 = e.stats()
    ms = []
    for i in range(steps):
        frame(100 + i)
        ms.append(e.stats()["last_frame_ms"])
    torch.cuda.synchronize(dev)
    barrier()
    r1 = e.stats()
    rays = (r1["closest_rays"] - r0["closest_rays"]) + (r1["shadow_rays"] - r0["shadow_rays"])
    dev_s = sum(ms) / 1e3
    # instance updates (every instance moved): top-level refit and rebuild, bottom levels kept
    import numpy as np
    from vitrum_b200.engine import Instance
    upd = {}
    for mode in ("refit", "rebuild"):
        t_ms = []
        for k in range(4):
            shift = np.eye(4, dtype=np.float32)
            shift[:3, 3] = (0.05 * (k + 1), 0.0, -0.03 * (k + 1))
            moved = [Instance(i.mesh, (shift @ np.asarray(i.local_to_world, np.float32)).astype(np.float32),
                              i.material) for i in sc.instances]
            t0 = time.perf_counter()
            e.update_instances(moved, rebuild=mode == "rebuild")
            t_ms.append((time.perf_counter() - t0) * 1e3)
        upd[mode + "_ms"] = round(float(np.median(t_ms)), 3)
    e.dispose()
    return {
        "workload": "two-level instanced cloud: 1024 instances of 8 prototype meshes (icospheres levels 3-6, "
                    "256x64 torus, cubes 32/64/128 cells per edge), 399,616 distinct / 50,961,408 instanced "
                    "triangles, gradient sky + 32 point lights, 1920x1080, 16 spp, max 8 bounces",
        "value": rays / dev_s / 1e6, "unit": "Mrays/s", "ms_per_frame": dev_s * 1e3 / steps,
        "samples_per_s": I_W * I_H * I_SPP * steps / dev_s, "frames": steps,
        "rays_per_frame": {"extension": (r1["closest_rays"] - r0["closest_rays"]) / steps,
                           "shadow": (r1["shadow_rays"] - r0["shadow_rays"]) / steps},
        "stages_ms": {k: round(v, 3) for k, v in stages.items() if k.endswith("_ms")},
        "scene_build_s": round(build_s, 3),
        "tuning": tuning,
        "instance_update": dict(upd, note="host wall clock of vt_update_instances for 1024 moved instances, "
                                          "including the top-level upload"),
    }


# ------------------------------------------------------------------ batched workload
def run_batch(args, dev, local, barrier):
    """64 box rooms (triangles log-uniform in [2^12, 2^21], 256^2..1024^2,
    2-8 bounces, 4-32 spp) rendered as one batch (one CUDA graph per batch
    frame, launch shape from the autotuner) against the same frames rendered
    one scene after another through the single-scene engine."""
    from vitrum_b200 import scenes
    from vitrum_b200.batch import Batch, BatchItem
    from vitrum_b200.engine import Engine
    work = scenes.box_room_batch(64)
    items = [BatchItem(sc, cam, w, h, spp, b, frame_seed=100 + i) for i, (sc, cam, w, h, b, spp) in enumerate(work)]
    t0 = time.perf_counter()
    probe = Batch([BatchItem(it.scene, it.camera, it.width, it.height, 4, it.bounces, it.frame_seed) for it in items],
                  device=local)
    trials = probe.autotune()
    tuned = probe.tuning
    probe.close()
    tune_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    b = Batch(items, device=local)
    build_s = time.perf_counter() - t0
    b.set_tuning(tuned["wave_paths"], bool(tuned["sort_by_material"]), tuned["trace_blocks_per_sm"],
                 sort_rays=bool(tuned["sort_rays"]))
    b.render()  # warm-up (graph capture)
    steps = max(1, min(args.steps, 3))
    ms, rays = 0.0, 0
    for _ in range(steps):
        st = b.render()
        ms += st["frame_ms"]
        rays += st["closest_rays"] + st["shadow_rays"]
    waves, launches = st["waves"], st["kernel_launches"]
    b.close()
    # the same frames, one scene at a time, through the engine (set_scene untimed)
    e = Engine(device=local, max_bounces=8)
    seq_ms, seq_rays, seq_launches = 0.0, 0, 0
    for it in items:
        e.set_scene(it.scene)
        e.reset()
        r0 = e.stats()
        e.render_frame(it.camera, it.width, it.height, samples=it.samples, bounces=it.bounces,
                       frame_seed=it.frame_seed)
        r1 = e.stats()
        seq_ms += r1["last_frame_ms"]
        seq_rays += (r1["closest_rays"] - r0["closest_rays"]) + (r1["shadow_rays"] - r0["shadow_rays"])
    e.dispose()
    return {
        "workload": "64 box rooms: triangles log-uniform in [2^12, 2^21] (%d total), resolution from "
                    "{256^2, 512^2, 768^2, 1024^2}, 2-8 bounces, 4-32 spp; %d paths per batch frame"
                    % (sum(it.scene.triangle_count for it in items),
                       sum(it.width * it.height * it.samples for it in items)),
        "value": rays / (ms / 1e3) / 1e6, "unit": "Mrays/s", "ms_per_batch_frame": ms / steps,
        "waves": waves, "kernels_per_batch_frame": launches,
        "sequential": {"value": seq_rays / (seq_ms / 1e3) / 1e6, "unit": "Mrays/s", "ms": seq_ms,
                       "note": "same frames through the single-scene engine, one scene after another"},
        "speedup_vs_sequential": (rays / ms) / (seq_rays / seq_ms) if seq_ms > 0 else None,
        "tuning": tuned, "autotune_trials": trials, "autotune_s": round(tune_s, 1),
        "scene_build_s": round(build_s, 2),
    }


# ------------------------------------------------------------------ radiance cache workload
NRC_SPP, NRC_WARM, NRC_FRAMES, NRC_SEEDS = 16, 8, 64, 5


# RNG keys are frame seed ^ sample index: the oracle's keys [2^20, 2^20 + 2^14)
# share none with the measured sequences' ((s + 1) 2^12 ^ [0, 1024))
ORACLE_SEED = 1 << 20


def _relmse(img, ref, ref_var=None):
    """mean((x - ref)^2 / (ref^2 + 1e-2)); with ref_var (the oracle mean's own
    variance per pixel) its noise is taken out: E(x - ref)^2 = E(x - mu)^2 + ref_var."""
    d2 = (img - ref) ** 2
    if ref_var is not None:
        d2 = d2 - ref_var
    return float(np.mean(d2 / (ref ** 2 + 1e-2)))


_CLOUD_ORACLE = {}


def _cloud_oracle(args, local):
    """The 1024-instance cloud at 1920x1080, 8 bounces, args.oracle_spp samples
    accumulated in FP64, rendered once per run: (mean, variance of the mean,
    seconds)."""
    if "ref" not in _CLOUD_ORACLE:
        from vitrum_b200 import scenes
        from vitrum_b200.engine import Engine
        sc, cam = scenes.instanced_cloud()
        t0 = time.perf_counter()
        o = Engine(device=local, max_bounces=I_BOUNCES, oracle_accumulation=True, max_samples_per_pixel=1 << 20)
        o.set_scene(sc)
        done = 0
        while done < args.oracle_spp:
            k = min(1024, args.oracle_spp - done)
            o.render_frame(cam, I_W, I_H, samples=k, frame_seed=ORACLE_SEED)
            done += k
        ref, var = o.capture_moments()
        o.dispose()
        _CLOUD_ORACLE["ref"] = (ref.astype(np.float32), (var / args.oracle_spp).astype(np.float32),
                                time.perf_counter() - t0)
    return _CLOUD_ORACLE["ref"]


LT_SPP, LT_SEEDS = 64, 16


def run_light_tree(args, dev, local, barrier):
    """Next-event light selection on the 1024-instance cloud with 32 point
    lights at 1920x1080: the light tree (power x proximity x orientation x
    receiver cosine bound, half the buckets spread evenly) against uniform
    selection.  Per selection: the device time of a 16-spp and a 64-spp frame,
    and the relMSE of the 64-spp frame against the FP64 oracle over LT_SEEDS
    seeds (median; also with the 0.1 % worst pixels dropped, the error being
    heavy-tailed through the metal and glass instances).  Equal time: relMSE x
    frame time, lower is better."""
    from vitrum_b200 import scenes
    from vitrum_b200.engine import Engine
    sc, cam = scenes.instanced_cloud()
    ref, rvar, _ = _cloud_oracle(args, local)

    def trimmed(img):
        e = np.sort((((img - ref) ** 2 - rvar) / (ref ** 2 + 1e-2)).ravel())
        return float(e[:int(e.size * 0.999)].mean())

    out = {}
    for sel in ("uniform", "tree"):
        e = Engine(device=local, max_bounces=I_BOUNCES, max_samples_per_pixel=1 << 20, light_selection=sel)
        e.set_scene(sc)
        for i in range(2):
            e.render_frame(cam, I_W, I_H, samples=I_SPP, frame_seed=900 + i)
        full = []
        for i in range(3):
            e.render_frame(cam, I_W, I_H, samples=I_SPP, frame_seed=910 + i)
            full.append(e.stats()["last_frame_ms"])
        e.reset()
        e.render_frame(cam, I_W, I_H, samples=LT_SPP, frame_seed=920)  # the 64-spp frame's graph
        ms, rel, rel_t = [], [], []
        for k in range(1, LT_SEEDS + 1):
            e.reset()
            e.render_frame(cam, I_W, I_H, samples=LT_SPP, frame_seed=k << 16)
            ms.append(e.stats()["last_frame_ms"])
            img = e.capture_frame()[..., :3]
            rel.append(_relmse(img, ref, rvar))
            rel_t.append(trimmed(img))
        e.dispose()
        out[sel] = {"frame_ms_16spp": round(float(np.median(full)), 3),
                    "frame_ms_64spp": round(float(np.median(ms)), 3),
                    "relmse": round(float(np.median(rel)), 6), "relmse_mean": round(float(np.mean(rel)), 6),
                    "relmse_trimmed": round(float(np.median(rel_t)), 6),
                    "relmse_per_seed": [round(r, 6) for r in rel]}
    u, t = out["uniform"], out["tree"]
    cost = t["frame_ms_64spp"] / u["frame_ms_64spp"]
    out["tree_cost_per_sample"] = round(cost, 3)
    out["equal_time_gain"] = round(u["relmse"] / (t["relmse"] * cost), 3)
    out["equal_time_gain_mean"] = round(u["relmse_mean"] / (t["relmse_mean"] * cost), 3)
    out["equal_time_gain_trimmed"] = round(u["relmse_trimmed"] / (t["relmse_trimmed"] * cost), 3)
    out["workload"] = ("1024-instance cloud, 32 point lights + gradient sky, 1920x1080, 8 bounces; relMSE of a "
                       "%d-spp frame vs the %d-spp FP64 oracle (its own variance taken out), %d seeds (median; "
                       "mean beside it)"
                       % (LT_SPP, args.oracle_spp, LT_SEEDS))
    out["metric"] = "equal_time_gain = (relMSE x frame ms) uniform / tree; > 1: the tree wins"
    return out


def run_nrc(args, dev, local, barrier, shape=None):
    """Neural radiance cache against plain path tracing on the 1024-instance
    cloud at 1920x1080, 8 bounces, 16 spp per frame, from a cold start: each
    arm is a fresh engine rendering NRC_FRAMES progressive frames, the NRC
    arm's cache freshly initialised, training online every frame (4 Adam steps
    x 65,536 samples), its first NRC_WARM frames plain path tracing while it
    learns -- all of it charged to its device time.  NRC_SEEDS seeds (frame
    seeds and cache initialisations); per budget (the NRC arm's device time
    after 1, 2, 4, ... frames) the median over seeds of the accumulated image's
    relMSE, plain interpolated to the same time; plus the steady-state
    single-frame relMSE and frame costs.  `shape`: the launch shape the
    instanced leg's autotuner chose for this scene, given to both arms."""
    from vitrum_b200 import scenes
    from vitrum_b200.engine import Engine
    from vitrum_b200.nrc import NrcConfig
    sc, cam = scenes.instanced_cloud()
    ref, rvar, oracle_s = _cloud_oracle(args, local)
    keys = ("wave_paths", "sort_by_material", "trace_blocks_per_sm", "stage_hot_nodes", "sort_rays")
    launch = {k: shape[k] for k in keys} if shape else None

    def arm(nrc, s):
        e = Engine(device=local, max_bounces=I_BOUNCES, max_samples_per_pixel=1 << 20)
        e.set_scene(sc)
        if launch:
            e.set_tuning(**launch)
        if nrc:
            e.set_nrc(prefix_bounces=1, train_steps=4, train_batch=65536, warmup_frames=NRC_WARM,
                      cache=NrcConfig(seed=s + 1))
        t, curve, restart, frame_rel, frame_ms = 0.0, [], [], [], []
        prev = np.zeros_like(ref)
        since = np.zeros_like(ref)  # the frames since the cache took over (all frames for plain)
        for f in range(NRC_FRAMES):
            e.render_frame(cam, I_W, I_H, samples=NRC_SPP, frame_seed=(s + 1) << 12)
            ms = e.stats()["last_frame_ms"]
            t += ms
            acc = e.capture_frame()[..., :3]
            cur = acc * (f + 1) - prev  # this frame's own image
            prev = acc * (f + 1)
            first = NRC_WARM if nrc else 0
            if f >= first:
                since += cur
                restart.append((t, _relmse(since / (f + 1 - first), ref, rvar)))
            curve.append((t, _relmse(acc, ref, rvar)))
            frame_rel.append(_relmse(cur, ref, rvar))
            frame_ms.append(ms)
        stages = e.profile_frame(cam, I_W, I_H, samples=NRC_SPP, frame_seed=(s + 1) << 12) if s == 0 else None
        e.dispose()
        return curve, frame_rel, frame_ms, stages, restart

    def at(pts, t):  # relMSE of the accumulated image at device time t (log-linear interpolation)
        ts = [p[0] for p in pts]
        if t <= ts[0]:
            return pts[0][1] * ts[0] / t  # less than one frame: variance ~ 1 / time
        for (ta, ra), (tb, rb) in zip(pts, pts[1:]):
            if t <= tb:
                w = (t - ta) / (tb - ta)
                return float(np.exp((1 - w) * np.log(max(ra, 1e-12)) + w * np.log(max(rb, 1e-12))))
        return pts[-1][1] * ts[-1] / t

    runs = [(arm(False, s), arm(True, s)) for s in range(NRC_SEEDS)]
    marks = [f for f in (1, 2, 4, 8, 16, 32, 64) if f <= NRC_FRAMES]
    table, table_restart = [], []
    for f in marks:
        b = [nrc[0][f - 1][0] for _, nrc in runs]
        rn = [nrc[0][f - 1][1] for _, nrc in runs]
        rp = [at(plain[0], nrc[0][f - 1][0]) for plain, nrc in runs]
        table.append({"frames": f, "ms": round(float(np.median(b)), 1), "nrc": round(float(np.median(rn)), 5),
                      "plain": round(float(np.median(rp)), 5),
                      "ratio": round(float(np.median([p / n for p, n in zip(rp, rn)])), 2)})
        if f > NRC_WARM:
            rn = [nrc[4][f - 1 - NRC_WARM][1] for _, nrc in runs]
            table_restart.append({"frames": f, "ms": round(float(np.median(b)), 1),
                                  "nrc": round(float(np.median(rn)), 5), "plain": round(float(np.median(rp)), 5),
                                  "ratio": round(float(np.median([p / n for p, n in zip(rp, rn)])), 2)})
    steady = slice(NRC_WARM + 16, NRC_FRAMES)
    pf = {k: float(np.median([np.median(r[i][1][steady]) for r in runs])) for i, k in ((0, "plain"), (1, "nrc"))}
    pm = {k: float(np.median([np.median(r[i][2][steady]) for r in runs])) for i, k in ((0, "plain"), (1, "nrc"))}
    st_plain, st_nrc = runs[0][0][3], runs[0][1][3]
    return {
        "workload": "1024-instance cloud, 1920x1080, 8 bounces, 16 spp per frame, %d frames from a cold start, %d "
                    "seeds; NRC: hash grid 16 x 2^19 x 2 fp16 (base 16, growth 1.5), 64-input MLP 5 x 64 ReLU + 3, "
                    "fp16/fp32-accumulate on tcgen05, 4 Adam steps x 65,536 samples per frame, 1-bounce prefix, "
                    "first %d frames plain while the cache trains (charged); both arms at the instanced leg's "
                    "autotuned launch shape" % (NRC_FRAMES, NRC_SEEDS, NRC_WARM),
        "launch_shape": launch,
        "oracle": {"spp": args.oracle_spp, "accumulation": "fp64", "seconds": round(oracle_s, 1),
                   "note": "its per-pixel variance of the mean is subtracted from every squared error"},
        "metric": "relMSE = mean((x - ref)^2 / (ref^2 + 1e-2)) of the accumulated image at equal device time "
                  "(median over seeds)",
        "equal_time": table,
        "equal_time_restart": table_restart,
        "restart_note": "the NRC arm's image accumulated from the first cache frame on (the warm-up frames shown "
                        "while the cache learns, their time still charged)",
        "steady_frame": {"relmse_plain": round(pf["plain"], 5), "relmse_nrc": round(pf["nrc"], 5),
                         "ms_plain": round(pm["plain"], 2), "ms_nrc": round(pm["nrc"], 2),
                         "equal_time_gain": round(pf["plain"] * pm["plain"] / (pf["nrc"] * pm["nrc"]), 2),
                         "frames": [steady.start, NRC_FRAMES]},
        "full_frame_1920x1080_16spp_ms": {"plain": round(st_plain["frame_ms"], 2),
                                          "nrc": round(st_nrc["frame_ms"], 2),
                                          "nrc_train_ms": round(st_nrc["nrc_train_ms"], 2),
                                          "nrc_query_ms": round(st_nrc["nrc_query_ms"], 2)},
    }


def run_build(args, dev, local):
    """Scene builds (host wall clock, the second of two calls so that module
    loading is not counted): the engine's set_scene with the trees built on the
    GPU (binned-SAH binary tree, SAH-optimal 8-wide encoding, top level)
    against the same words built on the host, for the box room and a
    2,097,152-triangle room; and the reference-facing BVH build of the
    65,536-triangle query soup (vt_bvh_build_device vs vt_bvh_build)."""
    import torch
    from vitrum_b200 import bvh as vb
    from vitrum_b200 import scenes
    from vitrum_b200.engine import Engine
    out = {}

    def scene_ms(sc, build):
        e = Engine(device=local, max_bounces=2, scene_build=build)
        ts = []
        for _ in range(2):
            t0 = time.perf_counter()
            e.set_scene(sc)
            ts.append((time.perf_counter() - t0) * 1e3)
        e.dispose()
        return round(ts[-1], 1)

    for name, sc in (("box_room_262146_tris", scenes.box_room()[0]),
                     ("room_2097152_tris", scenes.box_room_sized(1 << 21)[0])):
        out[name] = {"gpu_ms": scene_ms(sc, "gpu"), "host_ms": scene_ms(sc, "host"),
                     "triangles": int(sc.triangle_count)}
    soup, _ = scenes.config1(Q_TRIS, 16, seed=Q_SEED)
    pos = np.ascontiguousarray(soup.positions, np.float32)
    idx = np.ascontiguousarray(soup.indices, np.uint32)
    dp = torch.from_numpy(pos.reshape(-1)).to(dev)
    di = torch.from_numpy(idx.reshape(-1).view(np.int32)).to(dev)
    g_ms, h_ms = [], []
    for _ in range(2):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        g = vb.build_compressed_wide_bvh_device(dp.data_ptr(), dp.numel(), di.data_ptr(), di.numel(), device=local)
        g_ms.append((time.perf_counter() - t0) * 1e3)
        g.close()
        t0 = time.perf_counter()
        h = vb.build_compressed_wide_bvh(pos, idx, device=local)
        h_ms.append((time.perf_counter() - t0) * 1e3)
        h.close()
    out["query_soup_65536_tris"] = {"gpu_ms": round(g_ms[-1], 1), "host_ms": round(h_ms[-1], 1),
                                    "note": "the reference options' tree (4 per leaf, 16 bins) for export plus the "
                                            "traversal tree (2 per leaf, 32 bins, SAH-optimal 8-wide grouping), "
                                            "incl. the publication proofs on the host copy"}
    return out


# ------------------------------------------------------------------ path tracing workload
def run_ours(args, rank, world, local):
    import torch
    from vitrum_b200 import _native as N
    from vitrum_b200 import scenes
    from vitrum_b200.engine import Engine

    from vitrum_b200.replicas import Group, replica_seed, whole_job_rate
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    group = Group(world, "nccl", dev)
    barrier = group.barrier
    max_over_ranks = group.max

    sc, cam = scenes.box_room()
    e = Engine(device=local, max_bounces=BOUNCES)
    t0 = time.perf_counter()
    e.set_scene(sc)
    build_s = time.perf_counter() - t0

    def frame(seed):
        e.reset()
        e.render_frame(cam, W, H, samples=SPP, frame_seed=seed)

    # tree shape (leaf size, collapse width) and launch shape from the project's
    # autotuners (outside the timed region)
    shape_trials = e.autotune_bvh(sc, cam, W, H, samples=SPP, frame_seed=555) if not args.no_autotune else []
    trials = e.autotune(cam, W, H, samples=SPP, frame_seed=555) if not args.no_autotune else []
    tuning = e.tuning
    for i in range(args.warmup):
        frame(1000 + i)
    # per-stage device times of one frame (profiling path: direct launches, not timed for `value`)
    e.reset()
    stages = e.profile_frame(cam, W, H, samples=SPP, frame_seed=999)
    st_before = e.stats()
    clocks = Clocks(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize(dev)
    frame_ms = []
    rays0 = e.stats()
    for i in range(args.steps):
        frame(replica_seed(rank, i))
        frame_ms.append(e.stats()["last_frame_ms"])
    torch.cuda.synchronize(dev)
    barrier()
    clk = clocks.stop()
    rays1 = e.stats()
    rays = (rays1["closest_rays"] - rays0["closest_rays"]) + (rays1["shadow_rays"] - rays0["shadow_rays"])
    closest = rays1["closest_rays"] - rays0["closest_rays"]
    shadow = rays1["shadow_rays"] - rays0["shadow_rays"]
    dev_s = max_over_ranks(sum(frame_ms) / 1e3)
    value = whole_job_rate(rays, world, dev_s) / 1e6
    samples_per_s = world * W * H * SPP * args.steps / dev_s

    # e2e: public Engine calls, image read back to host every step (into a page-locked array)
    pinned = torch.empty((H, W, 4), dtype=torch.float32).pin_memory().numpy()
    t0 = time.perf_counter()
    for i in range(args.steps):
        frame(replica_seed(rank, i))
        img = e.capture_frame(out=pinned)
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e = world * rays / e2e_s / 1e6

    # the sub-workloads are reported from single-GPU runs (replicas would repeat them)
    solo = world == 1
    query = run_query(args, dev, local, rank, world, barrier) if solo and not args.no_query else None
    instanced = run_instanced(args, dev, local, barrier) if solo and not args.no_instanced else None
    nrc = run_nrc(args, dev, local, barrier, instanced["tuning"] if instanced else None) \
        if solo and not args.no_nrc else None
    light_tree = run_light_tree(args, dev, local, barrier) if solo and not args.no_light_tree else None
    builds = run_build(args, dev, local) if solo and not args.no_build else None
    batch = run_batch(args, dev, local, barrier) if solo and not args.no_batch else None

    if rank == 0:
        vc = _visits()["box_room_pt_512_64spp_5b"]
        per_frame_closest = closest / args.steps
        per_frame_shadow = shadow / args.steps
        alg_bytes = (per_frame_closest * vc["closest_bytes_per_ray"] + per_frame_shadow * vc["shadow_bytes_per_ray"])
        trace_s = (stages["trace_closest_ms"] + stages["trace_shadow_ms"]) / 1e3
        achieved = alg_bytes / trace_s / 1e9
        peak, peak_kind = _peaks()
        launches = stages["trace_closest_launches"]  # one per bounce per wave
        waves = launches // BOUNCES if launches else 0
        kernels_per_frame = waves * (1 + BOUNCES * (5 + (2 if tuning["sort_by_material"] else 0)) + 2)
        cpu = None
        if not args.no_cpu_baseline:
            S, cpu_cam, cpu_build_s = _cpu_pt_scene()
            cpu = cpu_pt_baseline(S, cpu_cam)
            cpu["scene_build_s"] = round(cpu_build_s, 3)
            S.close()
            if query is not None:
                query["cpu_baseline"] = cpu_query_baseline()
        line = {
            "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_s * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (procedural box room)",
            "config": {"workload": WORKLOAD, "parallelism": f"replicas{world}", "resolution": [W, H], "spp": SPP,
                       "max_bounces": BOUNCES, "triangles": sc.triangle_count,
                       "l2": "per-frame wave state ~400 MB > 126 MB L2; BVH L2-resident",
                       "tuning": tuning, "autotune_trials": trials, "bvh_shape_trials": shape_trials,
                       "scene_build_s": round(build_s, 3)},
            "samples_per_s": samples_per_s, "ms_per_frame": dev_s * 1e3 / args.steps,
            "rays_per_frame": {"extension": per_frame_closest, "shadow": per_frame_shadow},
            "stages_ms": {k: round(v, 3) for k, v in stages.items() if k.endswith("_ms")},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": _scaled_traffic(per_frame_closest + per_frame_shadow),
                         "peak_kind": peak_kind, "kernel": "k_trace (extension + shadow launches)",
                         "model": f"extension {vc['closest_bytes_per_ray']:.1f} B/ray, shadow "
                                  f"{vc['shadow_bytes_per_ray']:.1f} B/ray (oracle visit counts)",
                         "trace_ms_per_frame": trace_s * 1e3,
                         "per": "frame (all k_trace launches of one frame)"},
            "e2e": {"value": e2e, "unit": "Mrays/s", "h2d_bytes_per_step": ctypes.sizeof(ctypes.c_float) * 32 + 20,
                    "d2h_bytes_per_step": W * H * 16},
            "gpu_launches": kernels_per_frame * args.steps,
            "clocks": clk,
            "cpu_baseline": cpu,
            "query": query,
            "instanced": instanced,
            "nrc": nrc,
            "light_tree": light_tree,
            "build": builds,
            "batch": batch,
        }
        print(json.dumps(line), flush=True)
    e.dispose()
    group.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-query", action="store_true")
    ap.add_argument("--no-instanced", action="store_true")
    ap.add_argument("--no-nrc", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-light-tree", action="store_true")
    ap.add_argument("--no-build", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--oracle-spp", type=int, default=16384)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank, world, local = _env_rank()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
