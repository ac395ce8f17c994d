"""Benchmark of the B200 ray-tracing hot path (one JSON line on rank 0).

Workload (N=1, per GPU): closest-hit query over 65,536 seeded float32
triangles with 1,048,576 rays per step (tmin 1e-4, tmax +inf), the
shared-bvh build + query configuration.  Metric: Mrays/s (whole job).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

* value: device-resident rays, K launches timed with CUDA events on the
  launching stream, barrier + synchronize on both sides, max over ranks.
  Four ray batches (4 x 48 MB of rays + hits) rotate so the per-step I/O is
  larger than the 126 MB L2 and never cached between steps; the BVH itself
  (3.4 MB) stays L2-resident by design.
* e2e: the same metric through the public host-buffer call
  (vt_bvh_trace_closest): pinned host rays copied in, hits copied out, per step.
* roofline: algorithmic bytes per launch (32 + 16 + 80 V_node + 48 V_tri per
  ray, V counted by the CPU oracle) / average launch time, against the
  measured HBM copy bandwidth.
* --impl reference: the reference algorithm's CPU query (C restatement of
  intersectCompressedWideBvhFirstHit) on all host cores, bounded sample per step.
* N > 1: independent replicas (rays shard across GPUs, no collective): weak scaling.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_TRIS = 65536
N_RAYS = 1 << 20
SEED = 2024
BATCHES = 4
WORKLOAD = "closest-hit query: 65,536 float32 triangles, 1,048,576 rays/step (tmin 1e-4, tmax inf)"
METRIC = "Mrays/s (closest-hit query, 65,536 tris / 1,048,576 rays per step)"


def _env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _traffic():
    """dram read+write bytes per launch of the traversal kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "traverse_closest_config1.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("dram_bytes_per_launch:"):
            return float(line.split(":")[1].split()[0])
    return None


def _visit_model():
    with open(os.path.join(ROOT, "tests", "golden", "visit_counts.json")) as f:
        return json.load(f)["closest_hit_65536_tris_1048576_rays_seed2024"]


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


def cpu_reference(rays: np.ndarray, soup, target_s: float = 8.0):
    """The reference query restated in C (oracle), all host cores, bounded sample."""
    import oracle
    threads = oracle.hw_threads()
    t0 = time.perf_counter()
    w = oracle.build_compressed_wide_bvh(soup.positions, soup.indices)
    build_ms = (time.perf_counter() - t0) * 1e3
    probe = rays[:16384]
    t0 = time.perf_counter()
    oracle.first_hit(w, soup.positions, probe, nthreads=threads)
    rate = probe.shape[0] / (time.perf_counter() - t0)
    n = int(min(rays.shape[0], max(probe.shape[0], rate * target_s)))
    return w, threads, build_ms, n


def run_reference(args, rank, world):
    from vitrum_b200 import scenes
    import oracle
    if rank != 0:
        return
    soup, rays = scenes.config1(N_TRIS, N_RAYS, seed=SEED)
    w, threads, build_ms, n = cpu_reference(rays, soup, target_s=max(2.0, 60.0 / max(1, args.steps + args.warmup)))
    sample = rays[:n]
    for _ in range(args.warmup):
        oracle.first_hit(w, soup.positions, sample, nthreads=threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oracle.first_hit(w, soup.positions, sample, nthreads=threads)
    dt = time.perf_counter() - t0
    value = n * args.steps / dt / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded splitmix64)",
        "config": {"workload": WORKLOAD, "seed": SEED},
        "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": threads, "kind": "port",
                         "sample": f"{n} of {N_RAYS} rays per step; C restatement of shared-bvh "
                                   f"intersectCompressedWideBvhFirstHit (FP64), build {build_ms:.1f} ms"},
        "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local):
    import torch
    import torch.distributed as dist
    from vitrum_b200 import bvh as vb
    from vitrum_b200 import scenes

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    soup, _ = scenes.config1(N_TRIS, 16, seed=SEED)
    g = vb.build_compressed_wide_bvh(soup.positions, soup.indices, device=local)
    info = g.info()
    # per-rank ray batches (distinct seeds per rank and batch)
    host_batches = [scenes.sphere_rays(N_RAYS, seed=SEED + 1 + 1000 * rank + b) for b in range(BATCHES)]
    d_rays = [torch.from_numpy(r).to(dev) for r in host_batches]
    d_hits = [torch.empty((N_RAYS, 4), dtype=torch.int32, device=dev) for _ in range(BATCHES)]
    stream = torch.cuda.current_stream(dev)
    sptr = stream.cuda_stream

    def step(i):
        b = i % BATCHES
        g.trace_closest_device(d_rays[b].data_ptr(), N_RAYS, d_hits[b].data_ptr(), sptr)

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize(dev)

    clocks = Clocks(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize(dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    ev[0].record(stream)
    for i in range(args.steps):
        step(i)
        ev[i + 1].record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    clk = clocks.stop()
    per_launch = [ev[i].elapsed_time(ev[i + 1]) for i in range(args.steps)]
    total_ms = ev[0].elapsed_time(ev[-1])
    t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    value = world * N_RAYS * args.steps / (total_ms / 1e3) / 1e6

    # ---- e2e through the public host-buffer call, pinned host memory
    pin_rays = [torch.from_numpy(r).pin_memory() for r in host_batches]
    pin_hits = torch.empty((N_RAYS, 4), dtype=torch.int32).pin_memory()
    from vitrum_b200 import _native as N
    import ctypes

    def e2e_step(i):
        N.call("vt_bvh_trace_closest", g.handle, ctypes.c_void_p(pin_rays[i % BATCHES].data_ptr()), N_RAYS,
               ctypes.c_void_p(pin_hits.data_ptr()))

    for i in range(max(1, args.warmup)):
        e2e_step(i)
    barrier()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for i in range(args.steps):
        e2e_step(i)
    torch.cuda.synchronize(dev)
    e2e_s = time.perf_counter() - t0
    t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_value = world * N_RAYS * args.steps / float(t.item()) / 1e6

    # check the last hits are sane (no timing)
    hits = pin_hits.numpy()
    hit_frac = float((hits[:, 0] >= 0).mean())

    if rank == 0:
        model = _visit_model()
        avg_launch_s = statistics.mean(per_launch) / 1e3
        bytes_per_launch = model["bytes_per_ray"] * N_RAYS
        achieved = bytes_per_launch / avg_launch_s / 1e9
        peak, peak_kind = _peaks()
        traffic = _traffic()
        cpu = None
        if not args.no_cpu_baseline:
            import oracle
            soup_c, rays_c = scenes.config1(N_TRIS, N_RAYS, seed=SEED)
            w, threads, build_ms, n = cpu_reference(rays_c, soup_c, target_s=8.0)
            sample = rays_c[:n]
            t0 = time.perf_counter()
            oracle.first_hit(w, soup_c.positions, sample, nthreads=threads)
            dt = time.perf_counter() - t0
            cpu = {"value": n / dt / 1e6, "unit": "Mrays/s", "cores": threads, "kind": "port",
                   "sample": f"{n} rays of the same workload; C restatement of shared-bvh "
                             f"intersectCompressedWideBvhFirstHit (FP64); CPU build {build_ms:.1f} ms"}
        line = {
            "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded splitmix64)",
            "config": {"workload": WORKLOAD, "seed": SEED, "parallelism": f"replicas{world}",
                       "l2": "4 rotating ray batches (192 MB rays+hits) > 126 MB L2; BVH L2-resident",
                       "bvh": {"wide_nodes": info["wide_node_count"], "binary_nodes": info["binary_node_count"],
                               "wide_depth": info["wide_depth"], "build_ms_host": round(info["build_ms"], 2)}},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_kind": peak_kind,
                         "model": f"{model['bytes_per_ray']:.1f} B/ray = 48 + 80*{model['v_node']:.3f} + "
                                  f"48*{model['v_tri']:.3f} (oracle near-first counts)",
                         "avg_launch_ms": avg_launch_s * 1e3},
            "e2e": {"value": e2e_value, "unit": "Mrays/s", "h2d_bytes_per_step": N_RAYS * 32,
                    "d2h_bytes_per_step": N_RAYS * 16},
            "gpu_launches": args.steps,
            "clocks": clk,
            "hit_fraction": hit_frac,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    g.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank, world, local = _env_rank()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
