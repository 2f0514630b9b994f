"""Benchmark of the path-tracing hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload trace|render] [--impl ours|reference]

Workloads (seeded synthetic inputs; no public scene set exists):
  render  (default) the many-light 720p render: 1280x720, 64 spp, 6 path
          segments; 2,000 bicubic patches, 500 sphere groups instanced through
          3 assembly levels with transform motion, 10,000 sphere lights sampled
          through the light tree with MIS, depth of field and camera motion.
          A step renders the whole frame (58,982,400 paths).
  trace   ray-stream trace microbenchmark: 4,194,304 rays (half Morton-coherent,
          half shuffled, cosine about -z) against a 256x256 bilinear-patch fBm
          heightfield diced to 8x8 cells per patch; a step traces all rays
          (closest hit id, t, uv).

One JSON line is printed by rank 0.  `value` is device-resident throughput
(inputs in HBM before the timed region), `e2e` the same metric through the
host-array C ABI call (host->device copies of the rays and device->host copies
of the hits inside the timed region).  Multi-GPU runs are independent
replicas of the workload per rank (the path has no exchange step).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_CLOSEST_RAY = 80  # 60 B read (o, d, t_max, time, ray width, id/flags) + 20 B written (id 8, t, u, v)
BYTES_PER_OCCLUSION_RAY = 64
# DRAM bytes per traced ray of the traversal kernel, from the ncu capture in
# profiles/trace_wave_kernel_many_light_640x360x4.md (dram read + write of the
# camera launch / its 921,600 rays)
TRAFFIC_BYTES_PER_RAY = 13396.0
BYTES_PER_PATH_EXTRA = 20   # sampler seed 4 + pixel 4 + XYZ 12
RENDER_RES = (1280, 720)
RENDER_SPP = 64
RENDER_PATH_LENGTH = 6
HEIGHTFIELD_N = 256
TRACE_RAYS = 4194304


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(x: float, pg, device) -> float:
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


# --------------------------------------------------------------------------
# trace workload
# --------------------------------------------------------------------------

def trace_workload():
    from psychopath_cpp_b200 import scenes
    sc = scenes.heightfield_scene(HEIGHTFIELD_N, seed=7)
    rays = scenes.heightfield_rays(TRACE_RAYS, n=HEIGHTFIELD_N, seed=11)
    return sc, rays


def run_trace_ours(args, rank, local, pg, world):
    import torch
    from psychopath_cpp_b200 import api
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    sc, rays = trace_workload()
    ctx = api.Context(local)
    ctx.upload(sc)
    tracer = api.Tracer(ctx)
    n = len(rays["time"])
    d_rays = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in rays.items() if k != "type"}
    d_rays["type"] = torch.from_numpy(rays["type"].astype(np.int16)).to(dev)
    hits = {"hit": torch.empty(n, dtype=torch.uint8, device=dev), "id": torch.empty(n, dtype=torch.int64, device=dev),
            "t": torch.empty(n, dtype=torch.float32, device=dev), "uv": torch.empty(n * 2, dtype=torch.float32, device=dev)}
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    for _ in range(args.warmup):
        tracer.trace_device(d_rays, hits, sp)
    ctx.sync(sp)
    if pg:
        pg.barrier()
    torch.cuda.synchronize(dev)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        start.record(stream)
        for _ in range(args.steps):
            tracer.trace_device(d_rays, hits, sp)
        end.record(stream)
        torch.cuda.synchronize(dev)
    ctx.sync(sp)
    if pg:
        pg.barrier()
    ms = start.elapsed_time(end) / args.steps
    ms = max_over_ranks(ms, pg, dev)
    value = world * n / (ms * 1e-3) / 1e6  # Mrays/s, whole job
    hbm, peak_kind = measured_peaks()
    achieved = BYTES_PER_CLOSEST_RAY * n / (ms * 1e-3) / 1e9
    # end-to-end through the host-array C ABI call (pinned host buffers)
    h_rays = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory().numpy() for k, v in rays.items()}
    out_fields = ("hit", "id", "t", "uv")
    for _ in range(max(1, args.warmup // 2)):
        tracer.trace(h_rays, fields=out_fields)
    torch.cuda.synchronize(dev)
    if pg:
        pg.barrier()
    t0 = time.perf_counter()
    e2e_steps = max(1, min(args.steps, 5))
    for _ in range(e2e_steps):
        tracer.trace(h_rays, fields=out_fields)
    e2e_ms = (time.perf_counter() - t0) * 1e3 / e2e_steps
    e2e_ms = max_over_ranks(e2e_ms, pg, dev)
    h2d = n * (6 * 12 + 4 + 2)
    d2h = n * (1 + 8 + 4 + 8)
    result = {
        "metric": "Mrays/s (ray-stream trace, 4M rays vs 256x256 bilinear heightfield)",
        "value": round(value, 3), "unit": "Mrays/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded fBm heightfield and ray stream)",
        "config": {"workload": "trace: 4,194,304 rays (half coherent) vs 256x256 bilinear patches, 8x8 dicing",
                   "rays_per_step": n, "patches": HEIGHTFIELD_N ** 2, "parallelism": "replicas" if world > 1 else "single",
                   "l2": "inputs (320 MB of rays) larger than L2"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": hbm, "unit": "GB/s",
                     "frac": round(achieved / hbm, 5), "traffic": None, "peak_source": peak_kind,
                     "basis": "80 B per closest-hit ray"},
        "e2e": {"value": round(world * n / (e2e_ms * 1e-3) / 1e6, 3), "unit": "Mrays/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": args.steps,
        "clocks": clk.summary(),
    }
    return result


def trace_cpu_baseline(seconds_target: float = 10.0):
    """The reference's own Tracer::trace (oracle/_ref) on this host's cores, on
    a bounded sample of the trace workload's rays."""
    from oracle import psyref
    if not psyref.available():
        return None
    sc, rays = trace_workload()
    ref = psyref.RefScene(scene=sc)
    threads = os.cpu_count() or 1
    n = len(rays["time"])
    ref.trace(rays, threads=threads, chunk=65536, full=False)  # warm-up
    secs = []
    for _ in range(3):
        secs.append(ref.trace(rays, threads=threads, chunk=65536, full=False)["seconds"])
    s = max(min(secs), 1e-9)
    s1 = ref.trace(rays, threads=1, chunk=65536, full=False)["seconds"]
    return {"value": round(n / s / 1e6, 4), "unit": "Mrays/s", "cores": threads, "kind": "reference",
            "cpu_model": cpu_model(),
            "sample": "the whole 4,194,304-ray stream, Tracer::trace in 65,536-ray chunks on %d threads, "
                      "best of 3" % threads,
            "one_core": {"value": round(n / max(s1, 1e-9) / 1e6, 4), "unit": "Mrays/s", "cores": 1,
                         "sample": "the whole stream once on 1 thread"}}


# --------------------------------------------------------------------------
# render workload
# --------------------------------------------------------------------------

def render_workload():
    from psychopath_cpp_b200 import scenes
    return scenes.many_light_scene(3, res=RENDER_RES, spp=RENDER_SPP)


RENDER_METRIC = "paths/s at 720p (1280x720, 64 spp, 6 segments, many-light scene)"


def render_workload_name():
    return ("render: %dx%d x %d spp, %d segments; 2,000 bicubic patches, 500 sphere groups through 3 assembly levels "
            "with transform motion, 10,000 sphere lights (light tree + MIS), DoF, camera motion"
            % (RENDER_RES[0], RENDER_RES[1], RENDER_SPP, RENDER_PATH_LENGTH))


def run_render_ours(args, rank, local, pg, world):
    import torch
    from psychopath_cpp_b200 import api
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    sc = render_workload()
    ctx = api.Context(local)
    ctx.upload(sc)
    w, h = RENDER_RES
    integ = api.PathTraceIntegrator(ctx, w, h, RENDER_SPP, seed=1, path_length=RENDER_PATH_LENGTH,
                                    stream_paths=args.stream_paths)
    xyz = torch.zeros(w * h * 3, dtype=torch.float32, device=dev)
    cnt = torch.zeros(w * h, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    for _ in range(args.warmup):
        integ.integrate_device(xyz, cnt, sp, with_stats=False)
    integ.integrate_device(xyz, cnt, sp, with_stats=True)  # rays and launches of one render
    rays_per_render = int(integ.stats.rays)
    occl_per_render = int(integ.stats.occlusion_rays)
    launches_per_render = int(integ.stats.launches)
    # every wave launches one closest-hit and one occlusion traversal per segment
    trace_launches_per_render = int(integ.stats.waves) * 2 * RENDER_PATH_LENGTH
    counters = ctx.trace_counters()
    paths = w * h * RENDER_SPP
    if pg:
        pg.barrier()
    torch.cuda.synchronize(dev)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # the traversal kernels (the dominant ones) are timed by the library with
    # CUDA events on the render stream around each of their launches
    ctx.check(ctx.L.psy_profile_enable(ctx.h, 1))
    with ClockSampler(local) as clk:
        start.record(stream)
        for _ in range(args.steps):
            integ.integrate_device(xyz, cnt, sp, with_stats=False)
        end.record(stream)
        torch.cuda.synchronize(dev)
    trace_ms, trace_launches = C.c_double(), C.c_uint32()
    ctx.check(ctx.L.psy_profile_read(ctx.h, C.byref(trace_ms), C.byref(trace_launches)))
    ctx.check(ctx.L.psy_profile_enable(ctx.h, 0))
    ctx.sync(sp)
    if pg:
        pg.barrier()
    ms = start.elapsed_time(end) / args.steps
    ms = max_over_ranks(ms, pg, dev)
    value = world * paths / (ms * 1e-3)
    mrays = world * rays_per_render / (ms * 1e-3) / 1e6
    rbar = rays_per_render / paths
    hbm, peak_kind = measured_peaks()
    # roofline of the traversal kernels: their algorithmic bytes (80 B per
    # closest-hit ray, 64 B per occlusion ray) over their own launch time
    closest = rays_per_render - occl_per_render
    trace_bytes = (closest * BYTES_PER_CLOSEST_RAY + occl_per_render * BYTES_PER_OCCLUSION_RAY) * args.steps
    n_trace = int(trace_launches.value)
    if n_trace != trace_launches_per_render * args.steps:
        raise RuntimeError("timed %d traversal launches, expected %d x %d steps" %
                           (n_trace, trace_launches_per_render, args.steps))
    achieved = trace_bytes / (trace_ms.value * 1e-3) / 1e9 if trace_ms.value > 0 else 0.0
    traffic = TRAFFIC_BYTES_PER_RAY * rays_per_render * args.steps / n_trace
    # end to end: the public call plus the device->host read of the film each step
    h_xyz = torch.empty(w * h * 3, dtype=torch.float32, pin_memory=True)
    h_cnt = torch.empty(w * h, dtype=torch.int32, pin_memory=True)
    torch.cuda.synchronize(dev)
    if pg:
        pg.barrier()
    e2e_steps = max(1, min(args.steps, 3))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        integ.integrate_device(xyz, cnt, sp, with_stats=False)
        h_xyz.copy_(xyz, non_blocking=True)
        h_cnt.copy_(cnt, non_blocking=True)
        torch.cuda.synchronize(dev)
    e2e_ms = (time.perf_counter() - t0) * 1e3 / e2e_steps
    e2e_ms = max_over_ranks(e2e_ms, pg, dev)
    ctx.sync(sp)
    return {
        "metric": RENDER_METRIC, "value": round(value, 1), "unit": "paths/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded many-light scene)",
        "config": {"workload": render_workload_name(), "paths_per_step": paths, "path_length": RENDER_PATH_LENGTH,
                   "stream_paths": args.stream_paths or "auto (2^21)",
                   "parallelism": "replicas" if world > 1 else "single",
                   "l2": "per-path state (~200 B x 2M paths in flight) larger than L2"},
        "mrays_per_s": round(mrays, 2), "rays_per_path": round(rbar, 4),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": hbm, "unit": "GB/s",
                     "frac": round(achieved / hbm, 5), "traffic": round(traffic),
                     "kernel": "trace_wave_kernel (closest-hit and occlusion traversal)",
                     "algorithmic_bytes_per_launch": round(trace_bytes / n_trace),
                     "avg_launch_ms": round(trace_ms.value / n_trace, 4), "launches_timed": n_trace,
                     "share_of_step": round(trace_ms.value / args.steps / ms, 3), "peak_source": peak_kind,
                     "basis": "80 B per closest-hit ray, 64 B per occlusion ray; traffic: DRAM bytes per launch "
                              "scaled from one ncu capture by rays (profiles/)"},
        "e2e": {"value": round(world * paths / (e2e_ms * 1e-3), 1), "unit": "paths/s",
                "h2d_bytes_per_step": 28, "d2h_bytes_per_step": w * h * 16},
        "gpu_launches": launches_per_render * args.steps,
        "clocks": clk.summary(),
        "traversal_counters": per_ray_counters(counters),
    }


def per_ray_counters(c: dict) -> dict:
    """Traversal work per ray of one render (psy_profile_counters): node
    visits, leaf visits and patch bisection iterations per ray, and the lanes
    of 32 that ran work per traversal warp-loop iteration."""
    out = {}
    for kind in ("closest", "occlusion"):
        k = c[kind]
        n = max(1, k["rays"])
        out[kind] = {"rays": k["rays"], "node_visits_per_ray": round(k["node_visits"] / n, 2),
                     "leaf_visits_per_ray": round(k["leaf_visits"] / n, 2),
                     "patch_iterations_per_ray": round(k["patch_iterations"] / n, 2),
                     "lanes_per_warp_step": round(k["lane_steps"] / max(1, k["warp_steps"]), 2)}
    return out


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _ref_render_child(q, res, spp, path_length, threads):
    from psychopath_cpp_b200 import scenes
    from oracle import psyref
    ref = psyref.RefScene(scene=scenes.many_light_scene(3, res=res, spp=spp))
    _, _, rays, secs = ref.render(threads=threads, spp=spp, path_length=path_length, seed=1)
    q.put((rays, secs))


def ref_render_bounded(spp: int, limit_s: float = 240.0, threads: int = 0):
    """The reference's render of the frame at `spp` in a child process (spawned,
    so no CUDA state is inherited) with a time limit: a ray with NaN
    differentials makes the reference's patch bisection run without end, so a
    sample that meets one never returns.  Returns (rays, seconds) or None."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_ref_render_child,
                    args=(q, RENDER_RES, spp, RENDER_PATH_LENGTH, threads or os.cpu_count() or 1))
    p.start()
    p.join(limit_s)
    if p.is_alive():
        p.kill()
        p.join()
        return None
    return q.get() if not q.empty() else None


def render_cpu_baseline(spp: int = 4):
    """The reference's PathTraceIntegrator::integrate (oracle/_ref) on this
    host's cores over a bounded sample of the render: the full frame at a
    few samples per pixel (fewer if the reference does not finish)."""
    from oracle import psyref
    if not psyref.available():
        return None
    threads = os.cpu_count() or 1
    out = None
    while spp >= 1 and out is None:
        out = ref_render_bounded(spp)
        if out is None:
            spp //= 2
    if out is None:
        return None
    rays, secs = out
    paths = RENDER_RES[0] * RENDER_RES[1] * spp
    res = {"value": round(paths / secs, 1), "unit": "paths/s", "cores": threads, "kind": "reference",
           "mrays_per_s": round(rays / secs / 1e6, 3), "cpu_model": cpu_model(),
           "sample": "the %dx%d frame at %d spp (%d paths) instead of %d, PathTraceIntegrator::integrate on "
                     "%d threads" % (RENDER_RES[0], RENDER_RES[1], spp, paths, RENDER_SPP, threads)}
    # the same on one core, over the frame at 1 spp
    one = ref_render_bounded(1, limit_s=300.0, threads=1)
    if one is not None:
        p1 = RENDER_RES[0] * RENDER_RES[1]
        res["one_core"] = {"value": round(p1 / one[1], 1), "unit": "paths/s", "cores": 1,
                           "mrays_per_s": round(one[0] / one[1] / 1e6, 3),
                           "sample": "the %dx%d frame at 1 spp (%d paths) on 1 thread" % (RENDER_RES[0],
                                                                                       RENDER_RES[1], p1)}
    return res


def run_render_reference(args, spp: int = 2):
    from oracle import psyref
    if not psyref.available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libpsyref.so (the reference built from source) is missing"}
    threads = os.cpu_count() or 1
    paths = RENDER_RES[0] * RENDER_RES[1] * spp
    tot, rays = 0.0, 0
    for k in range(args.warmup + args.steps):
        out = ref_render_bounded(spp)
        if out is None:
            return {"impl": "reference", "unavailable": "the reference's render of the frame at %d spp did not finish "
                                                         "within 240 s (NaN ray differentials stall its patch "
                                                         "bisection)" % spp}
        if k >= args.warmup:
            rays += out[0]
            tot += out[1]
    ms = tot * 1e3 / args.steps
    value = paths / (ms * 1e-3)
    return {"metric": RENDER_METRIC, "impl": "reference", "value": round(value, 1), "unit": "paths/s", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded many-light scene)",
            "config": {"workload": render_workload_name(), "sample_paths_per_step": paths},
            "mrays_per_s": round(rays / tot / 1e6, 3),
            "cpu_baseline": {"value": round(value, 1), "unit": "paths/s", "cores": threads, "kind": "reference",
                             "cpu_model": cpu_model(),
                             "sample": "the %dx%d frame at %d spp per step (%d paths), PathTraceIntegrator::"
                                       "integrate on %d threads" % (RENDER_RES[0], RENDER_RES[1], spp, paths,
                                                                    threads)},
            "e2e": {"value": round(value, 1), "unit": "paths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_trace_reference(args):
    from oracle import psyref
    if not psyref.available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libpsyref.so (the reference built from source) is missing"}
    sc, rays = trace_workload()
    ref = psyref.RefScene(scene=sc)
    threads = os.cpu_count() or 1
    sample = len(rays["time"])
    sub = rays
    for _ in range(args.warmup):
        ref.trace(sub, threads=threads, chunk=65536, full=False)
    t0 = time.perf_counter()
    inner = 0.0
    for _ in range(args.steps):
        inner += ref.trace(sub, threads=threads, chunk=65536, full=False)["seconds"]
    wall = time.perf_counter() - t0
    ms = wall * 1e3 / args.steps
    value = sample / (ms * 1e-3) / 1e6
    return {"metric": "Mrays/s (ray-stream trace, 4M rays vs 256x256 bilinear heightfield)", "impl": "reference",
            "value": round(value, 4), "unit": "Mrays/s", "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded fBm heightfield and ray stream)",
            "config": {"workload": "trace: 4,194,304 rays (half coherent) vs 256x256 bilinear patches, 8x8 dicing",
                       "rays_per_step": sample},
            "cpu_baseline": {"value": round(value, 4), "unit": "Mrays/s", "cores": threads, "kind": "reference",
                             "sample": "all %d rays per step, Tracer::trace in 65,536-ray chunks" % sample},
            "e2e": {"value": round(value, 4), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


BATCH_METRIC = "paths/s batched (48 renders, one persistent wave stream + CUDA graph) vs plain (one render at a time)"


def run_batch_ours(args, rank, local, pg, world):
    """48 independent renders of uneven size: psy_render_batch (autotuned
    wave length and block size, CUDA graph) against psy_render called once
    per render, both timed with CUDA events over whole passes."""
    import torch
    from psychopath_cpp_b200 import api, scenes
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    cfgs = scenes.batch_configs(48, seed=0)
    ctxs, entries = [], []
    # scene build and upload, the root's BVH4 and light tree built on the
    # device against the host build (library call only, the fastest of two
    # per scene); both builds give the same trees, and the renders below run
    # on the device-built ones
    build = {"device_s": 0.0, "host_s": 0.0, "device_bvh4_nodes": 0, "device_light_nodes": 0}
    for c in cfgs:
        ctx = api.Context(local)
        flat = api.flatten(scenes.batch_scene(c["seed"], c["res"], c["spp"], c["n_prims"], c["n_lights"]))
        build["host_s"] += min(ctx.upload_flat(flat) for _ in range(2))
        build["device_s"] += min(ctx.upload_flat(flat, gpu_bvh=True) for _ in range(2))
        st = ctx.stats()
        build["device_bvh4_nodes"] += st["gpu_bvh4_nodes"]
        build["device_light_nodes"] += st["gpu_light_nodes"]
        del flat
        ctxs.append(ctx)
        entries.append({"scene": ctx, "width": c["res"][0], "height": c["res"][1], "spp": c["spp"],
                        "seed": c["seed"] + 1, "path_length": 4})
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    paths = sum(e["width"] * e["height"] * e["spp"] for e in entries)
    # plain: one psy_render per render
    integs = [api.PathTraceIntegrator(e["scene"], e["width"], e["height"], e["spp"], seed=e["seed"], path_length=4)
              for e in entries]
    films = [(torch.zeros(e["width"] * e["height"] * 3, dtype=torch.float32, device=dev),
              torch.zeros(e["width"] * e["height"], dtype=torch.int32, device=dev)) for e in entries]

    def plain_pass():
        for it, (x, c) in zip(integs, films):
            it.integrate_device(x, c, sp, with_stats=False)

    def timed(fn, steps):
        torch.cuda.synchronize(dev)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        for _ in range(steps):
            fn()
        e.record(stream)
        torch.cuda.synchronize(dev)
        return s.elapsed_time(e) / steps

    log = lambda *a: print(*a, file=sys.stderr, flush=True)
    log("batch: %d renders, %d paths per pass" % (len(entries), paths))
    for _ in range(args.warmup):
        plain_pass()
    plain_ms = timed(plain_pass, args.steps)
    log("batch: plain pass %.1f ms" % plain_ms)
    # each render alone (one pass, CUDA events around each), so that the
    # plain rate can be taken over any subset of the renders
    torch.cuda.synchronize(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in entries]
    for (a, z), it, (x, c) in zip(ev, integs, films):
        a.record(stream)
        it.integrate_device(x, c, sp, with_stats=False)
        z.record(stream)
    torch.cuda.synchronize(dev)
    per_render_ms = [a.elapsed_time(z) for a, z in ev]
    per_render_paths = [e["width"] * e["height"] * e["spp"] for e in entries]
    owner = api.Context(local)
    b = api.BatchRenderer(owner, entries, use_graph=False)
    tune = b.autotune(spp_divisor=16)
    log("batch: tuned %r" % tune)
    b = api.BatchRenderer(owner, entries, use_graph=True)
    for _ in range(args.warmup):
        b.render(sp, with_stats=False)
    b.render(sp, with_stats=True)
    launches = int(b.stats.launches)
    rays = int(b.stats.rays)
    with ClockSampler(local) as clk:
        batch_ms = timed(lambda: b.render(sp, with_stats=False), args.steps)
    owner.sync(sp)
    value = paths / (batch_ms * 1e-3)
    plain_value = paths / (plain_ms * 1e-3)
    hbm, peak_kind = measured_peaks()
    rbar = rays / paths
    achieved = (rbar * BYTES_PER_CLOSEST_RAY + BYTES_PER_PATH_EXTRA) * paths / (batch_ms * 1e-3) / 1e9
    return {
        "metric": BATCH_METRIC, "value": round(value, 1), "unit": "paths/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(batch_ms, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (48 seeded scenes: spheres + bilinear patches)",
        "config": {"workload": "batch: 48 renders, 64x64..1024x768, 8-128 spp, 10-50,000 primitives, 1-100 lights, "
                               "4 segments", "paths_per_step": paths, "tuned": tune,
                   "l2": "per-wave path state larger than L2"},
        "plain_paths_per_s": round(plain_value, 1), "plain_ms_per_step": round(plain_ms, 3),
        "plain_per_render": {"ms": [round(x, 3) for x in per_render_ms], "paths": per_render_paths},
        "batched_over_plain": round(value / plain_value, 3), "mrays_per_s": round(rays / (batch_ms * 1e-3) / 1e6, 2),
        "scene_build": {"scenes": len(cfgs), "host_s": round(build["host_s"], 4),
                        "device_s": round(build["device_s"], 4),
                        "device_bvh4_nodes": build["device_bvh4_nodes"],
                        "device_light_nodes": build["device_light_nodes"],
                        "basis": "psy_scene_upload vs psy_scene_upload_ex(PSY_UPLOAD_GPU_BVH) per scene, "
                                 "library call (scene build and copies to the device, the Python flattening "
                                 "left out), fastest of 2"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": hbm, "unit": "GB/s",
                     "frac": round(achieved / hbm, 5), "traffic": None, "peak_source": peak_kind,
                     "basis": "R*80 + 20 B per path (R = rays per path)"},
        "gpu_launches": launches * args.steps, "clocks": clk.summary(),
    }


def _ref_batch_child(q, start, passes):
    """Renders batch scenes start.. in order, each `passes` times at 1 spp,
    and reports each scene's passes as soon as they are done."""
    from oracle import psyref
    from psychopath_cpp_b200 import scenes
    threads = os.cpu_count() or 1
    cfgs = scenes.batch_configs(48, seed=0)
    for i in range(start, len(cfgs)):
        c = cfgs[i]
        ref = psyref.RefScene(scene=scenes.batch_scene(c["seed"], c["res"], 1, c["n_prims"], c["n_lights"]))
        out = []
        for _ in range(passes):
            _, _, r, t = ref.render(threads=threads, spp=1, path_length=4, seed=c["seed"] + 1)
            out.append((c["res"][0] * c["res"][1], r, t))
        q.put((i, out))
    q.put(None)


def ref_batch_bounded(passes: int, scene_limit_s: float = 30.0):
    """The reference's PathTraceIntegrator::integrate over the 48 batch
    renders, each at 1 spp, `passes` times, in spawned child processes.  A
    scene whose renders do not finish within scene_limit_s (a ray with NaN
    differentials makes the reference's patch bisection run without end) is
    left out: its child is stopped and a new one carries on with the next
    scene.  Returns ([(paths, rays, seconds)] per pass, [left-out scenes])."""
    import multiprocessing as mp
    import queue as queue_mod
    ctx = mp.get_context("spawn")
    per_pass = [[0, 0, 0.0] for _ in range(passes)]
    skipped = []
    start = 0
    while start < 48:
        q = ctx.Queue()
        p = ctx.Process(target=_ref_batch_child, args=(q, start, passes))
        p.start()
        while True:
            try:
                item = q.get(timeout=scene_limit_s)
            except queue_mod.Empty:
                p.kill()
                p.join()
                skipped.append(start)
                start += 1
                break
            if item is None:
                p.join()
                start = 48
                break
            i, out = item
            for k, (paths, rays, secs) in enumerate(out):
                per_pass[k][0] += paths
                per_pass[k][1] += rays
                per_pass[k][2] += secs
            start = i + 1
    return [tuple(x) for x in per_pass], skipped


def _batch_sample(threads, skipped):
    s = "the 48 renders at 1 spp each, one after another, PathTraceIntegrator::integrate on %d threads" % threads
    if skipped:
        s += ("; left out: render(s) %s, whose reference render did not finish within 30 s (NaN ray differentials "
              "stall its patch bisection)" % ", ".join(str(k) for k in skipped))
    return s


def batch_cpu_baseline():
    from oracle import psyref
    if not psyref.available():
        return None
    out, skipped = ref_batch_bounded(1)
    paths, rays, secs = out[0]
    if secs <= 0.0:
        return None
    threads = os.cpu_count() or 1
    return {"value": round(paths / secs, 1), "unit": "paths/s", "cores": threads, "kind": "reference",
            "mrays_per_s": round(rays / secs / 1e6, 3), "sample": _batch_sample(threads, skipped),
            "left_out": list(skipped), "cpu_model": cpu_model()}


def run_batch_reference(args):
    """The reference has no batched renderer: its arm renders the 48 scenes
    one after another with PathTraceIntegrator, each at 1 spp per step."""
    from oracle import psyref
    if not psyref.available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libpsyref.so (the reference built from source) is missing"}
    out, skipped = ref_batch_bounded(args.warmup + args.steps)
    timed_passes = out[args.warmup:]
    paths = sum(o[0] for o in timed_passes)
    rays = sum(o[1] for o in timed_passes)
    secs = sum(o[2] for o in timed_passes)
    threads = os.cpu_count() or 1
    if secs <= 0.0:
        return {"impl": "reference", "unavailable": "none of the reference's batch renders finished"}
    value = paths / secs
    return {"metric": BATCH_METRIC, "impl": "reference", "value": round(value, 1), "unit": "paths/s", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(secs * 1e3 / args.steps, 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (48 seeded scenes: spheres + bilinear patches)",
            "config": {"workload": "batch: 48 renders, 64x64..1024x768, 10-50,000 primitives, 1-100 lights, "
                                   "4 segments", "sample_paths_per_step": paths // args.steps},
            "mrays_per_s": round(rays / secs / 1e6, 3),
            "cpu_baseline": {"value": round(value, 1), "unit": "paths/s", "cores": threads, "kind": "reference",
                             "sample": _batch_sample(threads, skipped)},
            "e2e": {"value": round(value, 1), "unit": "paths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_adjoint_reference(args):
    return {"impl": "reference", "unavailable": "the reference has no differentiable render or adjoint (it shades "
                                                "fixed RGB albedos and emission)"}


ADJOINT_METRIC = "adjoint/forward time ratio (path-replay adjoint vs differentiable forward render)"


def run_adjoint_ours(args, rank, local, pg, world):
    """Differentiable render at 256x256, 32 spp, 4 segments (the plain
    scene's geometry with 8 lights; 256 albedo weights + 8 emission scales)
    and its path-replay adjoint for an L2 image loss, timed with CUDA events."""
    import numpy as np
    import torch
    from psychopath_cpp_b200 import api, scenes
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    res, spp = (256, 256), 32
    sc = scenes.adjoint_scene(1, res=res, spp=spp)
    ctx = api.Context(local)
    ctx.upload(sc)
    shaders, objects, ns, no = api.flat_indices(sc)
    sp = np.full(ns, -1, np.int32)
    op = np.full(no, -1, np.int32)
    count = 0
    init = []
    for name in sorted((n for n in sc.root.shaders if n.startswith("mat")), key=lambda n: int(n[3:])):
        sp[shaders[id(sc.root.shaders[name])]] = count
        init += [0.8 * float(sc.root.shaders[name].color[0])] * 4
        count += 4
    for name in sorted((n for n in sc.root.objects if n.startswith("light")), key=lambda n: int(n[5:])):
        op[objects[(0, name)]] = count
        init.append(1.0)
        count += 1
    r = api.DiffRenderer(ctx, res[0], res[1], spp, sp, op, count, seed=1, path_length=4)
    params = torch.tensor(init, dtype=torch.float32, device=dev)
    rng = np.random.default_rng(0)
    target_p = params + torch.from_numpy(rng.normal(0, 0.1, count).astype(np.float32)).to(dev)
    tx, tc = r.forward(target_p)
    target = tx.view(-1, 3) / tc.view(-1, 1).float()
    stream = torch.cuda.current_stream(dev)
    sp_ = stream.cuda_stream
    xyz = torch.zeros(res[0] * res[1] * 3, dtype=torch.float32, device=dev)
    cnt = torch.zeros(res[0] * res[1], dtype=torch.int32, device=dev)
    grad = torch.zeros(count, dtype=torch.float32, device=dev)

    def fwd():
        xyz.zero_()
        cnt.zero_()
        r.forward(params, xyz, cnt, sp_)

    def adj():
        img = xyz.view(-1, 3) / cnt.view(-1, 1).float()
        dl = (2.0 * (img - target) / cnt.view(-1, 1).float()).reshape(-1)
        grad.zero_()
        r.adjoint(params, dl, grad, sp_)

    def timed(fn, steps):
        torch.cuda.synchronize(dev)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        for _ in range(steps):
            fn()
        e.record(stream)
        torch.cuda.synchronize(dev)
        return s.elapsed_time(e) / steps

    for _ in range(args.warmup):
        fwd()
        adj()
    with ClockSampler(local) as clk:
        f_ms = timed(fwd, args.steps)
        a_ms = timed(adj, args.steps)
    paths = res[0] * res[1] * spp
    return {
        "metric": ADJOINT_METRIC, "value": round(a_ms / f_ms, 4), "unit": "x", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(a_ms, 3), "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded plain scene, 8 lights)",
        "config": {"workload": "adjoint: 256x256, 32 spp, 4 segments, 256 albedo weights + 8 emission scales, "
                               "L2 image loss", "paths_per_step": paths, "l2": "per-wave path state larger than L2"},
        "forward_ms": round(f_ms, 3), "adjoint_ms": round(a_ms, 3),
        "forward_paths_per_s": round(paths / (f_ms * 1e-3), 1), "clocks": clk.summary(),
    }


def run_batch_small(local) -> dict:
    """Many small renders (previews): 48 renders of 64x64 to 256x192 at 4 to
    16 spp, 100 to 5,000 primitives, psy_render_batch (autotuned, graph)
    against one psy_render per render, each timed over 5 passes with CUDA
    events.  This is the case batching is for: one render alone leaves most
    of the GPU idle."""
    import torch
    from psychopath_cpp_b200 import api, scenes
    dev = torch.device("cuda", local)
    rng = np.random.default_rng(5)
    entries = []
    for i in range(48):
        res = [(64, 64), (128, 96), (160, 120), (256, 192)][i % 4]
        spp = int(rng.choice([4, 8, 16]))
        ctx = api.Context(local)
        ctx.upload(scenes.batch_scene(100 + i, res, spp, int(rng.integers(100, 5000)), int(rng.integers(1, 20))))
        entries.append({"scene": ctx, "width": res[0], "height": res[1], "spp": spp, "seed": i + 1, "path_length": 4})
    paths = sum(e["width"] * e["height"] * e["spp"] for e in entries)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    integs = [api.PathTraceIntegrator(e["scene"], e["width"], e["height"], e["spp"], seed=e["seed"], path_length=4)
              for e in entries]
    films = [(torch.zeros(e["width"] * e["height"] * 3, device=dev),
              torch.zeros(e["width"] * e["height"], dtype=torch.int32, device=dev)) for e in entries]

    def plain():
        for it, (x, c) in zip(integs, films):
            it.integrate_device(x, c, sp, with_stats=False)

    def timed(fn, n=5):
        torch.cuda.synchronize(dev)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        for _ in range(n):
            fn()
        e.record(stream)
        torch.cuda.synchronize(dev)
        return s.elapsed_time(e) / n

    for _ in range(2):
        plain()
    plain_ms = timed(plain)
    owner = api.Context(local)
    b = api.BatchRenderer(owner, entries, use_graph=True)
    tune = b.autotune(spp_divisor=1)
    rb = lambda: b.render(sp, with_stats=False)
    for _ in range(2):
        rb()
    batch_ms = timed(rb)
    return {"value": round(plain_ms / batch_ms, 3), "batched_paths_per_s": round(paths / (batch_ms * 1e-3), 1),
            "plain_paths_per_s": round(paths / (plain_ms * 1e-3), 1), "paths": paths, "tuned": tune,
            "workload": "48 small renders: 64x64..256x192, 4-16 spp, 100-5,000 primitives, 1-19 lights, 4 segments",
            "steps": 5}


def render_line_extras(args, rank, local, pg, world) -> dict:
    """The other two figures of the headline metric, measured after the
    render's timed region, each with its own CUDA events and clock record:
    batched over plain paths/s (48 renders) and adjoint over forward time."""
    small = argparse.Namespace(**vars(args))
    small.steps, small.warmup = 1, 1
    out = {}
    b = run_batch_ours(small, rank, local, pg, world)
    out["batched_over_plain"] = {"value": b["batched_over_plain"], "batched_paths_per_s": b["value"],
                                 "plain_paths_per_s": b["plain_paths_per_s"], "workload": b["config"]["workload"],
                                 "steps": 1, "clocks": b["clocks"], "scene_build": b["scene_build"]}
    out["batched_over_plain"]["small_renders"] = run_batch_small(local)
    small.steps, small.warmup = 10, 3
    a = run_adjoint_ours(small, rank, local, pg, world)
    out["adjoint_over_forward"] = {"value": a["value"], "forward_ms": a["forward_ms"], "adjoint_ms": a["adjoint_ms"],
                                   "workload": a["config"]["workload"], "steps": 10, "clocks": a["clocks"]}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="render", choices=["render", "trace", "batch", "adjoint"])
    ap.add_argument("--stream-paths", type=int, default=0)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="render workload: leave out the batched/plain and adjoint/forward figures")
    ap.add_argument("--render-size", default="",
                    help="WxHxSPP: a smaller frame of the render workload (profiling captures); not a bench line")
    args = ap.parse_args()
    if args.render_size:
        global RENDER_RES, RENDER_SPP
        w, h, spp = (int(x) for x in args.render_size.lower().split("x"))
        RENDER_RES, RENDER_SPP = (w, h), spp
    args.warmup = max(3, args.warmup)
    world, rank, local, pg = dist_setup(args)
    if args.impl == "reference":
        if rank == 0:
            fn = {"render": run_render_reference, "trace": run_trace_reference, "batch": run_batch_reference,
                  "adjoint": run_adjoint_reference}[args.workload]
            print(json.dumps(fn(args)))
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return
    if args.workload == "render":
        res = run_render_ours(args, rank, local, pg, world)
        if world == 1 and not args.no_extras and not args.render_size:
            res.update(render_line_extras(args, rank, local, pg, world))
    elif args.workload == "batch":
        res = run_batch_ours(args, rank, local, pg, world)
    elif args.workload == "adjoint":
        res = run_adjoint_ours(args, rank, local, pg, world)
    else:
        res = run_trace_ours(args, rank, local, pg, world)
    if rank == 0:
        if world == 1 and not args.no_cpu_baseline and args.workload in ("render", "trace", "batch"):
            res["cpu_baseline"] = {"render": render_cpu_baseline, "trace": trace_cpu_baseline,
                                   "batch": batch_cpu_baseline}[args.workload]()
            cb = res["cpu_baseline"]
            if args.workload == "batch" and cb and cb.get("left_out"):
                # the plain GPU rate over the renders the reference sample kept
                pr = res["plain_per_render"]
                keep = [i for i in range(len(pr["ms"])) if i not in cb["left_out"]]
                res["plain_paths_per_s_reference_subset"] = round(
                    sum(pr["paths"][i] for i in keep) / (sum(pr["ms"][i] for i in keep) * 1e-3), 1)
        print(json.dumps(res))
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
