"""Benchmark of the render hot path on B200 (one process per GPU).

Workload (default): the full-frame scene -- a 64x64 grid of displaced
spheres (2,064,418 triangles with ground and 16 quad lights; 50% Lambert,
30% glossy, 20% mirror), 1920x1080, max depth 16, NEE+MIS, Russian roulette
from depth 3, firefly clamp 10, FP32.  One step = one sample of every pixel
(2,073,600 camera paths), rendered through the wavefront kernels with the
scene and BVH resident in HBM.  metric = camera paths per second.

The line also carries: e2e (the same metric through the public C-ABI call
with host buffers, film read back every step), the ray-query workload
(8,388,608 rays on the 1,046,904-triangle sphere, Mrays/s), the traversal
roofline of the dominant kernel, nvidia-smi clocks during the timed region,
and the reference CPU tracer timed on this host (cpu_baseline).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from vkpathtracer_b200 import scenes  # noqa: E402

METRIC = "paths/s"
UNIT = "paths/s"
WORKLOAD = "sphere_grid_64x64_1080p_depth16"
# Algorithmic bytes of one traversal step: a 128-byte wide node, a 48-byte
# triangle record; each ray reads its 24-byte ray and writes an 8-byte hit.
NODE_BYTES, TRI_BYTES, RAY_IO_BYTES = 128, 48, 32


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(s[1]) for s in self.samples if len(s) > 2 and s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if len(s) > 2 and s[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            for k, n in enumerate(names):
                if len(s) > 5 + k and s[5 + k].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, value, device=None):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(world, value, device=None):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# ------------------------------------------------------------------ CPU side
def cpu_sample_paths(scene, settings, seconds: float, threads: int, kind: str, seed: int = 0):
    """Times the CPU oracle on a random pixel subset at 1 spp, grown until the
    render takes about `seconds`.  Returns (paths/s, sample description)."""
    import oracle
    o = oracle.load(kind)
    npx = settings.width * settings.height
    rng = np.random.default_rng(seed)
    n = 4096
    while True:
        px = np.sort(rng.choice(npx, size=min(n, npx), replace=False)).astype(np.uint32)
        r = o.render(scene, settings, first_sample=0, n_samples=1, threads=threads, pixels=px)
        ms = r["counters"]["render_ms"]
        if ms >= 1000.0 * seconds * 0.5 or n >= npx:
            return px.size / (ms / 1e3), {"pixels": int(px.size), "render_ms": ms,
                                          "segments": r["counters"]["rays"],
                                          "shadow_rays": r["counters"]["shadow_tests"]}
        n = int(min(npx, n * max(2.0, 1000.0 * seconds / max(ms, 1.0))))


def run_reference(args, world, rank):
    if rank != 0:
        return
    import oracle
    kind = "reference" if oracle.have_reference() else "port"
    threads = os.cpu_count() or 1
    scene = scenes.sphere_grid()
    settings = scenes.sphere_grid_settings(spp=1)
    settings.firefly_clamp = 0.0 if kind == "reference" else settings.firefly_clamp
    # size the per-step sample so the whole run stays within a few minutes
    per_step_s = max(2.0, min(20.0, 120.0 / max(1, args.steps + args.warmup)))
    vals = []
    sample = None
    for i in range(args.warmup + args.steps):
        v, sample = cpu_sample_paths(scene, settings, per_step_s, threads, kind, seed=i)
        if i >= args.warmup:
            vals.append(v)
    value = float(np.mean(vals))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * settings.width * settings.height / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded generator)",
            "config": {"workload": WORKLOAD, "width": 1920, "height": 1080, "spp_per_step": 1, "max_depth": 16,
                       "triangles": scene.triangle_count, "parallelism": "cpu threads"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": f"random {sample['pixels']} of 2,073,600 pixels at 1 spp per step "
                                       f"(TiledCpuPathTracer-equivalent scalar tracers over a shared accelerator)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ GPU side
def run_ours(args, world, rank, local):
    import torch
    from vkpathtracer_b200.tracer import CudaPathTracer, RenderTile
    torch.cuda.set_device(local)
    hbm_peak, peak_kind = peaks()
    scene = scenes.sphere_grid()
    settings = scenes.sphere_grid_settings(spp=args.warmup + args.steps)
    W, H = settings.width, settings.height
    paths_per_step = W * H
    stream = torch.cuda.Stream()
    first = rank * (args.warmup + args.steps)   # each rank renders its own samples of the frame

    # ---------------------------------------------------------- device-resident timing
    t = CudaPathTracer(device=local)
    assert t.configure(settings) and t.load_scene_snapshot(scene)
    b0 = time.time()
    assert t.build_or_update_acceleration()
    build_ms = 1e3 * (time.time() - b0)
    accel = t.accel_info()
    t.set_stream(stream.cuda_stream)
    assert t.reset_accumulation()
    with torch.cuda.stream(stream):
        for i in range(args.warmup):
            t.render_frame(first + i, 1, sync=False)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        with torch.cuda.stream(stream):
            e0.record(stream)
            for i in range(args.steps):
                t.render_frame(first + args.warmup + i, 1, sync=False)
            e1.record(stream)
        stream.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    ms = e0.elapsed_time(e1)
    t.synchronize()
    counters = t.read_counters()
    ms_max = max_over_ranks(world, ms, device=torch.device("cuda", local))
    total_paths = sum_over_ranks(world, paths_per_step * args.steps, device=torch.device("cuda", local))
    value = total_paths / (ms_max / 1e3)
    segs = counters["rays"]
    shadow = counters["shadow_tests"]
    mrays = (segs + shadow) / (ms / 1e3) / 1e6   # counters cover warm-up + timed steps: rescale
    mrays *= args.steps / (args.warmup + args.steps)
    t.close()

    # ---------------------------------------------------------- end to end (host buffers)
    e2e = None
    with CudaPathTracer(device=local) as te:
        assert te.configure(settings) and te.load_scene_snapshot(scene) and te.build_or_update_acceleration()
        te.reset_accumulation()
        hdr = np.empty((H, W, 3), np.float32)
        for i in range(args.warmup):
            te.render_tile(RenderTile(0, 0, W, H, first + i), 0)
            hdr[:] = te.resolve_hdr()
        barrier(world)
        w0 = time.perf_counter()
        for i in range(args.steps):
            assert te.render_tile(RenderTile(0, 0, W, H, first + args.warmup + i), 0)
            hdr[:] = te.resolve_hdr()
        w1 = time.perf_counter()
        e2e_ms = max_over_ranks(world, 1e3 * (w1 - w0), device=torch.device("cuda", local))
        e2e = {"value": total_paths / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": 28,
               "d2h_bytes_per_step": W * H * 3 * 4,
               "path": "vkptc_render(full-frame tile) + vkptc_resolve_hdr to host, every step"}

    # ---------------------------------------------------------- roofline of the traversal kernel
    roof = None
    if rank == 0 and not args.no_roofline:
        rsteps = min(args.steps, 4)
        with CudaPathTracer(device=local, stage_timing=True) as tt:
            tt.configure(settings)
            tt.load_scene_snapshot(scene)
            tt.build_or_update_acceleration()
            tt.set_stream(stream.cuda_stream)
            tt.reset_accumulation()
            tt.render_frame(first, 1)
            tt.read_stage_times()
            tt.reset_accumulation()
            tt.render_frame(first, rsteps)
            stages = tt.read_stage_times()
        ext_ms, ext_launches = stages["extend"]
        ext = extension_stats(scene, settings, first, rsteps, local)
        alg_bytes = NODE_BYTES * ext["nodes"] + TRI_BYTES * ext["tris"] + RAY_IO_BYTES * ext["rays"]
        achieved = alg_bytes / (ext_ms / 1e3) / 1e9
        traffic_path = os.path.join(ROOT, "profiles", "traffic_extend.json")
        traffic = None
        if os.path.exists(traffic_path):
            try:
                tr = json.load(open(traffic_path))
                traffic = tr.get("bytes_per_launch_full_scale")
            except Exception:
                traffic = None
        roof = {"kernel": "k_extend (closest-hit traversal)", "bound": "hbm", "achieved": achieved,
                "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                "peak_kind": f"{peak_kind} HBM copy bandwidth", "traffic": traffic,
                "alg_bytes_per_launch": alg_bytes / max(1, ext_launches),
                "avg_launch_ms": ext_ms / max(1, ext_launches), "launches": ext_launches,
                "nodes_per_ray": ext["nodes"] / max(1, ext["rays"]),
                "tris_per_ray": ext["tris"] / max(1, ext["rays"]),
                "stage_ms": {k: v[0] for k, v in stages.items()}}

    # ---------------------------------------------------------- ray-query workload
    rq = None
    if rank == 0 and not args.no_rayquery:
        rq = ray_query(local)

    # ---------------------------------------------------------- CPU baseline
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        import oracle
        kind = "reference" if oracle.have_reference() else "port"
        cs = scenes.sphere_grid_settings(spp=1)
        cs.firefly_clamp = 0.0 if kind == "reference" else cs.firefly_clamp
        threads = os.cpu_count() or 1
        v, sample = cpu_sample_paths(scene, cs, 10.0, threads, kind)
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": kind,
               "sample": f"random {sample['pixels']} of {W * H} pixels of this frame at 1 spp, "
                         f"{sample['render_ms']:.0f} ms render on {threads} threads"}

    if rank == 0:
        launches_per_step = 2 + 3 * settings.max_depth
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator)",
                "config": {"workload": WORKLOAD, "width": W, "height": H, "spp_per_step": 1,
                           "max_depth": settings.max_depth, "triangles": scene.triangle_count,
                           "wide_nodes": accel["wide_node_count"], "bvh_build_ms": build_ms,
                           "l2": "inputs larger than L2 (BVH+triangles %.0f MB, wave state %.0f MB)" % (
                               accel["device_bytes"] / 1e6, 140 * W * H / 1e6),
                           "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
                "mrays_per_s": mrays, "segments_per_path": segs / max(1, counters["samples"]),
                "reference_paths_per_sec_def": segs / max(1, counters["samples"]) * value,
                "gpu_launches": launches_per_step * args.steps,
                "clocks": clocks.summary(), "e2e": e2e, "roofline": roof, "ray_query": rq,
                "cpu_baseline": cpu}
        print(json.dumps(line), flush=True)


def extension_stats(scene, settings, first, steps, device):
    """Extension-ray traversal counts of the same samples (deterministic)."""
    import ctypes
    from vkpathtracer_b200.tracer import CudaPathTracer
    with CudaPathTracer(device=device, collect_stats=True) as t:
        t.configure(settings)
        t.load_scene_snapshot(scene)
        t.build_or_update_acceleration()
        t.reset_accumulation()
        t.render_frame(first, steps)
        return t.extension_counters()


def ray_query(device):
    import torch
    from vkpathtracer_b200.tracer import CudaPathTracer
    sc = scenes.displaced_sphere()
    rays = scenes.ray_query_rays(sc)
    n = rays.shape[0]
    out = {"workload": "displaced_sphere_1046904_tris_8388608_rays"}
    s = torch.cuda.Stream()
    with CudaPathTracer(device=device) as t:
        t.configure(scenes.RenderSettings(width=8, height=8, spp=1))
        t.load_scene_snapshot(sc)
        t.build_or_update_acceleration()
        d_rays = torch.from_numpy(rays).cuda()
        prim = torch.empty(n, dtype=torch.int32, device="cuda")
        dist = torch.empty(n, dtype=torch.float32, device="cuda")
        for mode, name in ((0, "closest"), (1, "any")):
            with torch.cuda.stream(s):
                for _ in range(3):
                    t.trace_rays_device(d_rays.data_ptr(), 0, n, mode, prim.data_ptr(), dist.data_ptr(), s.cuda_stream)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(s)
                for _ in range(10):
                    t.trace_rays_device(d_rays.data_ptr(), 0, n, mode, prim.data_ptr(), dist.data_ptr(), s.cuda_stream)
                e1.record(s)
            s.synchronize()
            ms = e0.elapsed_time(e1) / 10
            out[f"{name}_mrays_per_s"] = n / ms / 1e3
        # end to end through the host-buffer call
        t0 = time.perf_counter()
        t.trace_rays(rays)
        out["closest_e2e_mrays_per_s"] = n / (time.perf_counter() - t0) / 1e6
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=16)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-roofline", action="store_true")
    ap.add_argument("--no-rayquery", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world, rank, local = dist_init(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
