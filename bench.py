"""Benchmark of the render hot path on B200 (one process per GPU).

Headline workload -- batched uneven jobs: 64 independent scenes, each a seeded
displaced-sphere field with a triangle count log-uniform in [1K, 500K], a
square resolution log-uniform in [128, 1024], spp in {4,8,16,32,64}, depth in
{4,8,16}, the mixed material set (50% Lambert, 30% glossy, 20% mirror), quad
lights, firefly clamp 10.  One step = rendering every sample of every job
(~0.4 G camera paths) in ONE persistent launch fed by a device work queue and
replayed from a CUDA graph, launch parameters picked by the autotuner.
metric = camera paths per second.  The same line reports the plain mode (one
frame per launch per job) on the same jobs, which produces bit-identical films.

Also on the line: e2e (batch run through the C ABI + every film read back to
host, each step), the full-frame scene (64x64 spheres, 2.06M triangles,
1920x1080, 64 spp, depth 16), the ray-query workload (8,388,608 rays on the
1,046,904-triangle sphere), the roofline of the persistent kernel, nvidia-smi
clocks during the timed region, and the reference CPU tracer on this host.

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
WORKLOAD = "batch_64_uneven_jobs"
NODE_BYTES, TRI_BYTES, RAY_IO_BYTES = 128, 48, 32   # wide node line, triangle record, ray in + hit out
PATH_STATE_BYTES = 2 * 64                            # path state read + written per segment
# DRAM bytes (read + write) per extension ray of k_lp_extend, from one ncu
# capture of a steady-state launch of the 4-job case (102.30 MB read + 8.86 MB
# written for a launch of 2,097,152 rays).
TRAFFIC_BYTES_PER_EXT_RAY = (102304512 + 8858880) / 2097152


def l2_roofline(device, achieved_gbs):
    """The L2 side of the traversal roofline: the device's L2 read bandwidth,
    measured here by the library's own probe kernel (vkptc_measure_read_bandwidth:
    16-byte loads cached in L2 only, 64 passes over a 48 MiB buffer, well under
    the 126 MB L2), and the traversal stage's algorithmic bytes per second as a
    fraction of it.  The probe's figure is measured by this function, apart
    from the HBM peak read from MEASURED_PEAKS.json."""
    from vkpathtracer_b200.tracer import CudaPathTracer
    with CudaPathTracer(device=device) as t:
        l2 = max(t.read_bandwidth(48 << 20, 64) for _ in range(3))
    return {"l2_peak": l2, "l2_peak_kind": "measured here: L2-resident read probe (48 MiB x 64, ld.global.cg)",
            "l2_frac": achieved_gbs / l2,
            "bound_note": "the stage's DRAM traffic is a few percent of its algorithmic bytes (upper BVH levels "
                          "and small scenes stay in L2/L1); l2_frac says how close the node and triangle "
                          "stream is to the L2 bandwidth"}


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
        pw = [float(s[3]) for s in self.samples if len(s) > 3 and s[3].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            for k, n in enumerate(names):
                if len(s) > 5 + k and s[5 + k].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "power_w_max": max(pw) if pw else None, "reasons": sorted(reasons), "samples": len(self.samples)}


def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def reduce_over_ranks(world, value, op, device=None):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def aggregate_throughput(world, units_local, ms_local, device=None):
    """Whole-job throughput of N replicas: the units all ranks processed over
    the slowest rank's device time.  Returns (units/s, max ms, total units)."""
    ms_max = reduce_over_ranks(world, float(ms_local), "max", device)
    units = reduce_over_ranks(world, float(units_local), "sum", device)
    return units / (ms_max / 1e3), ms_max, units


def make_jobs(count: int, seed: int = 5):
    return scenes.batch_jobs(count=count, seed=seed)


# ------------------------------------------------------------------ CPU side
# The CPU baseline renders this fraction of every job's pixels (a seeded random
# subset, distinct pixels) at the job's full spp, in both the reference arm and
# the cpu_baseline leg of this arm.
PIXEL_FRACTION = 0.02
CPU_TRACER = ("ScalarCpuPathTracer::render_sample_pixels on a pool of {t} worker threads created once per "
              "call (one tracer per worker and job over the job's shared CpuBvhAccelerator, as "
              "TiledCpuPathTracer's tiles share theirs); a chunk of pixels renders all its samples in order")


def workload_config(jobs):
    """The `config` of both arms' lines: the workload and its sizes."""
    return {"workload": WORKLOAD, "jobs": len(jobs),
            "paths_per_step": sum(j.settings.width * j.settings.height * j.settings.spp for j in jobs),
            "triangles": sum(j.scene.triangle_count for j in jobs),
            "l2": "inputs larger than L2 (all scenes, BVHs and the path pool resident in HBM)"}


def cpu_batch(jobs, frac: float, threads: int, kind: str, seed: int = 0):
    """The CPU oracle over a seeded random `frac` of every job's pixels at the
    job's spp (vko_render_jobs).  Returns a dict with the paths, the render
    time (the timed region: the workers' render phases only, scene set-up
    excluded as ptbench excludes it), the pixel lists and the films."""
    import oracle
    o = oracle.load(kind)
    rng = np.random.default_rng(seed)
    specs = []
    for j in jobs:
        npx = j.settings.width * j.settings.height
        k = min(npx, max(1, int(round(npx * frac))))
        specs.append((j.scene, j.settings, np.sort(rng.choice(npx, size=k, replace=False)).astype(np.uint32)))
    t0 = time.perf_counter()
    outs, ms = o.render_jobs(specs, threads=threads)
    wall = time.perf_counter() - t0
    paths = sum(px.size * st.spp for _, st, px in specs)
    return {"paths": paths, "render_ms": ms, "wall_s": wall, "paths_per_s": paths / (ms / 1e3),
            "specs": specs, "outs": outs}


def tiled_check(jobs, threads: int, kind: str):
    """The reference's own TiledCpuPathTracer (worker_count = threads, 16-row
    tiles) rendering one whole job, the one whose path count is closest to
    one million: a cross-check that the pooled harness is not slower than
    the reference's tiled tracer on the same host."""
    import oracle
    o = oracle.load(kind)
    j = min(jobs, key=lambda j: abs(j.settings.width * j.settings.height * j.settings.spp - 1_000_000))
    r = o.render(j.scene, j.settings, threads=threads)
    paths = j.settings.width * j.settings.height * j.settings.spp
    # the pooled harness on every pixel of the same job
    outs, pool_ms = o.render_jobs([(j.scene, j.settings, np.arange(j.settings.width * j.settings.height,
                                                                   dtype=np.uint32))], threads=threads)
    return {"tracer": "TiledCpuPathTracer" if kind == "reference" else "port", "worker_count": threads,
            "tile_height": 16, "job": {"side": j.settings.width, "spp": j.settings.spp,
                                       "depth": j.settings.max_depth, "triangles": j.scene.triangle_count},
            "paths": paths, "render_ms": r["counters"]["render_ms"],
            "paths_per_s": paths / (r["counters"]["render_ms"] / 1e3),
            "pooled_harness_paths_per_s": paths / (pool_ms / 1e3),
            "films_equal": bool(np.array_equal(r["sum"].reshape(-1, 3).view(np.uint32),
                                               outs[0]["sum"].view(np.uint32)))}


def avx2_baseline(jobs, frac: float, threads: int, seed: int = 0):
    """The same CPU sample through the reference's AVX2 build (its 8-wide
    leaf test, -mavx2 -mfma): a second timing of the reference's CPU path, not
    a parity checker (its leaves and arithmetic differ from the default build)."""
    import oracle
    if not oracle.have_reference_avx2():
        return None
    r = cpu_batch(jobs, frac, threads, "reference_avx2", seed=seed)
    return {"value": r["paths_per_s"], "unit": UNIT, "cores": threads, "kind": "reference",
            "build": "-O2 -mavx2 -mfma -DPT_ENABLE_AVX2 (BvhTriangleIntersectorAvx2, leaf threshold 8)",
            "sample": f"random {frac:g} of every job's pixels at the job's spp ({r['paths']} paths, "
                      f"{r['render_ms']:.0f} ms; " + CPU_TRACER.format(t=threads) + ")"}


def film_parity(cpu, sums, counts):
    """GPU films (full films per job) against the CPU oracle's films of the same
    jobs on the oracle's pixel subset: bit-identical pixels, relative RMSE of
    the per-pixel means, the fraction of channels outside 3 sigma of the
    oracle's own per-sample spread, and sample-count mismatches."""
    exact = px_total = fails = chans = count_bad = 0
    dsq = rsum = 0.0
    for (sc, st, px), out, g, c in zip(cpu["specs"], cpu["outs"], sums, counts):
        gs = np.ascontiguousarray(g.reshape(-1, 3)[px], np.float32)
        gc = np.asarray(c).reshape(-1)[px].astype(np.uint32)
        rs, rc, m2 = out["sum"], out["count"], out["m2"].astype(np.float64)
        count_bad += int(np.sum(gc != rc))
        exact += int(np.sum(np.all(gs.view(np.uint32) == rs.view(np.uint32), axis=1)))
        px_total += px.size
        n = np.maximum(rc, 1).astype(np.float64)[:, None]
        gm, rm = gs / n, rs.astype(np.float64) / n
        diff = gm - rm
        dsq += float(np.sum(diff ** 2))
        rsum += float(np.sum(rm))
        chans += diff.size
        var = np.maximum(0.0, (m2 - rs.astype(np.float64) ** 2 / n) / np.maximum(n - 1.0, 1.0))
        fails += int(np.sum(np.abs(diff) > 3.0 * np.sqrt(var / n) + 1e-6 * (1.0 + np.abs(rm))))
    mean = rsum / max(1, chans)
    return {"pixels": px_total, "bit_exact_frac": exact / max(1, px_total),
            "rmse_rel": (dsq / max(1, chans)) ** 0.5 / max(mean, 1e-12),
            "sigma3_fail": fails / max(1, chans), "count_mismatch": count_bad}


def run_reference(args, world, rank):
    if rank != 0:
        return
    import oracle
    kind = "reference" if oracle.have_reference() else "port"
    threads = os.cpu_count() or 1
    jobs = make_jobs(args.jobs)
    cfg = workload_config(jobs)
    frac = args.cpu_fraction or PIXEL_FRACTION
    paths = render_ms = 0.0
    sample = None
    for i in range(args.warmup + args.steps):
        r = cpu_batch(jobs, frac, threads, kind, seed=i)
        sample = r
        if i >= args.warmup:
            paths += r["paths"]
            render_ms += r["render_ms"]
    value = paths / (render_ms / 1e3)
    tiled = tiled_check(jobs, threads, kind)
    avx2 = avx2_baseline(jobs, frac, threads, seed=args.warmup + args.steps) if kind == "reference" else None
    tracer = CPU_TRACER.format(t=threads) if kind == "reference" else f"the oracle port on {threads} threads"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": render_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded generator)", "config": cfg, "parallelism": f"cpu threads x{threads}",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": f"random {frac:g} of every job's pixels at the job's spp per step "
                                       f"({sample['paths']} paths per step; {tracer})",
                             "tracer": "ScalarCpuPathTracer" if kind == "reference" else "port",
                             "threads": threads, "pixel_fraction": frac},
            "timing": {"ms_per_step": "measured render time of each step's sampled paths (scene set-up "
                                      "excluded, as ptbench times only its render loop)",
                       "full_workload_ms_estimate": 1e3 * cfg["paths_per_step"] / value,
                       "step_wall_s_with_setup": sample["wall_s"]},
            "tiled_check": tiled, "avx2_build": avx2,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ GPU side
def full_frame(device, tunings=None):
    """The full-frame scene: 1920x1080, 64 spp, depth 16 as one batched job
    (both drivers, with the batch workload's tuning), plus one sample per
    launch through the wavefront path."""
    import torch
    from vkpathtracer_b200.tracer import BatchRenderer, CudaPathTracer
    sc = scenes.sphere_grid()
    st = scenes.sphere_grid_settings()
    out = {"workload": "sphere_grid_64x64_1080p_64spp_depth16", "triangles": sc.triangle_count}
    tunings = tunings or {"loop": {}, "persistent": {}}
    with BatchRenderer(device=device, bvh="sah") as b:
        b.add_job(sc, st)
        for m, cfg in tunings.items():
            b.run(m, **cfg)
            runs = [b.run(m, **cfg) for _ in range(2)]
            ms = min(r["device_ms"] for r in runs)
            r = runs[0]
            out[m] = {"paths_per_s": r["paths"] / (ms / 1e3),
                      "mrays_per_s": (r["segments"] + r["shadow_rays"]) / (ms / 1e3) / 1e6,
                      "ms_per_frame_64spp": ms}
        best = max(out[m]["paths_per_s"] for m in tunings)
        out["paths_per_s"] = best
    with CudaPathTracer(device=device, bvh="sah") as t:
        t.configure(st)
        t.load_scene_snapshot(sc)
        t.build_or_update_acceleration()
        s = torch.cuda.Stream()
        t.set_stream(s.cuda_stream)
        t.reset_accumulation()
        t.render_frame(0, 1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        t.render_frame(1, 8, sync=False)
        e1.record(s)
        s.synchronize()
        out["wavefront_one_sample_per_launch_paths_per_s"] = 8 * st.width * st.height / (e0.elapsed_time(e1) / 1e3)
    return out


def sdf_scene(device, cpu_fraction: float = 0.0):
    """SDF primitives next to the triangle BVH (the SDF gallery: analytic
    ellipsoid, five sphere-traced shapes, a triangle ground) at 1280x720,
    16 spp, depth 8, as one job of the loop driver; per-stage times from a
    host-driven run; SDF work from one counted sample through the wavefront
    path; optionally the CPU oracle on a random fraction of the same job's pixels."""
    from vkpathtracer_b200.tracer import BatchRenderer, CudaPathTracer
    sc = scenes.sdf_gallery()
    st = scenes.RenderSettings(width=1280, height=720, spp=16, max_depth=8, seed=1234)
    paths = st.width * st.height * st.spp
    out = {"workload": "sdf_gallery_720p_16spp_depth8", "sdf_primitives": int(sc.sdf.shape[0]),
           "triangles": sc.triangle_count}
    with BatchRenderer(device=device) as b:
        b.add_job(sc, st)
        b.run("loop")
        ms = min(b.run("loop")["device_ms"] for _ in range(2))
        out["paths_per_s"] = paths / (ms / 1e3)
        out["ms_per_frame"] = ms
    with BatchRenderer(device=device, stage_timing=True) as b:
        b.add_job(sc, st)
        stage = b.run("loop", use_graph=False)["stage_ms"]
        out["stage_share"] = {k: v / max(1e-9, sum(stage.values())) for k, v in stage.items()}
    with CudaPathTracer(device=device) as t:
        one = scenes.RenderSettings(**{**st.__dict__, "spp": 1})
        t.configure(one)
        t.load_scene_snapshot(sc)
        t.build_or_update_acceleration()
        t.reset_accumulation()
        t.render_frame(0, 1)
        c = t.read_counters()
        out["per_path"] = {"segments": c["rays"] / (st.width * st.height),
                           "sdf_tests": c["sdf_tests"] / (st.width * st.height),
                           "sdf_steps": c["sdf_steps"] / (st.width * st.height)}
        out["sdf_steps_per_s"] = out["per_path"]["sdf_steps"] * out["paths_per_s"]
    if cpu_fraction > 0.0:
        import oracle
        kind = "reference" if oracle.have_reference() else "port"
        threads = os.cpu_count() or 1
        r = cpu_batch([scenes.Job(sc, st, 0)], cpu_fraction, threads, kind)
        out["cpu_baseline"] = {"value": r["paths_per_s"], "unit": UNIT, "cores": threads, "kind": kind,
                               "sample": f"random {cpu_fraction:g} of the pixels at 16 spp ({r['paths']} paths; "
                                         + CPU_TRACER.format(t=threads) + ")"}
        out["speedup_vs_cpu"] = out["paths_per_s"] / r["paths_per_s"]
    return out


def bvh_build(device, cpu: bool = True):
    """Acceleration-structure build of the 2,064,418-triangle sphere grid:
    the device build (reference tree alone, and with the SAH traversal tree)
    and the host build (the parity mode), each through
    vkptc_build_acceleration from the scene already loaded; and the
    reference's own CPU builder (ParallelBvhBuilder) on the same triangles."""
    from vkpathtracer_b200.tracer import CudaPathTracer
    sc = scenes.sphere_grid()
    st = scenes.RenderSettings(width=64, height=64, spp=1)
    n = sc.triangle_count
    out = {"workload": "sphere_grid_64x64_2064418_triangles", "triangles": n}
    for build, bvh, reps in (("device", "reference", 6), ("device", "sah", 6), ("host", "reference", 1)):
        with CudaPathTracer(device=device, bvh=bvh, build=build) as t:
            t.configure(st)
            t.load_scene_snapshot(sc)
            ms = []
            for _ in range(reps):
                t0 = time.perf_counter()
                t.build_or_update_acceleration()
                ms.append(1e3 * (time.perf_counter() - t0))
            out[f"{build}_{bvh}_ms"] = min(ms)
    out["device_sah_triangles_per_s"] = n / (out["device_sah_ms"] / 1e3)
    # moving objects: 4096 dynamic instances of one local mesh; every instance moved per frame,
    # refit (apply_instance_transform_update) against a full rebuild of the moved scene
    dyn = scenes.dynamic_sphere_field()
    with CudaPathTracer(device=device, bvh="sah") as t:
        t.configure(st)
        t.load_scene_snapshot(dyn)
        t.build_or_update_acceleration()
        ids = [i for i in range(dyn.instances.shape[0]) if dyn.instance_local[i, 0] & 1]
        ms = []
        for k in range(6):
            ups = [{"instance": i, "translation": (float(dyn.instance_transforms[i, 0]),
                                                   float(dyn.instance_transforms[i, 1]) + 0.1 * (k + 1),
                                                   float(dyn.instance_transforms[i, 2])),
                    "rotation": tuple(float(x) for x in dyn.instance_transforms[i, 3:7]),
                    "scale": tuple(float(x) for x in dyn.instance_transforms[i, 7:10])} for i in ids]
            t0 = time.perf_counter()
            t.update_instance_transforms(ups)
            ms.append(1e3 * (time.perf_counter() - t0))
        rebuilds = []
        for _ in range(3):
            t0 = time.perf_counter()
            t.build_or_update_acceleration()
            rebuilds.append(1e3 * (time.perf_counter() - t0))
        rebuild = min(rebuilds)
    out["dynamic_refit"] = {"workload": "dynamic_sphere_field_64: 4096 instances of one 504-triangle local mesh, "
                                        "every instance moved", "triangles": dyn.triangle_count,
                            "refit_ms": float(np.median(ms)), "device_rebuild_ms": rebuild}
    out["speedup_device_vs_host_reference_tree"] = out["host_reference_ms"] / out["device_reference_ms"]
    if cpu:
        import oracle
        kind = "reference" if oracle.have_reference() else "port"
        o = oracle.load(kind)
        t0 = time.perf_counter()
        o.build_bvh(sc)
        ms = 1e3 * (time.perf_counter() - t0)
        out["cpu_baseline"] = {"value": ms, "unit": "ms", "cores": 1, "kind": kind,
                               "sample": "ParallelBvhBuilder (deterministic, leaf threshold 4) on the full scene, "
                                         "primitive bounds included"}
        out["speedup_device_vs_reference_builder"] = ms / out["device_reference_ms"]
    return out


def film_resolve(device, cpu: bool = True):
    """LDR resolve of a 1920x1080 film (ACES, gamma): the device resolve with
    the image read back to the host (what IPathTracer::resolve_ldr returns),
    against the reference's ApplyFilmResolve of the same HDR film on one
    host thread."""
    from vkpathtracer_b200.tracer import CudaPathTracer
    sc = scenes.cornell_box(seed=1)
    st = scenes.RenderSettings(width=1920, height=1080, spp=2, max_depth=6, seed=3)
    out = {"workload": "film_1920x1080_aces_gamma"}
    with CudaPathTracer(device=device) as t:
        t.configure(st)
        t.load_scene_snapshot(sc)
        t.build_or_update_acceleration()
        t.render_frame(0, st.spp)
        t.resolve_ldr(tone_map="aces")
        ms = []
        for _ in range(10):
            t0 = time.perf_counter()
            t.resolve_ldr(tone_map="aces")
            ms.append(1e3 * (time.perf_counter() - t0))
        out["device_resolve_ldr_ms"] = float(np.median(ms))
        if cpu:
            import oracle
            kind = "reference" if oracle.have_reference() else "port"
            hdr = t.resolve_hdr().reshape(st.height, st.width, 3)
            o = oracle.load(kind)
            t0 = time.perf_counter()
            o.apply_film_resolve(hdr, tone_map="aces")
            out["cpu_baseline"] = {"value": 1e3 * (time.perf_counter() - t0), "unit": "ms", "cores": 1, "kind": kind,
                                   "sample": "ApplyFilmResolve of the full film (HDR already on the host)"}
    return out


def ray_query(device):
    import torch
    from vkpathtracer_b200.tracer import CudaPathTracer
    sc = scenes.displaced_sphere()
    rays = scenes.ray_query_rays(sc)
    n = rays.shape[0]
    out = {"workload": "displaced_sphere_1046904_tris_8388608_rays"}
    s = torch.cuda.Stream()
    d_rays = torch.from_numpy(rays).cuda()
    closest = {}
    # The reference's Moller-Trumbore test (the parity mode), then the
    # watertight extension on the same tree and rays.
    for test, prefix in (("mt", ""), ("watertight", "watertight_")):
        with CudaPathTracer(device=device, bvh="sah", triangle_test=test) as t:
            t.configure(scenes.RenderSettings(width=8, height=8, spp=1))
            t.load_scene_snapshot(sc)
            t.build_or_update_acceleration()
            prim = torch.empty(n, dtype=torch.int32, device="cuda")
            dist = torch.empty(n, dtype=torch.float32, device="cuda")
            for mode, name in ((1, "any"), (0, "closest")):
                with torch.cuda.stream(s):
                    for _ in range(3):
                        t.trace_rays_device(d_rays.data_ptr(), 0, n, mode, prim.data_ptr(), dist.data_ptr(),
                                            s.cuda_stream)
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(s)
                    for _ in range(10):
                        t.trace_rays_device(d_rays.data_ptr(), 0, n, mode, prim.data_ptr(), dist.data_ptr(),
                                            s.cuda_stream)
                    e1.record(s)
                s.synchronize()
                out[f"{prefix}{name}_mrays_per_s"] = n / (e0.elapsed_time(e1) / 10) / 1e3
                if test == "mt" and name == "any":
                    occluded = prim.cpu().numpy().astype(np.uint32)
            closest[test] = prim.cpu().numpy()
            if test == "mt":
                # kept for the parity block (not printed)
                out["_ids"] = (sc, rays, closest["mt"].view(np.uint32).copy(), dist.cpu().numpy(), occluded)
            if test == "mt":
                t0 = time.perf_counter()
                t.trace_rays(rays)
                out["closest_e2e_mrays_per_s"] = n / (time.perf_counter() - t0) / 1e6
    out["watertight_ids_equal_to_mt"] = float(np.mean(closest["mt"] == closest["watertight"]))
    return out


def ray_query_parity(ids, threads: int, kind: str):
    """Closest-hit primitive ids and distances of the ray-query workload
    (8,388,608 rays, 1,046,904 triangles) against the CPU oracle's
    CpuBvhAccelerator::intersect on the same rays, and any-hit (unbounded)
    against 'the closest hit exists'."""
    import oracle
    sc, rays, prim, dist, occluded = ids
    t0 = time.perf_counter()
    rp, rt, _, ms = oracle.load(kind).intersect(sc, rays, threads=threads)
    wall = time.perf_counter() - t0
    return {"ray_query": {"rays": int(rays.shape[0]), "ids_mismatch": int(np.sum(prim != rp)),
                          "t_mismatch": int(np.sum(dist.view(np.uint32) != rt.view(np.uint32))),
                          "any_hit_mismatch": int(np.sum(occluded.astype(bool) != np.isfinite(rt))),
                          "against": f"{kind} CpuBvhAccelerator::intersect on {threads} threads "
                                     f"({wall:.1f} s with its build)"}}


def inverse_rendering(device, gd_steps: int = 200):
    """Inverse rendering: the box room with 16 boxes, 64 parameters (per-box RGB
    albedo and roughness), 128x128, 32 spp, depth 6, MSE loss.  grads/s = full
    forward+backward passes per second through the C ABI (parameters uploaded,
    loss and the gradient read back every pass).  Then 200 Adam steps from a
    seeded start towards a 1024-spp target rendered with the held-out
    parameters: fresh samples every step, the backward on samples independent
    of the forward's (decorrelated), firefly clamp 10 on every image; the loss
    of the 512-spp image is reported at the first and last parameters."""
    from vkpathtracer_b200.tracer import CudaPathTracer, material_params
    sc = scenes.inverse_box_scene()
    st = scenes.inverse_settings()
    out = {"workload": "inverse_box_16_objects_64_params_128x128_32spp_depth6", "params": 64,
           "paths_per_pass": st.width * st.height * st.spp}
    p_true = material_params(sc.materials)
    rs = np.random.RandomState(11)
    p0 = p_true.copy()
    p0[5:21, :3] = rs.uniform(0.1, 0.8, (16, 3))
    p0[5:21, 3] = rs.uniform(0.1, 0.8, 16)
    with CudaPathTracer(device=device, bvh="sah") as t:
        t.configure(st)
        t.load_scene_snapshot(sc)
        t.build_or_update_acceleration()
        t.adjoint_setup(st.spp)
        _, target = t.forward(p_true, image=True)
        t.adjoint_setup(st.spp, target)
        for _ in range(3):
            t.forward(p0)
            t.backward()
        n = 20
        fwd_ms = bwd_ms = 0.0
        t0 = time.perf_counter()
        for _ in range(n):
            t.forward(p0)
            t.backward()
            s = t.adjoint_stats()
            fwd_ms += s["forward_ms"]
            bwd_ms += s["backward_ms"]
        wall = time.perf_counter() - t0
        out["grads_per_s"] = n / wall
        out["device_grads_per_s"] = n / ((fwd_ms + bwd_ms) / 1e3)
        out["forward_ms"] = fwd_ms / n
        out["backward_ms"] = bwd_ms / n
        out["forward_paths_per_s"] = out["paths_per_pass"] / (out["forward_ms"] / 1e3)
        out["backward_paths_per_s"] = out["paths_per_pass"] / (out["backward_ms"] / 1e3)
        out["e2e"] = {"h2d_bytes_per_pass": 7 * 4 * 2 * len(p_true), "d2h_bytes_per_pass": 8 + 7 * 4 * len(p_true)}

    # gradient descent (Adam) on the 64 box parameters
    gst = scenes.inverse_settings()
    gst.firefly_clamp = 10.0
    with CudaPathTracer(device=device, bvh="sah") as t:
        t.configure(gst)
        t.load_scene_snapshot(sc)
        t.build_or_update_acceleration()
        t.adjoint_setup(1024)
        _, target = t.forward(p_true, image=True)

        def converged_loss(q):
            t.adjoint_setup(512, target, frame=7777)
            return t.forward(q)
        mask = np.zeros_like(p0, bool)
        mask[5:21, :4] = True
        conv0 = converged_loss(p0)
        t.adjoint_setup(gst.spp, target, decorrelated=True)
        p = p0.copy()
        m = np.zeros_like(p)
        v = np.zeros_like(p)
        losses = []
        t0 = time.perf_counter()
        for k in range(1, gd_steps + 1):
            t.adjoint_frames(k, 1_000_000 + k)
            losses.append(t.forward(p))
            g = t.backward()
            m = 0.9 * m + 0.1 * g
            v = 0.999 * v + 0.001 * g * g
            step = 0.01 * (m / (1 - 0.9 ** k)) / (np.sqrt(v / (1 - 0.999 ** k)) + 1e-8)
            p = np.where(mask, np.clip(p - step, 0.02, 1.0), p)
        gd_s = time.perf_counter() - t0
        conv1 = converged_loss(p)
        conv_true = converged_loss(p_true)

    def rmse(q, cols):
        mm = np.zeros_like(mask)
        mm[5:21, cols] = True
        return float(np.sqrt(np.mean((q[mm] - p_true[mm]) ** 2)))
    out["gradient_descent"] = {
        "steps": gd_steps, "optimizer": "adam lr 0.01, parameters clipped to [0.02, 1]",
        "setup": "fresh samples each step, decorrelated backward, 1024-spp target, firefly clamp 10",
        "loss_32spp_first": losses[0], "loss_32spp_last": losses[-1],
        "loss_512spp_first": conv0, "loss_512spp_last": conv1, "loss_512spp_at_true_params": conv_true,
        "albedo_rmse_first": rmse(p0, [0, 1, 2]), "albedo_rmse_last": rmse(p, [0, 1, 2]),
        "roughness_rmse_first": rmse(p0, [3]), "roughness_rmse_last": rmse(p, [3]), "seconds": gd_s}
    return out


def profile_run(args, local):
    """Small fixed run for profilers: the job set rendered by one driver
    without a CUDA graph (every stage a plain launch), with the tuning from
    the autotuner's cache when there is one.  Prints the run's stats."""
    from vkpathtracer_b200 import autotune
    from vkpathtracer_b200.tracer import BatchRenderer
    jobs = make_jobs(args.jobs)
    key = autotune.workload_key((j.scene.triangle_count, j.settings.width, j.settings.spp, j.settings.max_depth)
                                for j in jobs)
    prefix = f"batch/{autotune._gpu_name()}/loop+persistent/"
    cache = autotune._load_cache()
    cached = next((v for k, v in cache.items() if k.startswith(prefix) and k.endswith("/" + key)), {})
    cfg = cached.get("per_mode", {}).get(args.profile_run, {})
    if args.tuning:
        cfg = json.loads(args.tuning)
    tuning = {k: cfg[k] for k in ("pool_paths", "block_size", "stack_depth", "steps", "occupancy") if k in cfg}
    with BatchRenderer(device=local, bvh="sah") as b:
        for j in jobs:
            b.add_job(j.scene, j.settings)
        for _ in range(2):
            r = b.run(args.profile_run, use_graph=False, **tuning)
    print(json.dumps({"profile_run": args.profile_run, "jobs": len(jobs), "tuning": tuning,
                      "iterations": r["iterations"], "device_ms": r["device_ms"], "paths": r["paths"]}), flush=True)


def profile_build(local):
    """Small fixed run for profilers: the 2,064,418-triangle sphere grid built
    twice on the device with each traversal tree (reference, SAH)."""
    from vkpathtracer_b200.tracer import CudaPathTracer
    sc = scenes.sphere_grid()
    for bvh in ("reference", "sah"):
        with CudaPathTracer(device=local, bvh=bvh) as t:
            t.configure(scenes.RenderSettings(width=64, height=64, spp=1))
            t.load_scene_snapshot(sc)
            for _ in range(2):
                t.build_or_update_acceleration()
            print(json.dumps({"profile_build": bvh, "build_ms": t.accel_info()["build_ms"]}), flush=True)


def profile_rays(local, triangle_test):
    """Small fixed run for profilers: the 8,388,608 ray-query rays on the
    1,046,904-triangle sphere (SAH traversal tree), closest hit twice then
    any hit twice, with the given triangle test ("mt" or "watertight")."""
    import torch
    from vkpathtracer_b200.tracer import CudaPathTracer
    sc = scenes.displaced_sphere()
    rays = scenes.ray_query_rays(sc)
    n = rays.shape[0]
    with CudaPathTracer(device=local, bvh="sah", triangle_test=triangle_test) as t:
        t.configure(scenes.RenderSettings(width=8, height=8, spp=1))
        t.load_scene_snapshot(sc)
        t.build_or_update_acceleration()
        d_rays = torch.from_numpy(rays).cuda()
        prim = torch.empty(n, dtype=torch.int32, device="cuda")
        dist = torch.empty(n, dtype=torch.float32, device="cuda")
        s = torch.cuda.Stream()
        for mode in (0, 0, 1, 1):
            t.trace_rays_device(d_rays.data_ptr(), 0, n, mode, prim.data_ptr(), dist.data_ptr(), s.cuda_stream)
        s.synchronize()
    print(json.dumps({"profile_rays": triangle_test, "rays": n, "triangles": sc.triangle_count}), flush=True)


def profile_adjoint(local):
    """Small fixed run for profilers: the inverse-rendering workload (64
    parameters, 128x128, 32 spp, depth 6), forward and backward twice."""
    from vkpathtracer_b200.tracer import CudaPathTracer, material_params
    sc = scenes.inverse_box_scene()
    st = scenes.inverse_settings()
    p = material_params(sc.materials)
    with CudaPathTracer(device=local, bvh="sah") as t:
        t.configure(st)
        t.load_scene_snapshot(sc)
        t.build_or_update_acceleration()
        t.adjoint_setup(st.spp)
        _, target = t.forward(p, image=True)
        t.adjoint_setup(st.spp, target)
        for _ in range(2):
            t.forward(p * 0.9)
            t.backward()
        s = t.adjoint_stats()
    print(json.dumps({"profile_adjoint": "inverse_box_16_objects", "forward_ms": s["forward_ms"],
                      "backward_ms": s["backward_ms"]}), flush=True)


def profile_sdf(local):
    """Small fixed run for profilers: the SDF gallery (640x360, 4 spp, depth 8)
    rendered twice by the loop driver without a CUDA graph."""
    from vkpathtracer_b200.tracer import BatchRenderer
    sc = scenes.sdf_gallery()
    st = scenes.RenderSettings(width=640, height=360, spp=4, max_depth=8, seed=1234)
    with BatchRenderer(device=local) as b:
        b.add_job(sc, st)
        for _ in range(2):
            r = b.run("loop", use_graph=False)
    print(json.dumps({"profile_sdf": sc.name, "iterations": r["iterations"], "device_ms": r["device_ms"],
                      "paths": r["paths"]}), flush=True)


def run_ours(args, world, rank, local):
    import torch
    from vkpathtracer_b200 import autotune
    from vkpathtracer_b200.tracer import BatchRenderer
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    hbm_peak, peak_kind = peaks()
    # Each rank renders its own replica of the job set (disjoint seeds).
    jobs = make_jobs(args.jobs, seed=5 + 1000 * rank)
    total_paths = sum(j.settings.width * j.settings.height * j.settings.spp for j in jobs)
    b = BatchRenderer(device=local, bvh="sah")
    t0 = time.time()
    for j in jobs:
        b.add_job(j.scene, j.settings)
    setup_s = time.time() - t0
    key = autotune.workload_key((j.scene.triangle_count, j.settings.width, j.settings.spp, j.settings.max_depth)
                                for j in jobs)
    tune = autotune.tune_batch(b, key, use_cache=not args.retune)
    keys = ("pool_paths", "block_size", "stack_depth", "steps", "occupancy")
    mode = tune["mode"]
    tuning = {k: tune.get(k, 0) for k in keys}

    # ---------------------------------------------------------- plain mode (one frame per launch)
    b.run("plain")   # warm-up: the first run allocates every job's wave buffers between its launches
    plain = min((b.run("plain") for _ in range(2)), key=lambda r: r["device_ms"])
    plain_ps = plain["paths"] / (plain["device_ms"] / 1e3)

    # ---------------------------------------------------------- timed persistent runs
    for _ in range(args.warmup):
        b.run(mode, **tuning)
    barrier(world)
    torch.cuda.synchronize()
    stats = []
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            stats.append(b.run(mode, **tuning))
    torch.cuda.synchronize()
    barrier(world)
    ms_total = sum(s["device_ms"] for s in stats)
    value, ms_max, all_paths = aggregate_throughput(world, total_paths * args.steps, ms_total, dev)
    st0 = stats[-1]
    mrays = (st0["segments"] + st0["shadow_rays"]) / (st0["device_ms"] / 1e3) / 1e6

    # ---------------------------------------------------------- end to end: C ABI + films to host
    # every job's film (rgb sums and sample counts) read into pinned host buffers each step
    hostsums = [torch.empty((j.settings.height, j.settings.width, 3), dtype=torch.float32, pin_memory=True).numpy()
                for j in jobs]
    hostcounts = [torch.empty((j.settings.height, j.settings.width), dtype=torch.int32, pin_memory=True).numpy()
                  .view(np.uint32) for j in jobs]
    d2h = sum(j.settings.width * j.settings.height * 16 for j in jobs)
    barrier(world)
    w0 = time.perf_counter()
    for _ in range(args.steps):
        b.run(mode, **tuning)
        b.read_films(hostsums, hostcounts)
    e2e_ms = reduce_over_ranks(world, 1e3 * (time.perf_counter() - w0), "max", dev)
    e2e = {"value": all_paths / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": d2h,
           "path": f"vkptc_batch_run ({mode} driver, graph) + vkptc_batch_read_films (every job's rgb sums and "
                   "sample counts into pinned host buffers), every step",
           "inputs": "no per-step input copies: the scenes, their BVHs and the job table are uploaded and built "
                     f"once before timing ({setup_s:.2f} s of set-up for the {len(jobs)} jobs), as ptbench loads "
                     "and builds the scene once before its timed render loop; each step's input is the work "
                     "counter, reset on the device"}
    # both drivers, each with its own best tuning, on the same jobs
    drivers = {}
    for m, cfg in tune.get("per_mode", {}).items():
        mt = {k: cfg.get(k, 0) for k in keys}
        b.run(m, **mt)
        ms = min(b.run(m, **mt)["device_ms"] for _ in range(2))
        drivers[m] = {"paths_per_s": total_paths / (ms / 1e3), "tuning": mt}
    # the same jobs with the watertight triangle test (loop driver, the same tuning)
    wt = None
    if rank == 0 and mode == "loop" and not args.no_watertight:
        with BatchRenderer(device=local, bvh="sah", triangle_test="watertight") as bw:
            for j in jobs:
                bw.add_job(j.scene, j.settings)
            bw.run("loop", **tuning)
            wms = min(bw.run("loop", **tuning)["device_ms"] for _ in range(2))
        wt = {"paths_per_s": total_paths / (wms / 1e3), "driver": "loop", "tuning": tuning,
              "relative_to_moller_trumbore": (total_paths / (wms / 1e3)) / (value / world)}

    roof = rq = ff = cpu = inv = sdf = bb = fr = parity = cpu_avx2 = None
    if rank == 0:
        # ------------------------------------------------------ roofline of the dominant kernel
        # traversal work counted in a stats run (same rays: the traversal is deterministic)
        with BatchRenderer(device=local, collect_stats=True, bvh="sah") as bs:
            for j in jobs:
                bs.add_job(j.scene, j.settings)
            ss = bs.run(mode, **tuning)
        rays = ss["ext_rays"] + ss["shadow_queries"]
        nodes = ss["ext_nodes"] + ss["shadow_nodes"]
        tris = ss["ext_tris"] + ss["shadow_tris"]
        if mode == "loop":
            # per-stage CUDA events (host-driven iterations of the same stage kernels)
            with BatchRenderer(device=local, stage_timing=True, bvh="sah") as bt:
                for j in jobs:
                    bt.add_job(j.scene, j.settings)
                tt = bt.run("loop", use_graph=False, **tuning)
            stage = tt["stage_ms"]
            alg = NODE_BYTES * ss["ext_nodes"] + TRI_BYTES * ss["ext_tris"] + RAY_IO_BYTES * ss["ext_rays"]
            iters = max(1, tt["iterations"])
            achieved = alg / (stage["extend"] / 1e3) / 1e9
            traffic = TRAFFIC_BYTES_PER_EXT_RAY * ss["ext_rays"] / iters
            roof = {"kernel": "k_lp_extend (closest-hit traversal stage of the loop driver)", "bound": "hbm",
                    "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                    "peak_kind": f"{peak_kind} HBM copy bandwidth", "traffic": traffic,
                    "traffic_note": "per launch: DRAM bytes per extension ray from an ncu capture of a "
                                    "steady-state launch of the 4-job case x extension rays per launch",
                    "alg_bytes_per_launch": alg / iters, "avg_launch_ms": stage["extend"] / iters,
                    "launches": iters, "stage_ms": stage,
                    "stage_share": {k: v / max(1e-9, sum(stage.values())) for k, v in stage.items()},
                    "shadow_stage_achieved_gbs": (NODE_BYTES * ss["shadow_nodes"] + TRI_BYTES * ss["shadow_tris"]
                                                  + RAY_IO_BYTES * ss["shadow_queries"]) / (stage["shadow"] / 1e3) / 1e9,
                    "nodes_per_ray": nodes / max(1, rays), "tris_per_ray": tris / max(1, rays)}
            roof.update(l2_roofline(local, achieved))
        else:
            alg = NODE_BYTES * nodes + TRI_BYTES * tris + RAY_IO_BYTES * rays + PATH_STATE_BYTES * ss["segments"] \
                + 16 * ss["paths"]
            kernel_ms = st0["device_ms"]
            achieved = alg / (kernel_ms / 1e3) / 1e9
            roof = {"kernel": "k_batch (persistent wavefront: regen, closest-hit, shade, any-hit, finish)",
                    "bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                    "peak_kind": f"{peak_kind} HBM copy bandwidth", "traffic": None,
                    "alg_bytes_per_launch": alg, "avg_launch_ms": kernel_ms, "launches": 1,
                    "nodes_per_ray": nodes / max(1, rays), "tris_per_ray": tris / max(1, rays)}
        if not args.no_rayquery:
            rq = ray_query(local)
        if not args.no_fullframe:
            ff = full_frame(local, {m: d["tuning"] for m, d in drivers.items()} or None)
        inv = None if args.no_adjoint else inverse_rendering(local)
        sdf = None if args.no_sdf else sdf_scene(local, 0.0 if (args.no_cpu or world > 1) else 0.4)
        bb = None if args.no_build else bvh_build(local, cpu=not args.no_cpu and world == 1)
        fr = film_resolve(local, cpu=not args.no_cpu and world == 1)
        if world == 1 and not args.no_cpu:
            import oracle
            kind = "reference" if oracle.have_reference() else "port"
            threads = os.cpu_count() or 1
            frac = args.cpu_fraction or PIXEL_FRACTION
            r = cpu_batch(jobs, frac, threads, kind, seed=0)
            tracer = CPU_TRACER.format(t=threads) if kind == "reference" else f"the oracle port on {threads} threads"
            cpu = {"value": r["paths_per_s"], "unit": UNIT, "cores": threads, "kind": kind,
                   "sample": f"random {frac:g} of every job's pixels at the job's spp ({r['paths']} paths, "
                             f"{r['render_ms']:.0f} ms; {tracer})",
                   "tracer": "ScalarCpuPathTracer" if kind == "reference" else "port", "threads": threads,
                   "pixel_fraction": frac}
            # the timed run's films against the CPU oracle on the same pixels
            parity = {"films": film_parity(r, hostsums, hostcounts),
                      "films_against": f"{kind} CPU tracer, the cpu_baseline pixel subset of every job "
                                       "(the films of the last timed step)"}
            if rq is not None and "_ids" in rq:
                parity.update(ray_query_parity(rq.pop("_ids"), threads, kind))
            cpu_avx2 = avx2_baseline(jobs, frac, threads)
        if rq is not None:
            rq.pop("_ids", None)
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator)",
                "config": workload_config(jobs),
                "parallelism": f"replicas x{world} (one job set per rank)" if world > 1 else "single GPU",
                "run": {"setup_s": setup_s, "bvh": "sah traversal tree (hit ids exact: ties and parallel-axis "
                                                   "rule through the reference tree)",
                        "driver": mode, "tuning": tuning,
                        "autotune": {k: tune.get(k) for k in ("ms", "trials", "cached")}},

                "mrays_per_s": mrays, "drivers": drivers,
                "plain_kernel_launches": plain["kernel_launches"],
                "gpu_launches": sum(s["kernel_launches"] for s in stats),
                "clocks": clocks.summary(), "e2e": e2e, "roofline": roof, "full_frame": ff, "ray_query": rq,
                "inverse_rendering": inv, "sdf_scene": sdf, "bvh_build": bb, "film_resolve": fr,
                "watertight_batch": wt,
                "cpu_baseline_avx2": cpu_avx2, "cpu_baseline": cpu, "parity": parity,
                "plain_paths_per_s": plain_ps, "speedup_vs_plain": value / world / plain_ps}
        print(json.dumps(line), flush=True)
    b.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--jobs", type=int, default=64)
    ap.add_argument("--retune", action="store_true")
    ap.add_argument("--no-rayquery", action="store_true")
    ap.add_argument("--no-fullframe", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-sdf", action="store_true")
    ap.add_argument("--no-build", action="store_true")
    ap.add_argument("--no-watertight", action="store_true")
    ap.add_argument("--profile-run", choices=["loop", "persistent"], default=None,
                    help="profiling aid: render the job set twice with one driver, no CUDA graph, and exit")
    ap.add_argument("--tuning", default="",
                    help="profiling aid: JSON launch parameters for --profile-run (pool_paths, block_size, "
                         "stack_depth, steps, occupancy) instead of the autotuner's cache")
    ap.add_argument("--profile-build", action="store_true",
                    help="profiling aid: build the 2M-triangle sphere grid twice per traversal tree and exit")
    ap.add_argument("--profile-rays", choices=["mt", "watertight"], default=None,
                    help="profiling aid: trace the ray-query rays closest hit twice and any hit twice, and exit")
    ap.add_argument("--profile-adjoint", action="store_true",
                    help="profiling aid: run the inverse-rendering forward and backward twice, and exit")
    ap.add_argument("--profile-sdf", action="store_true",
                    help="profiling aid: render the SDF gallery twice with the loop driver, no CUDA graph, and exit")
    ap.add_argument("--cpu-fraction", type=float, default=0.0,
                    help=f"pixel fraction of every job the CPU baseline renders (0 = {PIXEL_FRACTION})")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        # One process per GPU: re-launch this command under torchrun.
        import socket
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(args.gpus),
               "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
        sys.exit(subprocess.call(cmd))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world != args.gpus:
        sys.exit(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}: launch one process per GPU")
    world, rank, local = dist_init(args)
    try:
        if args.profile_build:
            profile_build(local)
        elif args.profile_sdf:
            profile_sdf(local)
        elif args.profile_rays:
            profile_rays(local, args.profile_rays)
        elif args.profile_adjoint:
            profile_adjoint(local)
        elif args.profile_run:
            profile_run(args, local)
        elif args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
