"""Autotuner for the batched renderer and the wavefront renderer.

Sweeps the launch parameters the kernels expose -- the driver (the
cooperative persistent kernel or the device-driven stage loop), path-pool
capacity (the device queue capacity), block size, traversal-stack entries
kept in shared memory, traversal steps between warp refills and the register
variant -- on the actual workload (the whole job set for the loop driver,
one sample per job for the persistent one, whose winner is then re-timed on
the whole set), keeps the fastest, and caches the choice in a JSON file keyed
by GPU name and workload signature.  Films do not depend on these parameters
(tests/test_gpu_batch.py), only speed does.
"""
from __future__ import annotations

import hashlib
import itertools
import json
import os
import time
from typing import Dict, Iterable, Optional

DEFAULT_POOLS = (1 << 20, 1 << 21, 1 << 22, 1 << 23, 1 << 24)
DEFAULT_BLOCKS = (128, 256)
DEFAULT_STACKS = (8, 16)
DEFAULT_STEPS = (8, 16)
DEFAULT_OCCUPANCY = (1, 2, 3)
# Register variants only the loop driver has; they run its stages in 128-thread
# blocks (variant 4: traversal stages at 72 registers, 28 warps per SM).
DEFAULT_LOOP_VARIANTS = (4,)
LOOP_VARIANT_BLOCK = 128


def cache_path() -> str:
    base = os.environ.get("VKPTC_AUTOTUNE_CACHE")
    if base:
        return base
    root = os.environ.get("XDG_CACHE_HOME", os.path.join(os.path.expanduser("~"), ".cache"))
    return os.path.join(root, "vkpathtracer_b200", "autotune.json")


def _gpu_name() -> str:
    try:
        import torch
        if torch.cuda.is_available():
            return torch.cuda.get_device_name(0)
    except Exception:
        pass
    return "unknown"


def workload_key(jobs_desc: Iterable) -> str:
    h = hashlib.sha256()
    for d in jobs_desc:
        h.update(repr(d).encode())
    return h.hexdigest()[:16]


def _load_cache() -> Dict:
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except Exception:
        return {}


def _store_cache(data: Dict) -> None:
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass


DEFAULT_MODES = ("loop", "persistent")


def tune_batch(batch, key: str, modes=DEFAULT_MODES, pools=DEFAULT_POOLS, blocks=DEFAULT_BLOCKS,
               stacks=DEFAULT_STACKS, steps=DEFAULT_STEPS, occupancy=DEFAULT_OCCUPANCY, sample_limit: int = 1,
               repeats: int = 2, use_cache: bool = True, log: Optional[callable] = None,
               refine_samples: Optional[int] = 0, refine_top: int = 1, full_modes=("loop",),
               loop_variants=DEFAULT_LOOP_VARIANTS) -> Dict:
    """Returns {"mode", "pool_paths", "block_size", "stack_depth", "steps", "occupancy", "ms", "trials",
    "per_mode"}.

    Coordinate search per driver: the pool capacity first (other parameters
    at their defaults), then block size x stack entries x steps x register
    variant at that pool, then the pool sizes next to it with the chosen
    shape (the loop driver also tries its own register variants, loop_variants,
    with 128-thread blocks and every stack / steps pair).  Trials replay a CUDA graph (the way the runs are timed), so the
    loop driver is measured as it runs.  Drivers in full_modes are searched on
    the whole workload (refine_samples per job; 0 = every sample): short runs
    under-fill large pools and rank close shapes only roughly (differences of
    ~1 % flip between short and full runs).  The others are searched on short
    runs (sample_limit per job), and the fastest trials of their refine_top
    fastest (block size, stack entries) pairs, each with its pool and the pool
    sizes next to it, are timed again on the whole workload (refine_samples
    None: no refinement, the short-run times decide).  The fastest driver on
    the whole workload wins."""
    cache = _load_cache() if use_cache else {}
    ckey = (f"batch/{_gpu_name()}/{'+'.join(modes)}/r{refine_samples}t{refine_top}"
            f"f{'+'.join(m for m in modes if m in full_modes)}v{'+'.join(map(str, loop_variants))}/{key}")
    if use_cache and ckey in cache:
        return dict(cache[ckey], cached=True)
    trials = []
    t0 = time.time()

    def measure(cfg, samples):
        mode = cfg["mode"]
        args = {k: v for k, v in cfg.items() if k not in ("mode", "ms", "samples")}
        batch.run(mode, sample_limit=samples, use_graph=True, **args)   # capture
        return min(batch.run(mode, sample_limit=samples, use_graph=True, **args)["device_ms"] for _ in range(repeats))

    def trial(cfg, samples):
        try:
            ms = measure(cfg, samples)
        except Exception as e:   # a shape that does not fit (e.g. shared memory) is skipped
            trials.append(dict(cfg, error=str(e), samples=samples))
            return None
        trials.append(dict(cfg, ms=ms, samples=samples))
        if log:
            log(trials[-1])
        return ms

    def neighbours(cfg):
        i = list(pools).index(cfg["pool_paths"]) if cfg["pool_paths"] in pools else -1
        return [dict(cfg, pool_paths=pools[j]) for j in (i - 1, i + 1) if i >= 0 and 0 <= j < len(pools)]

    full = refine_samples if refine_samples is not None else sample_limit
    per_mode = {}
    for mode in modes:
        samples = full if mode in full_modes else sample_limit
        mine = []   # (ms, cfg) of this driver's search

        def run(cfg):
            ms = trial(cfg, samples)
            if ms is not None:
                mine.append((ms, cfg))
            return ms

        for pool in pools:
            run({"mode": mode, "pool_paths": pool, "block_size": 0, "stack_depth": 0, "steps": 0, "occupancy": 0})
        if not mine:
            continue
        pool = min(mine, key=lambda r: r[0])[1]["pool_paths"]
        shapes = list(itertools.product(blocks, stacks, steps, occupancy))
        if mode == "loop":
            shapes += [(LOOP_VARIANT_BLOCK, stack, st, occ)
                       for stack, st, occ in itertools.product(stacks, steps, loop_variants)]
        for block, stack, st, occ in shapes:
            run({"mode": mode, "pool_paths": pool, "block_size": block, "stack_depth": stack, "steps": st,
                 "occupancy": occ})
        tried = [c for _, c in mine]
        for c in neighbours(min(mine, key=lambda r: r[0])[1]):
            if c not in tried:
                run(c)
        if samples == full:
            ms, cfg = min(mine, key=lambda r: r[0])
            per_mode[mode] = dict(cfg, ms=ms, samples=samples)
            continue
        if refine_samples is None:
            ms, cfg = min(mine, key=lambda r: r[0])
            per_mode[mode] = dict(cfg, ms=ms, samples=samples)
            continue
        shapes, cands = [], []
        for _, cfg in sorted(mine, key=lambda r: r[0]):
            shape = (cfg["block_size"], cfg["stack_depth"])
            if shape in shapes:
                continue
            shapes.append(shape)
            for c in [cfg] + neighbours(cfg):
                if c not in cands:
                    cands.append(c)
            if len(shapes) >= refine_top:
                break
        refined = []
        for c in cands:
            ms = trial(c, full)
            if ms is not None:
                refined.append((ms, c))
        if refined:
            ms, cfg = min(refined, key=lambda r: r[0])
            per_mode[mode] = dict(cfg, ms=ms, samples=full)
    if not per_mode:
        raise RuntimeError("autotune: no launch configuration ran")
    best = dict(min(per_mode.values(), key=lambda r: r["ms"]))
    best["refine_samples"] = best.pop("samples")
    best["per_mode"] = per_mode
    best["trials"] = len(trials)
    best["tune_seconds"] = time.time() - t0
    if use_cache:
        cache[ckey] = best
        _store_cache(cache)
    return dict(best, cached=False, all=trials)


def tune_wavefront(make_tracer, render_samples: int = 1, blocks=DEFAULT_BLOCKS, stacks=DEFAULT_STACKS,
                   steps=DEFAULT_STEPS, log: Optional[callable] = None) -> Dict:
    """Sweeps block size, stack entries and steps of the wavefront renderer.
    make_tracer(block_size, stack_depth, steps) must return a ready CudaPathTracer."""
    import torch
    best = None
    for block, stack, st in itertools.product(blocks, stacks, steps):
        t = make_tracer(block, stack, st)
        s = torch.cuda.Stream()
        t.set_stream(s.cuda_stream)
        t.reset_accumulation()
        t.render_frame(0, 1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        t.render_frame(1, render_samples, sync=False)
        e1.record(s)
        s.synchronize()
        ms = e0.elapsed_time(e1) / render_samples
        t.close()
        rec = {"block_size": block, "stack_depth": stack, "steps": st, "ms": ms}
        if log:
            log(rec)
        if best is None or ms < best["ms"]:
            best = rec
    return best
