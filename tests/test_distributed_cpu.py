"""The N>1 path of bench.py, on CPU with the gloo backend, world size 2.

bench.py --gpus N runs one process per GPU (replicas, no data-path
collective); ranks meet only in a barrier and two reductions (max of the
device time, sum of the paths), and rank 0 alone prints the line.  These
tests run those pieces as two gloo ranks, and the reference arm end to end
under torchrun (rank 0 renders with the reference CPU code, rank 1 exits 0).
"""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, ROOT)
    import argparse
    import bench
    import torch.distributed as dist
    w, r, local = bench.dist_init(argparse.Namespace(impl="reference"))
    assert (w, r, local) == (world, rank, rank)
    bench.barrier(w)
    # rank k processed (k+1) * 1000 paths in (k+1) * 10 ms
    value, ms_max, units = bench.aggregate_throughput(w, (rank + 1) * 1000, (rank + 1) * 10.0)
    mx = bench.reduce_over_ranks(w, float(rank), "max")
    sm = bench.reduce_over_ranks(w, float(rank + 1), "sum")
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"value": value, "ms_max": ms_max, "units": units, "max": mx, "sum": sm}, f)
    dist.destroy_process_group()


def test_rank_reductions_gloo_world2(tmp_path):
    world = 2
    mp.spawn(_rank_main, args=(world, free_port(), str(tmp_path)), nprocs=world, join=True)
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    for r in res:
        assert r["ms_max"] == 20.0
        assert r["units"] == 3000.0
        assert r["value"] == pytest.approx(3000.0 / 0.020)
        assert r["max"] == 1.0 and r["sum"] == 3.0


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_over_ranks(1, 5.0, "max") == 5.0
    assert bench.aggregate_throughput(1, 500, 250.0)[0] == pytest.approx(2000.0)


def test_reference_arm_under_torchrun_rank0_only():
    import oracle
    oracle.build_port()
    env = dict(os.environ, PYTHONPATH=ROOT)
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3", "--jobs", "2",
           "--cpu-fraction", "0.002"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["value"] > 0 and line["unit"] == "paths/s"
    assert line["cpu_baseline"]["kind"] in ("reference", "port")
    assert line["e2e"]["h2d_bytes_per_step"] == 0


def test_gpus_flag_launches_one_process_per_rank_without_torchrun():
    """bench.py --gpus 2 started as a plain process re-launches itself under
    torchrun with two ranks; the reference arm's line then reports n_gpus 2."""
    import oracle
    oracle.build_port()
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    env["PYTHONPATH"] = ROOT
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
           "--warmup", "3", "--jobs", "2", "--cpu-fraction", "0.002"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    assert lines[0]["n_gpus"] == 2 and lines[0]["impl"] == "reference"


def test_gpus_flag_must_match_world_size():
    env = dict(os.environ, PYTHONPATH=ROOT, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode != 0 and "WORLD_SIZE" in r.stderr
