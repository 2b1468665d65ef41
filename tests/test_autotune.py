"""The batch autotuner's search and refinement, against a stand-in batch whose
timings are a fixed function of the launch shape (no GPU)."""
from vkpathtracer_b200 import autotune


class FakeBatch:
    """Short runs (one sample per job) rank block 128 first; full runs
    (sample_limit 0) rank block 256 with 16 stack entries first, and an 8M pool
    over the 4M one -- the situation the refinement exists for."""

    def __init__(self):
        self.calls = []

    def run(self, mode, sample_limit=0, use_graph=True, pool_paths=0, block_size=0, stack_depth=0, steps=0,
            occupancy=0, **_):
        self.calls.append((mode, sample_limit, pool_paths, block_size, stack_depth, steps, occupancy))
        if mode == "persistent":
            return {"device_ms": 2000.0}
        if block_size == 64:
            raise RuntimeError("does not fit")
        if sample_limit == 1:
            ms = 100.0 - (5.0 if block_size == 128 else 0.0) - (1.0 if stack_depth == 16 else 0.0)
            ms -= {1 << 22: 3.0, 1 << 23: 2.0}.get(pool_paths, 0.0)
            ms -= 0.5 if occupancy == 2 else 0.0
        else:
            ms = 710.0 - (8.0 if (block_size, stack_depth) == (256, 16) else 0.0)
            ms -= {1 << 23: 2.0, 1 << 22: 1.0}.get(pool_paths, 0.0)
        return {"device_ms": ms}


def test_refinement_picks_the_fastest_full_run_among_the_top_shapes(tmp_path, monkeypatch):
    monkeypatch.setenv("VKPTC_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    b = FakeBatch()
    best = autotune.tune_batch(b, "k", blocks=(64, 128, 256), stacks=(8, 16), steps=(8,), occupancy=(1, 2),
                               refine_top=3)
    # the short trials alone would keep block 128; the full runs choose 256 / 16 on the 8M pool
    assert best["mode"] == "loop"
    assert (best["block_size"], best["stack_depth"], best["pool_paths"]) == (256, 16, 1 << 23)
    assert best["refine_samples"] == 0
    assert any("error" in t for t in best["all"])          # the shape that does not fit is skipped
    # cached: the second call runs nothing
    n = len(b.calls)
    again = autotune.tune_batch(b, "k", blocks=(64, 128, 256), stacks=(8, 16), steps=(8,), occupancy=(1, 2),
                                refine_top=3)
    assert again["cached"] and len(b.calls) == n
    assert (again["block_size"], again["stack_depth"], again["pool_paths"]) == (256, 16, 1 << 23)


def test_refine_top_one_keeps_the_short_run_winner_pair(tmp_path, monkeypatch):
    monkeypatch.setenv("VKPTC_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    best = autotune.tune_batch(FakeBatch(), "k", blocks=(128, 256), stacks=(8, 16), steps=(8,), occupancy=(1, 2),
                               refine_top=1)
    assert best["block_size"] == 128 and best["stack_depth"] == 16
    # its pool and the pools next to it were re-timed; 8M wins the full run
    assert best["pool_paths"] == 1 << 23
