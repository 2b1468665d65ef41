"""The batch autotuner's search and refinement, against a stand-in batch whose
timings are a fixed function of the launch shape (no GPU)."""
from vkpathtracer_b200 import autotune


class FakeBatch:
    """Short runs (one sample per job) rank block 128 first; full runs
    (sample_limit 0) rank block 256 with 16 stack entries first, and an 8M pool
    over the 4M one -- the situation a search on short runs gets wrong.  The
    persistent driver is the same shape function, 1000 ms slower."""

    def __init__(self):
        self.calls = []

    def run(self, mode, sample_limit=0, use_graph=True, pool_paths=0, block_size=0, stack_depth=0, steps=0,
            occupancy=0, **_):
        self.calls.append((mode, sample_limit, pool_paths, block_size, stack_depth, steps, occupancy))
        if block_size == 64:
            raise RuntimeError("does not fit")
        if sample_limit == 1:
            ms = 100.0 - (5.0 if block_size == 128 else 0.0) - (1.0 if stack_depth == 16 else 0.0)
            ms -= {1 << 22: 3.0, 1 << 23: 2.0}.get(pool_paths, 0.0)
            ms -= 0.5 if occupancy == 2 else 0.0
        else:
            ms = 710.0 - (8.0 if (block_size, stack_depth) == (256, 16) else 0.0)
            ms -= {1 << 23: 2.0, 1 << 22: 1.0}.get(pool_paths, 0.0)
        return {"device_ms": ms + (1000.0 if mode == "persistent" else 0.0)}


SHAPES = dict(blocks=(64, 128, 256), stacks=(8, 16), steps=(8,), occupancy=(1, 2))


def test_loop_driver_is_searched_on_the_whole_workload(tmp_path, monkeypatch):
    monkeypatch.setenv("VKPTC_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    b = FakeBatch()
    best = autotune.tune_batch(b, "k", **SHAPES)
    assert best["mode"] == "loop"
    assert (best["block_size"], best["stack_depth"], best["pool_paths"]) == (256, 16, 1 << 23)
    assert best["refine_samples"] == 0 and best["ms"] == 700.0
    assert all(c[1] == 0 for c in b.calls if c[0] == "loop")          # every loop trial on the whole set
    assert any("error" in t for t in best["all"])                       # the shape that does not fit is skipped
    # both drivers are reported with their whole-workload times
    assert set(best["per_mode"]) == {"loop", "persistent"}
    assert best["per_mode"]["persistent"]["samples"] == 0
    # cached: the second call runs nothing
    n = len(b.calls)
    again = autotune.tune_batch(b, "k", **SHAPES)
    assert again["cached"] and len(b.calls) == n
    assert (again["block_size"], again["stack_depth"], again["pool_paths"]) == (256, 16, 1 << 23)


def test_short_run_search_is_refined_on_the_whole_workload(tmp_path, monkeypatch):
    monkeypatch.setenv("VKPTC_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    b = FakeBatch()
    best = autotune.tune_batch(b, "k", modes=("persistent",), refine_top=1, **SHAPES)
    # short runs chose block 128 / 16 entries; its pool and the pools next to it
    # were re-timed on the whole set, where the 8M pool wins
    assert (best["block_size"], best["stack_depth"], best["pool_paths"]) == (128, 16, 1 << 23)
    assert best["refine_samples"] == 0 and best["ms"] == 1708.0
    full = [c for c in b.calls if c[1] == 0]
    assert full and all(c[3] == 128 and c[4] == 16 for c in full)


def test_refinement_can_be_switched_off(tmp_path, monkeypatch):
    monkeypatch.setenv("VKPTC_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    b = FakeBatch()
    best = autotune.tune_batch(b, "k", modes=("persistent",), refine_samples=None, **SHAPES)
    assert all(c[1] == 1 for c in b.calls)
    assert best["block_size"] == 128 and best["refine_samples"] == 1


def test_loop_register_variants_run_at_128_threads(tmp_path, monkeypatch):
    monkeypatch.setenv("VKPTC_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    b = FakeBatch()
    autotune.tune_batch(b, "k", **SHAPES)
    v4 = [c for c in b.calls if c[6] == 4]
    assert v4 and all(c[0] == "loop" and c[3] == 128 for c in v4)
    assert {(c[4], c[5]) for c in v4} == {(8, 8), (16, 8)}     # every stack / steps pair
