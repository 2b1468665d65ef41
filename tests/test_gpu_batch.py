"""Batched rendering: many uneven jobs in one persistent launch.

* The persistent launch (device work queue, path regeneration, CUDA graph)
  produces films bit-identical to rendering each job one frame per launch.
* Every job matches the CPU oracle at the same seed and spp, checked on a
  seeded pixel subset of each job (the oracle renders just those pixels --
  exact, because the RNG is keyed per pixel and sample).
"""
import numpy as np
import pytest

import oracle
from tests.golden import cases
from vkpathtracer_b200 import scenes
from vkpathtracer_b200.tracer import BatchRenderer

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def small_jobs():
    jobs = []
    jobs.append((scenes.cornell_box(seed=1), scenes.cornell_settings(48, 40, 3)))
    jobs.append((scenes.sphere_field(3, 9, 10, seed=21, n_lights=3, light_size=1.5, light_height=5.0),
                 scenes.RenderSettings(width=40, height=30, spp=2, max_depth=6, seed=77, firefly_clamp=10.0)))
    jobs.append((scenes.sphere_field(5, 12, 14, seed=8, n_lights=4, light_size=2.0, light_height=6.0),
                 scenes.RenderSettings(width=64, height=64, spp=4, max_depth=16, seed=5, firefly_clamp=10.0)))
    jobs.append((scenes.cornell_box(seed=4), scenes.RenderSettings(width=33, height=17, spp=5, max_depth=4, seed=9)))
    # thin lens with a polygonal iris and anamorphic squeeze
    jobs.append((cases.lens_scene("pentagon_sharp"), scenes.RenderSettings(width=40, height=32, spp=3, max_depth=5,
                                                                          seed=13)))
    return jobs


@pytest.fixture(scope="module")
def batch():
    b = BatchRenderer()
    for sc, st in small_jobs():
        b.add_job(sc, st)
    yield b
    b.close()


def films(b, n):
    return [b.film(j) for j in range(n)]


def test_persistent_equals_plain_bitwise(batch):
    n = len(small_jobs())
    s_plain = batch.run("plain")
    plain = films(batch, n)
    s_pers = batch.run("persistent", use_graph=False)
    pers = films(batch, n)
    s_graph = batch.run("persistent", use_graph=True)
    graph = films(batch, n)
    assert s_graph["graph_used"] == 1
    for (a, ca), (b, cb), (c, cc) in zip(plain, pers, graph):
        assert np.array_equal(ca, cb) and np.array_equal(ca, cc)
        assert np.array_equal(bits(a), bits(b))
        assert np.array_equal(bits(a), bits(c))
    assert s_plain["paths"] == s_pers["paths"] == sum(st.width * st.height * st.spp for _, st in small_jobs())
    assert s_plain["segments"] == s_pers["segments"]
    assert s_plain["shadow_rays"] == s_pers["shadow_rays"]
    assert s_pers["kernel_launches"] < s_plain["kernel_launches"]


@pytest.mark.parametrize("use_graph", [True, False])
def test_loop_mode_equals_plain_bitwise(batch, use_graph):
    """One kernel per stage in a CUDA graph while-node (or host-driven)."""
    n = len(small_jobs())
    s_plain = batch.run("plain")
    plain = films(batch, n)
    s_loop = batch.run("loop", use_graph=use_graph)
    assert s_loop["graph_used"] == int(use_graph)
    assert s_loop["iterations"] > 0
    # per iteration: regen, extend, shadow, drain, shade, decide (the jobs have no SDF primitives)
    assert s_loop["kernel_launches"] == 1 + 6 * s_loop["iterations"] + n
    for (a, ca), (b, cb) in zip(plain, films(batch, n)):
        assert np.array_equal(ca, cb) and np.array_equal(bits(a), bits(b))
    assert s_loop["segments"] == s_plain["segments"]
    assert s_loop["shadow_rays"] == s_plain["shadow_rays"]
    # the persistent driver runs the same pool iterations; the loop driver traces an
    # iteration's NEE queries in the next one, so it adds one for the last bounce's
    s_pers = batch.run("persistent", use_graph=use_graph)
    assert s_loop["iterations"] == s_pers["iterations"] + 1


@pytest.mark.parametrize("mode", ["persistent", "loop"])
@pytest.mark.parametrize("pool,block,stack,steps", [(1024, 64, 4, 1), (4096, 256, 8, 16), (1 << 18, 128, 32, 4)])
def test_tuning_does_not_change_films(batch, mode, pool, block, stack, steps):
    n = len(small_jobs())
    batch.run("plain")
    ref = films(batch, n)
    batch.run(mode, pool_paths=pool, block_size=block, stack_depth=stack, steps=steps)
    got = films(batch, n)
    for (a, ca), (b, cb) in zip(ref, got):
        assert np.array_equal(ca, cb) and np.array_equal(bits(a), bits(b))


@pytest.mark.parametrize("mode,occupancy", [("loop", o) for o in range(5)] + [("persistent", o) for o in (0, 3, 4)])
def test_register_variants_do_not_change_films(batch, mode, occupancy):
    # Variant 4 runs the loop driver's stages in 128-thread blocks whatever the
    # block size asked for; the persistent driver takes it as variant 3.
    n = len(small_jobs())
    batch.run("plain")
    ref = films(batch, n)
    batch.run(mode, block_size=256, stack_depth=16, steps=8, occupancy=occupancy)
    got = films(batch, n)
    for (a, ca), (b, cb) in zip(ref, got):
        assert np.array_equal(ca, cb) and np.array_equal(bits(a), bits(b))


def test_sample_limit(batch):
    n = len(small_jobs())
    s = batch.run("persistent", sample_limit=1)
    assert s["paths"] == sum(st.width * st.height for _, st in small_jobs())
    for j in range(n):
        _, c = batch.film(j)
        assert np.all(c == 1)


def test_each_job_matches_oracle_on_pixel_subset(batch):
    """Unclamped jobs against the reference itself where it is built; jobs with
    the firefly clamp (an extension the reference lacks) against the port."""
    batch.run("persistent")
    ref_oracle, port = oracle.load("auto"), oracle.load("port")
    rng = np.random.default_rng(0)
    for j, (sc, st) in enumerate(small_jobs()):
        g, gc = batch.film(j)
        npx = st.width * st.height
        px = np.sort(rng.choice(npx, size=max(32, npx // 10), replace=False)).astype(np.uint32)
        o = port if st.firefly_clamp > 0.0 else ref_oracle
        r = o.render(sc, st, pixels=px, threads=8)
        ref = r["sum"].reshape(-1, 3)[px]
        got = g.reshape(-1, 3)[px]
        assert np.array_equal(gc.reshape(-1)[px], r["count"].reshape(-1)[px])
        exact = np.mean(np.all(bits(got) == bits(ref), axis=1))
        rel = np.sqrt(np.mean((got - ref) ** 2)) / (np.mean(ref) + 1e-9)
        assert exact >= 0.95 and rel < 1e-3, (j, o.kind, exact, rel)


def test_sah_batch_equals_reference_tree_batch(batch):
    n = len(small_jobs())
    batch.run("persistent")
    ref = films(batch, n)
    with BatchRenderer(bvh="sah") as b2:
        for sc, st in small_jobs():
            b2.add_job(sc, st)
        b2.run("persistent")
        for j in range(n):
            f, c = b2.film(j)
            assert np.array_equal(c, ref[j][1]) and np.array_equal(bits(f), bits(ref[j][0]))


def test_sdf_jobs_equal_across_drivers_and_match_oracle():
    """Jobs with SDF primitives (one without triangles) in the batched
    drivers: loop and persistent films equal the plain ones bit for bit, and
    each job matches the oracle on a pixel subset."""
    jobs = [(scenes.sdf_gallery(), scenes.RenderSettings(width=48, height=40, spp=3, max_depth=6, seed=2)),
            (scenes.cornell_box(seed=2), scenes.cornell_settings(32, 24, 2)),
            (scenes.sdf_complexity(), scenes.RenderSettings(width=40, height=30, spp=2, max_depth=5, seed=6))]
    with BatchRenderer() as b:
        for sc, st in jobs:
            b.add_job(sc, st)
        b.run("plain")
        plain = films(b, len(jobs))
        for mode in ("loop", "persistent"):
            b.run(mode)
            for (f, c), (pf, pc) in zip(films(b, len(jobs)), plain):
                assert np.array_equal(c, pc) and np.array_equal(bits(f), bits(pf)), mode
    o = oracle.load("auto")
    rng = np.random.default_rng(1)
    for (sc, st), (g, gc) in zip(jobs, plain):
        npx = st.width * st.height
        px = np.sort(rng.choice(npx, size=npx // 4, replace=False)).astype(np.uint32)
        r = o.render(sc, st, pixels=px, threads=8)
        ref, got = r["sum"].reshape(-1, 3)[px], g.reshape(-1, 3)[px]
        assert np.array_equal(gc.reshape(-1)[px], r["count"].reshape(-1)[px])
        exact = np.mean(np.all(bits(got) == bits(ref), axis=1))
        rel = np.sqrt(np.mean((got - ref) ** 2)) / (np.mean(ref) + 1e-9)
        assert exact >= 0.95 and rel < 1e-3, (sc.name, exact, rel)


def test_read_films_equals_per_job_reads(batch):
    """vkptc_batch_read_films (all jobs, one wait) returns what the per-job
    reads return."""
    n = len(small_jobs())
    batch.run("loop")
    ref = films(batch, n)
    sums = [np.zeros_like(f) for f, _ in ref]
    counts = [np.zeros_like(c) for _, c in ref]
    batch.read_films(sums, counts)
    for (f, c), s, k in zip(ref, sums, counts):
        assert np.array_equal(bits(f), bits(s)) and np.array_equal(c, k)
