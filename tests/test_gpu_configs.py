"""Parity at the benchmark configurations' own sizes, not only on small fixtures.

* Closed box (36 triangles, 256x256, 16 spp, depth 8, NEE+MIS, seed 1234): the
  GPU film of the whole frame against the reference CPU tracer's.
* Ray query (1,046,904-triangle displaced sphere scaled x16, 8,388,608 rays:
  2048^2 primary + 4,194,304 random): closest-hit primitive ids and distances
  bit-exact against CpuBvhAccelerator::intersect
  (src/pathtracer/CpuBvhAccelerator.cpp:360-477) with both traversal trees,
  and any-hit equal to "closest t < tmax".
* Full frame (64x64 displaced spheres, 2,064,386 triangles, 1920x1080, 64 spp,
  depth 16): the loop driver's whole-frame film on a seeded subset of 2,000
  pixels against the CPU oracle on those pixels (exact, since the RNG is
  keyed per pixel and sample) -- without the firefly clamp against the
  reference, with the clamp (an extension) against the port.
* Counters (SampleCounters, src/pathtracer/PathTracer.h:218-230): on the
  pixels whose films are bit-identical, the GPU's samples, rays (segments, the
  numerator of ptbench's paths_per_sec) and shadow_tests equal the
  reference's exactly.
"""
import os

import numpy as np
import pytest

import oracle
from tests.golden import cases
from vkpathtracer_b200 import native, scenes
from vkpathtracer_b200.tracer import BatchRenderer, CudaPathTracer, RenderTile

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 8
RMSE_REL_TOL = 1e-3
SIGMA3_FAIL_FRAC = 0.003
BIT_EXACT_FRAC = 0.97


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def subset_report(g_sum, g_cnt, ref):
    """GPU film values on a pixel subset against render_jobs output for it."""
    rs, rc, m2 = ref["sum"], ref["count"], ref["m2"].astype(np.float64)
    n = np.maximum(rc, 1).astype(np.float64)[:, None]
    diff = g_sum / n - rs.astype(np.float64) / n
    mean = float(np.mean(rs / n)) + 1e-12
    var = np.maximum(0.0, (m2 - rs.astype(np.float64) ** 2 / n) / np.maximum(n - 1.0, 1.0))
    fail = np.abs(diff) > 3.0 * np.sqrt(var / n) + 1e-6 * (1.0 + np.abs(rs / n))
    return {"rmse_rel": float(np.sqrt(np.mean(diff ** 2))) / mean, "sigma3_fail": float(np.mean(fail)),
            "bit_exact": float(np.mean(np.all(bits(g_sum) == bits(rs), axis=1))),
            "count_equal": bool(np.array_equal(g_cnt, rc))}


def test_box_config_full_frame_matches_reference():
    sc = scenes.cornell_box(seed=1)
    st = scenes.cornell_settings(256, 256, 16)
    ref = oracle.load("auto").render(sc, st, threads=THREADS, per_sample=True)
    with CudaPathTracer() as t:
        assert t.configure(st) and t.load_scene_snapshot(sc) and t.build_or_update_acceleration()
        assert t.reset_accumulation()
        for s in range(st.spp):
            assert t.render_tile(RenderTile(0, 0, st.width, st.height, s), 0), t.status().last_error
        g, cnt, _ = t.film()
        c = t.read_counters()
    assert np.array_equal(cnt, ref["count"])
    r = ref["sum"] / st.spp
    diff = g / st.spp - r
    sd = np.std(ref["samples"], axis=0, ddof=1) / np.sqrt(st.spp)
    sigma3 = float(np.mean(np.abs(diff) > 3.0 * sd + 1e-6 * (1.0 + np.abs(r))))
    rmse_rel = float(np.sqrt(np.mean(diff ** 2)) / (np.mean(r) + 1e-12))
    exact = float(np.mean(np.all(bits(g) == bits(ref["sum"]), axis=-1)))
    print({"rmse_rel": rmse_rel, "sigma3_fail": sigma3, "bit_exact": exact})
    assert rmse_rel < RMSE_REL_TOL and sigma3 < SIGMA3_FAIL_FRAC and exact >= BIT_EXACT_FRAC
    assert c["samples"] == ref["counters"]["samples"] == 256 * 256 * 16


@pytest.fixture(scope="module")
def ray_query_case():
    sc = scenes.displaced_sphere()
    rays = scenes.ray_query_rays(sc)
    assert sc.triangle_count == 1_046_904 and rays.shape[0] == 8_388_608
    pr, tr, _, _ = oracle.load("auto").intersect(sc, rays, threads=THREADS)
    return sc, rays, pr, tr


@pytest.mark.parametrize("bvh", ["reference", "sah"])
def test_ray_query_config_full_size_ids_bit_exact(ray_query_case, bvh):
    sc, rays, pr, tr = ray_query_case
    with CudaPathTracer(bvh=bvh) as t:
        assert t.configure(scenes.RenderSettings(width=8, height=8, spp=1))
        assert t.load_scene_snapshot(sc) and t.build_or_update_acceleration()
        p, tt = t.trace_rays(rays)
        assert np.array_equal(p, pr), f"{int(np.sum(p != pr))} of {len(p)} ids differ"
        assert np.array_equal(bits(tt), bits(tr))
        occ_inf, _ = t.trace_rays(rays, mode=native.QUERY_ANY)
        rng = np.random.default_rng(12)
        tmax = np.where(np.isfinite(tr), tr * rng.uniform(0.5, 1.5, tr.shape), rng.uniform(1.0, 80.0, tr.shape))
        tmax = tmax.astype(np.float32)
        occ, _ = t.trace_rays(rays, mode=native.QUERY_ANY, tmax=tmax)
    assert np.array_equal(occ_inf.astype(bool), np.isfinite(tr))
    assert np.array_equal(occ.astype(bool), np.isfinite(tr) & (tr < tmax))


@pytest.fixture(scope="module")
def full_frame_case():
    sc = scenes.sphere_grid()
    rng = np.random.default_rng(2024)
    st = scenes.sphere_grid_settings()
    px = np.sort(rng.choice(st.width * st.height, size=2000, replace=False)).astype(np.uint32)
    return sc, px


@pytest.mark.parametrize("clamp", [0.0, 10.0])
def test_full_frame_config_pixel_subset_matches_oracle(full_frame_case, clamp):
    sc, px = full_frame_case
    st = scenes.sphere_grid_settings()
    st.firefly_clamp = clamp
    kind = "auto" if clamp == 0.0 else "port"       # the reference has no firefly clamp
    outs, _ = oracle.load(kind).render_jobs([(sc, st, px)], threads=THREADS)
    with BatchRenderer(device=0, bvh="sah") as b:
        b.add_job(sc, st)
        b.run("loop")
        f, c = b.film(0)
    rep = subset_report(f.reshape(-1, 3)[px], c.reshape(-1)[px], outs[0])
    print(clamp, rep)
    assert rep["count_equal"]
    assert rep["rmse_rel"] < RMSE_REL_TOL and rep["sigma3_fail"] < SIGMA3_FAIL_FRAC
    assert rep["bit_exact"] >= BIT_EXACT_FRAC


@pytest.mark.parametrize("name", ["box", "field", "sdf"])
def test_counters_equal_reference_on_bit_identical_pixels(name):
    d = cases.load_fixture(name)
    sc, st = cases.scene_from_arrays(d), cases.settings_from_arrays(d)
    W, H = st.width, st.height
    o = oracle.load("auto")
    with CudaPathTracer() as t:
        assert t.configure(st) and t.load_scene_snapshot(sc) and t.build_or_update_acceleration()
        assert t.reset_accumulation()
        t.render_frame(0, st.spp)
        g, _, _ = t.film()
    same = np.all(bits(g) == bits(d["film_sum"]), axis=-1).reshape(-1)
    px = np.nonzero(same)[0].astype(np.uint32)
    assert px.size >= 0.9 * W * H
    ref = o.render(sc, st, threads=THREADS, pixels=px)["counters"]
    with CudaPathTracer() as t:
        assert t.configure(st) and t.load_scene_snapshot(sc) and t.build_or_update_acceleration()
        assert t.reset_accumulation()
        # every sample of the selected pixels as 1x1 tiles, sample by sample
        tiles = [RenderTile(int(p % W), int(p // W), 1, 1, s) for s in range(st.spp) for p in px]
        assert t.render_tiles(tiles, 0), t.status().last_error
        c = t.read_counters()
    print(name, px.size, {k: (c[k], ref[k]) for k in ("samples", "rays", "shadow_tests")})
    assert c["samples"] == ref["samples"] == px.size * st.spp
    assert c["rays"] == ref["rays"]
    assert c["shadow_tests"] == ref["shadow_tests"]
