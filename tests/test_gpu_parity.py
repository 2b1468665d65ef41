"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

* Closest-hit primitive ids and distances: bit-exact.
* Any-hit: exactly the oracle's (closest t < tmax).
* Films: per-pixel agreement with the oracle at the same seed and spp --
  bit-identical for the pixels whose paths take no transcendental whose
  last bit differs from glibc's, and within a stated RMSE and a 3-sigma
  per-pixel mean test over the oracle's own per-sample spread.
"""
import numpy as np
import pytest

import oracle
from tests.golden import cases
from vkpathtracer_b200 import native, scenes
from vkpathtracer_b200.tracer import CudaPathTracer, RenderTile

pytestmark = pytest.mark.gpu

# Film tolerances (float32 radiance, same seed and spp as the oracle).
RMSE_REL_TOL = 1e-3        # RMSE(gpu - oracle) / mean(oracle)
SIGMA3_FAIL_FRAC = 0.003   # fraction of pixel channels allowed outside 3 sigma
BIT_EXACT_FRAC = 0.97      # fraction of pixels expected bit-identical in parity math mode
EFFECT_BIT_EXACT_FRAC = 0.93  # the same with procedural effects (their hash magnifies sin's last bit)
EFFECT_FAR_FRAC = 0.05        # with effects: pixels allowed to differ by more than 1 %
EFFECT_BIAS = 0.02            # with effects: relative difference of the image means
ENV_BIT_EXACT_FRAC = 0.85     # with an environment map: every sky pixel runs atan2/acos


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def make_tracer(scene, st, **kw):  # kw: CudaPathTracer options (bvh="sah" selects the SAH traversal tree)
    t = CudaPathTracer(**kw)
    assert t.configure(st)
    assert t.load_scene_snapshot(scene)
    assert t.build_or_update_acceleration()
    assert t.reset_accumulation()
    return t


def film_report(gpu_sum, ref_sum, ref_samples, spp):
    g = gpu_sum / spp
    r = ref_sum / spp
    diff = g - r
    rmse = float(np.sqrt(np.mean(diff ** 2)))
    mean = float(np.mean(r)) + 1e-12
    if ref_samples is not None and ref_samples.shape[0] > 1:
        sd = np.std(ref_samples, axis=0, ddof=1) / np.sqrt(ref_samples.shape[0])
        fail = np.abs(diff) > 3.0 * sd + 1e-6 * (1.0 + np.abs(r))
        sigma3 = float(np.mean(fail))
    else:
        sigma3 = 0.0
    exact = float(np.mean(np.all(bits(gpu_sum) == bits(ref_sum), axis=-1)))
    return {"rmse_rel": rmse / mean, "sigma3_fail": sigma3, "bit_exact": exact}


# ------------------------------------------------------------------ hit ids
BVHS = ["reference", "sah"]


@pytest.mark.parametrize("bvh", BVHS)
@pytest.mark.parametrize("name", ["box", "field", "sphere"])
def test_closest_hit_ids_bit_exact_vs_reference_golden(name, bvh):
    d = cases.load_fixture(name)
    sc = cases.scene_from_arrays(d)
    st = scenes.RenderSettings(width=8, height=8, spp=1)
    with make_tracer(sc, st, bvh=bvh) as t:
        p, tt = t.trace_rays(d["rays"])
    assert np.array_equal(p, d["hit_prim"]), f"{np.sum(p != d['hit_prim'])} mismatching ids"
    assert np.array_equal(bits(tt), bits(d["hit_t"]))


@pytest.mark.parametrize("bvh", BVHS)
def test_closest_hit_ids_bit_exact_larger_sphere(bvh):
    sc = scenes.displaced_sphere(resolution=256, seed=2)
    rays = scenes.ray_query_rays(sc, primary_side=256, random_count=65536, seed=4)
    o = oracle.load("auto")
    pr, tr, _, _ = o.intersect(sc, rays, threads=8)
    with make_tracer(sc, scenes.RenderSettings(width=8, height=8, spp=1), bvh=bvh) as t:
        p, tt = t.trace_rays(rays)
        info = t.accel_info()
    assert info["primitive_count"] == sc.triangle_count
    assert np.array_equal(p, pr), f"{np.sum(p != pr)} mismatching ids of {len(p)}"
    assert np.array_equal(bits(tt), bits(tr))


@pytest.mark.parametrize("bvh", BVHS)
def test_exact_ties_follow_reference_visit_order(bvh):
    """Rays through shared quad diagonals and box edges produce exact-t ties."""
    sc = scenes.cornell_box(seed=1)
    cam = sc.camera
    rays = scenes.primary_rays(cam, 512, 512)
    o = oracle.load("auto")
    pr, tr, _, _ = o.intersect(sc, rays, threads=8)
    with make_tracer(sc, scenes.RenderSettings(width=8, height=8, spp=1), bvh=bvh) as t:
        p, tt = t.trace_rays(rays)
    assert np.array_equal(p, pr)
    assert np.array_equal(bits(tt), bits(tr))


@pytest.mark.parametrize("bvh", BVHS)
def test_parallel_axis_rays_match_reference_rule(bvh):
    sc = scenes.displaced_sphere(resolution=64, seed=5)
    rng = np.random.default_rng(7)
    n = 20000
    o = rng.uniform(-30, 30, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d[: n // 3, 1] = rng.uniform(-1e-4, 1e-4, n // 3)
    d[n // 3: 2 * n // 3, 2] = 0.0
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.ascontiguousarray(np.concatenate([o, d.astype(np.float32)], 1), np.float32)
    pr, tr, _, _ = oracle.load("auto").intersect(sc, rays, threads=8)
    with make_tracer(sc, scenes.RenderSettings(width=8, height=8, spp=1), bvh=bvh) as t:
        p, tt = t.trace_rays(rays)
    assert np.array_equal(p, pr)
    # any-hit must apply the same rule: occluded exactly when the closest hit lies before tmax
    tmax = np.where(np.isfinite(tr), tr * np.float32(1.5), np.float32(100.0)).astype(np.float32)
    with make_tracer(sc, scenes.RenderSettings(width=8, height=8, spp=1), bvh=bvh) as t:
        occ, _ = t.trace_rays(rays, mode=native.QUERY_ANY, tmax=tmax)
    assert np.array_equal(occ.astype(bool), np.isfinite(tr) & (tr < tmax))


@pytest.mark.parametrize("bvh", BVHS)
def test_any_hit_equals_closest_hit_before_tmax(bvh):
    d = cases.load_fixture("sphere")
    sc = cases.scene_from_arrays(d)
    rays = d["rays"]
    tref = d["hit_t"]
    rng = np.random.default_rng(3)
    tmax = np.where(np.isfinite(tref), tref * rng.uniform(0.5, 1.5, tref.shape), rng.uniform(1, 80, tref.shape))
    tmax = tmax.astype(np.float32)
    tmax[:50] = tref[:50]          # t == tmax exactly: not occluded (strict)
    with make_tracer(sc, scenes.RenderSettings(width=8, height=8, spp=1), bvh=bvh) as t:
        occ, _ = t.trace_rays(rays, mode=native.QUERY_ANY, tmax=tmax)
        occ_inf, _ = t.trace_rays(rays, mode=native.QUERY_ANY)
    expect = (tref < tmax) & np.isfinite(tref)
    assert np.array_equal(occ.astype(bool), expect)
    assert np.array_equal(occ_inf.astype(bool), np.isfinite(tref))


def test_external_bvh_gives_same_hits():
    d = cases.load_fixture("field")
    sc = cases.scene_from_arrays(d)
    nodes, prim = oracle.load("auto").build_bvh(sc)
    t = CudaPathTracer()
    assert t.configure(scenes.RenderSettings(width=8, height=8, spp=1))
    assert t.load_scene_snapshot(sc)
    assert t.load_bvh(nodes, prim)
    p, _ = t.trace_rays(d["rays"])
    t.close()
    assert np.array_equal(p, d["hit_prim"])


# ------------------------------------------------------------------ films
@pytest.mark.parametrize("name", ["box", "field", "sdf", "lens"])
def test_film_matches_reference_golden(name):
    d = cases.load_fixture(name)
    sc, st = cases.scene_from_arrays(d), cases.settings_from_arrays(d)
    with make_tracer(sc, st) as t:
        for s in range(st.spp):
            assert t.render_tile(RenderTile(0, 0, st.width, st.height, s), 0)
        g, cnt, inv = t.film()
        c = t.read_counters()
    assert np.array_equal(cnt, d["film_count"])
    rep = film_report(g, d["film_sum"], d["samples"], st.spp)
    print(name, rep)
    assert rep["rmse_rel"] < RMSE_REL_TOL
    assert rep["sigma3_fail"] < SIGMA3_FAIL_FRAC
    assert rep["bit_exact"] >= BIT_EXACT_FRAC
    assert c["samples"] == int(d["counters"][0])


def test_film_matches_oracle_sphere_field_mixed_materials():
    sc = scenes.sphere_field(8, 15, 18, seed=4, light_size=3.0, light_height=8.0)
    st = scenes.RenderSettings(width=96, height=64, spp=4, max_depth=10, seed=1234)
    ref = oracle.load("auto").render(sc, st, threads=8, per_sample=True)
    with make_tracer(sc, st) as t:
        t.render_frame(0, st.spp)
        g, cnt, _ = t.film()
    rep = film_report(g, ref["sum"], ref["samples"], st.spp)
    print(rep)
    assert np.array_equal(cnt, ref["count"])
    assert rep["rmse_rel"] < RMSE_REL_TOL
    assert rep["sigma3_fail"] < SIGMA3_FAIL_FRAC


@pytest.mark.parametrize("nee", [True, False])
def test_film_matches_oracle_material_effects(nee):
    """Procedural material effects 1..19 (one box each, parquet floor, check
    wall), evaluated in the trace loop and in next-event estimation."""
    sc = scenes.effect_gallery()
    st = scenes.RenderSettings(width=96, height=80, spp=4, max_depth=6, seed=21, enable_nee=nee, enable_mis=nee)
    ref = oracle.load("auto").render(sc, st, threads=8, per_sample=True)
    with make_tracer(sc, st) as t:
        t.render_frame(0, st.spp)
        g, cnt, _ = t.film()
    rep = film_report(g, ref["sum"], ref["samples"], st.spp)
    # The effects' hash, fract(sin(.) * 43758.5), magnifies a last-bit
    # difference of sin into a visibly different value, so a few paths take
    # other roulette decisions and become independent samples: those pixels
    # differ by sampling noise (the 3-sigma test), the rest agree exactly or
    # nearly, and the image has no bias.
    rel = np.abs(g - ref["sum"]) / np.maximum(np.abs(ref["sum"]), 1e-3)
    far = float(np.mean(np.any(rel > 1e-2, axis=-1)))
    bias = abs(float(np.mean(g)) - float(np.mean(ref["sum"]))) / float(np.mean(ref["sum"]))
    print(rep, "pixels off by > 1%:", far, "mean bias:", bias)
    assert np.array_equal(cnt, ref["count"])
    assert rep["sigma3_fail"] < SIGMA3_FAIL_FRAC
    assert rep["bit_exact"] >= EFFECT_BIT_EXACT_FRAC
    assert far < EFFECT_FAR_FRAC
    assert bias < EFFECT_BIAS


def test_film_matches_oracle_environment_map():
    """Escaping paths sample an equirectangular sky map; the lookup's atan2 and
    acos are the only new transcendentals, and they touch no path decision."""
    sc = scenes.sky_scene()
    st = scenes.RenderSettings(width=96, height=64, spp=4, max_depth=8, seed=17)
    ref = oracle.load("auto").render(sc, st, threads=8, per_sample=True)
    with make_tracer(sc, st) as t:
        t.render_frame(0, st.spp)
        g, cnt, _ = t.film()
    rep = film_report(g, ref["sum"], ref["samples"], st.spp)
    print(rep)
    assert np.array_equal(cnt, ref["count"])
    assert rep["rmse_rel"] < RMSE_REL_TOL
    assert rep["sigma3_fail"] < SIGMA3_FAIL_FRAC
    assert rep["bit_exact"] >= ENV_BIT_EXACT_FRAC


@pytest.mark.parametrize("name", cases.SCENE_DOCUMENTS)
def test_film_matches_reference_scene_documents(name):
    """The reference's own scene files as its converter produces them
    (dynamic-transform instances, SDF primitives, transmissive materials),
    against the reference CPU tracer's film of the same snapshot."""
    d = cases.load_scene_fixture(name)
    sc, st = cases.scene_from_arrays(d), cases.settings_from_arrays(d)
    with make_tracer(sc, st) as t:
        t.render_frame(0, st.spp)
        g, cnt, _ = t.film()
        c = t.read_counters()
    rep = film_report(g, d["film_sum"], d["samples"], st.spp)
    print(name, rep)
    assert np.array_equal(cnt, d["film_count"])
    assert c["samples"] == int(d["counters"][0])
    assert rep["rmse_rel"] < RMSE_REL_TOL
    assert rep["sigma3_fail"] < SIGMA3_FAIL_FRAC
    assert rep["bit_exact"] >= BIT_EXACT_FRAC


@pytest.mark.parametrize("variant", ["gallery", "glass", "complexity"])
def test_film_matches_oracle_sdf_primitives(variant):
    """SDF primitives next to the triangle BVH: analytic ellipsoid, marched
    box / rounded box / torus / capsule / plane; "glass" makes the ellipsoid
    transmissive (the shadow loop steps through it), "complexity" has no
    triangles at all."""
    sc = {"gallery": scenes.sdf_gallery, "glass": lambda: scenes.sdf_gallery(glass=True),
          "complexity": scenes.sdf_complexity}[variant]()
    st = scenes.RenderSettings(width=96, height=72, spp=4, max_depth=8, seed=23)
    ref = oracle.load("auto").render(sc, st, threads=8, per_sample=True)
    with make_tracer(sc, st) as t:
        t.render_frame(0, st.spp)
        g, cnt, _ = t.film()
        c = t.read_counters()
    rep = film_report(g, ref["sum"], ref["samples"], st.spp)
    print(variant, rep, {k: c[k] for k in ("sdf_tests", "sdf_steps", "sdf_hits", "sdf_misses")},
          {k: ref["counters"][k] for k in ("sdf_tests", "sdf_hits")})
    assert np.array_equal(cnt, ref["count"])
    assert rep["rmse_rel"] < RMSE_REL_TOL
    assert rep["sigma3_fail"] < SIGMA3_FAIL_FRAC
    assert rep["bit_exact"] >= BIT_EXACT_FRAC
    # every extension ray tests every primitive; shadow rays stop at the first occluder
    assert c["sdf_tests"] >= c["rays"] * sc.sdf.shape[0]
    assert 0 < c["sdf_hits"] <= c["sdf_tests"] and c["sdf_misses"] == c["sdf_tests"] - c["sdf_hits"]


def test_unknown_sdf_shape_never_hits():
    """A shape code outside the six (SdfShape::Unknown) is skipped, as the
    reference's switch default does: the film equals the scene without it."""
    sc = scenes.sdf_gallery()
    st = scenes.RenderSettings(width=48, height=36, spp=2, max_depth=6, seed=3)
    with make_tracer(sc, st) as t:
        t.render_frame(0, st.spp)
        a, _, _ = t.film()
    bad = sc.sdf.copy()
    bad[0, 0] = 6.0
    sc2 = scenes.sdf_gallery()
    sc2.sdf = np.concatenate([bad[:1], sc.sdf[1:]])
    sc3 = scenes.sdf_gallery()
    sc3.sdf = np.ascontiguousarray(sc.sdf[1:])
    with make_tracer(sc2, st) as t:
        t.render_frame(0, st.spp)
        b, _, _ = t.film()
    with make_tracer(sc3, st) as t:
        t.render_frame(0, st.spp)
        c, _, _ = t.film()
    assert np.array_equal(b, c) and not np.array_equal(a, b)


def test_render_frame_batches_equal_per_tile_calls():
    sc = scenes.cornell_box(seed=1)
    st = scenes.cornell_settings(40, 32, 5)
    with make_tracer(sc, st) as a:
        for s in range(st.spp):
            assert a.render_tile(RenderTile(0, 0, 40, 32, s), 0)
        fa, ca, _ = a.film()
    with make_tracer(sc, st, wave_paths=40 * 32 * 2) as b:
        b.render_frame(0, st.spp)
        fb, cb, _ = b.film()
    assert np.array_equal(bits(fa), bits(fb)) and np.array_equal(ca, cb)


def test_tiles_equal_full_frame_and_partial_tile_touches_only_its_pixels():
    """The reference's CheckScalarRenderTilePrimitive (tests/snapshot_bus_smoke.cpp:1368-1435)."""
    sc = scenes.cornell_box(seed=1)
    st = scenes.cornell_settings(40, 32, 2)
    with make_tracer(sc, st) as full, make_tracer(sc, st) as tiled, make_tracer(sc, st) as part:
        for s in range(2):
            assert full.render_tile(RenderTile(0, 0, 40, 32, s), 0)
            assert tiled.render_tiles([RenderTile(0, 0, 40, 16, s), RenderTile(0, 16, 40, 16, s)], 0)
        assert part.render_tile(RenderTile(8, 4, 10, 7, 0), 0)
        ff, fc, _ = full.film()
        tf, tc, _ = tiled.film()
        pf, pc, _ = part.film()
    assert np.array_equal(bits(ff), bits(tf)) and np.array_equal(fc, tc)
    mask = np.zeros((32, 40), bool)
    mask[4:11, 8:18] = True
    assert np.all(pc[mask] == 1) and np.all(pc[~mask] == 0)
    assert np.all(pf[~mask] == 0)


def test_lifecycle_and_reset_preserve_acceleration():
    sc = scenes.cornell_box(seed=1)
    st = scenes.cornell_settings(16, 16, 1)
    t = CudaPathTracer()
    assert t.status().lifecycle == "uninitialized"
    assert not t.render_tile(RenderTile(0, 0, 16, 16, 0), 0)
    assert t.load_scene_snapshot(sc).code == native.NOT_READY
    assert t.configure(st)
    assert t.status().lifecycle == "configured"
    assert t.build_or_update_acceleration().code == native.NOT_READY
    assert t.load_scene_snapshot(sc)
    assert t.status().lifecycle == "scene_loaded"
    assert not t.render_tile(RenderTile(0, 0, 16, 16, 0), 0)
    assert "acceleration" in t.status().last_error
    assert t.build_or_update_acceleration()
    s = t.status()
    assert s.lifecycle == "ready" and s.ready_to_render
    assert t.render_tile(RenderTile(0, 0, 16, 16, 0), 0)
    a, _, _ = t.film()
    gen = t.status().accumulation_gen
    assert t.reset_accumulation()
    s = t.status()
    assert s.accel_valid and s.accumulation_gen == gen + 1 and s.total_samples == 0
    assert t.render_tile(RenderTile(0, 0, 16, 16, 0), 0)
    b, _, _ = t.film()
    assert np.array_equal(bits(a), bits(b))
    t.shutdown()
    assert t.status().lifecycle == "uninitialized"
    t.close()


def test_resolve_hdr_and_film_resume():
    sc = scenes.cornell_box(seed=1)
    st = scenes.cornell_settings(24, 16, 4)
    with make_tracer(sc, st) as a:
        a.render_frame(0, 4)
        fa, ca, _ = a.film()
        hdr = a.resolve_hdr()
    assert np.array_equal(bits(hdr), bits(fa * (np.float32(1.0) / ca[..., None].astype(np.float32))))
    with make_tracer(sc, st) as b:
        b.render_frame(0, 2)
        half_f, half_c, _ = b.film()
    with make_tracer(sc, st) as c:
        assert c.replace_film_history(half_f, half_c)
        c.render_frame(2, 2)
        fc, cc, _ = c.film()
    assert np.array_equal(bits(fa), bits(fc)) and np.array_equal(ca, cc)


def test_fast_math_mode_is_statistically_equal():
    sc = scenes.cornell_box(seed=1)
    st = scenes.cornell_settings(48, 40, 16)
    ref = oracle.load("auto").render(sc, st, threads=8, per_sample=True)
    with make_tracer(sc, st, math_mode=1) as t:
        t.render_frame(0, st.spp)
        g, _, _ = t.film()
    rep = film_report(g, ref["sum"], ref["samples"], st.spp)
    print(rep)
    assert rep["rmse_rel"] < 0.05


def test_sah_traversal_tree_renders_identical_films():
    """The SAH traversal tree changes only the visiting order: every hit (id, t)
    is the reference's, so films are bit-identical to the reference tree's."""
    cases_ = [(scenes.cornell_box(seed=1), scenes.cornell_settings(48, 40, 3)),
              (scenes.sphere_field(8, 15, 18, seed=4, light_size=3.0, light_height=8.0),
               scenes.RenderSettings(width=96, height=64, spp=3, max_depth=12, seed=7, firefly_clamp=10.0))]
    for sc, st in cases_:
        with make_tracer(sc, st) as a, make_tracer(sc, st, bvh="sah") as b:
            a.render_frame(0, st.spp)
            b.render_frame(0, st.spp)
            fa, ca, _ = a.film()
            fb, cb, _ = b.film()
        assert np.array_equal(ca, cb) and np.array_equal(bits(fa), bits(fb))


RESOLVES = [dict(), dict(tone_map="reinhard", exposure=1.7), dict(tone_map="filmic", white_balance_kelvin=3200.0),
            dict(tone_map="aces", output_transform="linear"), dict(tone_map="linear", clamp_output=False, gamma=1.8,
                                                                   white_balance_kelvin=9000.0)]


def test_device_ldr_resolve_matches_apply_film_resolve():
    """resolve_ldr on the device against the reference's ApplyFilmResolve of
    the same HDR film (the film's per-pixel mean): equal bytes except where
    gamma's pow lands on a rounding boundary (at most one step)."""
    sc = scenes.cornell_box(seed=1)
    st = scenes.cornell_settings(96, 64, 3)
    o = oracle.load("auto")
    with make_tracer(sc, st) as t:
        t.render_frame(0, st.spp)
        hdr = t.resolve_hdr().reshape(st.height, st.width, 3)
        for kw in RESOLVES:
            g = t.resolve_ldr(**kw)
            r = o.apply_film_resolve(hdr, **kw)
            d = np.abs(g.astype(np.int32) - r.astype(np.int32))
            print(kw, "identical", float(np.mean(d == 0)), "max", int(d.max()))
            assert d.max() <= 1 and np.mean(d == 0) >= 0.999, kw


def test_split_film_readback():
    """request_film_readback / poll_film: pending until the GPU work behind the
    token is done, then the resolved image; an unknown token is invalid."""
    import time
    sc = scenes.cornell_box(seed=1)
    st = scenes.cornell_settings(256, 192, 8)
    with make_tracer(sc, st) as t:
        t.render_frame(0, st.spp, sync=False)
        tok = t.request_film_readback(tone_map="aces")
        deadline = time.time() + 30.0
        state, img = t.poll_film(tok)
        while state == native.READBACK_PENDING and time.time() < deadline:
            time.sleep(0.001)
            state, img = t.poll_film(tok)
        assert state == native.READBACK_READY
        assert np.array_equal(img, t.resolve_ldr(tone_map="aces"))
        assert t.poll_film(tok + 7)[0] == native.READBACK_INVALID
