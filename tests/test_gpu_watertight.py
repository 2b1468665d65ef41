"""The watertight triangle test on the device (VKPTC_TRIANGLE_WATERTIGHT)
against the oracle port's restatement of the same test (itself validated
against FP64 in tests/test_watertight_oracle.py):

* closest-hit ids and distances bit-exact, any-hit exactly the port's closest
  t < tmax, with either traversal tree;
* no ray from inside a closed mesh aimed at its vertices and edges misses;
* films of watertight renders within the film tolerances of the port's
  watertight render, also after instance transform refits;
* the modes that keep Moller-Trumbore records refuse the option.
"""
import ctypes

import numpy as np
import pytest

import oracle
from tests.golden import cases
from tests.test_gpu_parity import BIT_EXACT_FRAC, RMSE_REL_TOL, SIGMA3_FAIL_FRAC, film_report
from vkpathtracer_b200 import native, scenes
from vkpathtracer_b200.tracer import BatchRenderer, CudaPathTracer, RenderTile

pytestmark = pytest.mark.gpu

MISS = 0xFFFFFFFF


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def wt_tracer(sc, st=None, **kw):
    t = CudaPathTracer(triangle_test="watertight", **kw)
    assert t.configure(st or scenes.RenderSettings(width=8, height=8, spp=1))
    assert t.load_scene_snapshot(sc)
    assert t.build_or_update_acceleration()
    return t


@pytest.fixture(scope="module")
def port():
    return oracle.load("port")


@pytest.mark.parametrize("bvh", ["reference", "sah"])
@pytest.mark.parametrize("name", ["box", "field", "sphere"])
def test_watertight_hits_bit_exact_vs_port(port, name, bvh):
    d = cases.load_fixture(name)
    sc = cases.scene_from_arrays(d)
    rays = d["rays"]
    with port.triangle_test("watertight"):
        pp, tp, _, _ = port.intersect(sc, rays, threads=8)
    with wt_tracer(sc, bvh=bvh) as t:
        p, tt = t.trace_rays(rays)
        tmax = np.where(np.isfinite(tp), tp * np.float32(1.0001), np.float32(50.0)).astype(np.float32)
        a, _ = t.trace_rays(rays, mode=native.QUERY_ANY, tmax=tmax)
    assert np.array_equal(p, pp), f"{np.sum(p != pp)} mismatching ids"
    assert np.array_equal(bits(tt), bits(tp))
    assert np.array_equal(a.astype(bool), (pp != MISS) & (tp < tmax))


@pytest.mark.parametrize("bvh", ["reference", "sah"])
def test_closed_mesh_has_no_leaks(port, bvh):
    sc = scenes.displaced_sphere(resolution=192, amplitude=0.05, octaves=6, seed=5, scale=16.0, weld_poles=True)
    origins = [(0.0, 0.0, 0.0), (2.9, -3.3, 1.1), (-7.25, 5.5, -0.75), (0.0, 12.0, 0.0), (1e-3, -14.0, 2e-3)]
    rays = scenes.edge_probe_rays(sc, origins, max_rays=400000, seed=1)
    with wt_tracer(sc, bvh=bvh) as t:
        p, tt = t.trace_rays(rays)
    with CudaPathTracer(bvh=bvh) as m:
        assert m.configure(scenes.RenderSettings(width=8, height=8, spp=1))
        assert m.load_scene_snapshot(sc) and m.build_or_update_acceleration()
        pm, _ = m.trace_rays(rays)
    print(f"{rays.shape[0]} rays at vertices and edges: watertight misses {int(np.sum(p == MISS))}, "
          f"Moller-Trumbore misses {int(np.sum(pm == MISS))}")
    assert np.all(p != MISS)
    with port.triangle_test("watertight"):
        pp, tp, _, _ = port.intersect(sc, rays[:50000], threads=8)
    assert np.array_equal(p[:50000], pp) and np.array_equal(bits(tt[:50000]), bits(tp))


@pytest.mark.parametrize("name", ["box", "field"])
def test_watertight_render_matches_port(port, name):
    d = cases.load_fixture(name)
    sc, st = cases.scene_from_arrays(d), cases.settings_from_arrays(d)
    with port.triangle_test("watertight"):
        ref = port.render(sc, st, threads=8, per_sample=True)
    with wt_tracer(sc, st) as t:
        assert t.reset_accumulation()
        t.render_frame(0, st.spp)
        g, cnt, _ = t.film()
    rep = film_report(g, ref["sum"], ref["samples"], st.spp)
    print(name, rep)
    assert np.array_equal(cnt, ref["count"])
    assert rep["rmse_rel"] < RMSE_REL_TOL and rep["sigma3_fail"] < SIGMA3_FAIL_FRAC
    assert rep["bit_exact"] >= BIT_EXACT_FRAC


def test_watertight_refit_matches_port(port):
    d = cases.load_scene_fixture("cornell_native")
    sc, st = cases.scene_from_arrays(d), cases.settings_from_arrays(d)
    ups = cases.transform_updates(sc, 1.0, 3)
    with port.triangle_test("watertight"):
        ref = port.render(sc, st, per_sample=True, updates=ups)
    with wt_tracer(sc, st) as t:
        t.update_instance_transforms(ups)
        assert t.reset_accumulation()
        t.render_frame(0, st.spp)
        g, cnt, _ = t.film()
    rep = film_report(g, ref["sum"], ref["samples"], st.spp)
    print(rep)
    assert np.array_equal(cnt, ref["count"])
    assert rep["rmse_rel"] < RMSE_REL_TOL and rep["bit_exact"] >= BIT_EXACT_FRAC


def test_watertight_records_hold_vertices():
    """Triangle records of the watertight build carry the vertices where the
    Moller-Trumbore build carries v0 and the two edges."""
    sc = scenes.cornell_box(seed=1)
    with wt_tracer(sc) as t:
        rec = t.read_accel(native.ACCEL_TRIANGLES).reshape(-1, 12)   # uint32 words
    prim = rec[:, 9]
    tri = sc.indices.reshape(-1, 3)[prim]   # one instance after another: primitive = triangle
    want = np.concatenate([sc.vertices[tri[:, 0]], sc.vertices[tri[:, 1]], sc.vertices[tri[:, 2]]], axis=1)
    assert np.array_equal(rec[:, 0:9], bits(want))


def test_modes_without_watertight_records_refuse_it():
    sc = scenes.cornell_box(seed=1)
    st = scenes.RenderSettings(width=16, height=16, spp=1)
    host = CudaPathTracer(triangle_test="watertight", build="host")
    assert host.configure(st) and host.load_scene_snapshot(sc)
    assert host.build_or_update_acceleration().code == native.UNSUPPORTED
    ext = CudaPathTracer(triangle_test="watertight")
    assert ext.configure(st) and ext.load_scene_snapshot(sc)
    nodes, prim = oracle.load("port").build_bvh(sc)
    assert ext.load_bvh(nodes, prim).code == native.UNSUPPORTED
    adj = wt_tracer(sc, st)
    with pytest.raises(native.VkptcError) as e:
        adj.adjoint_setup(1)
    assert e.value.code == native.UNSUPPORTED
    lib = native.load()
    cfg = native.Config()
    cfg.triangle_test = 2
    handle = ctypes.c_void_p()
    assert lib.vkptc_create(ctypes.byref(cfg), ctypes.byref(handle)) == native.INVALID_ARGUMENT
    assert lib.vkptc_batch_create(ctypes.byref(cfg), ctypes.byref(handle)) == native.INVALID_ARGUMENT


def test_watertight_batch_equals_single_context_renders():
    """Every batch driver traverses watertight jobs with the watertight test:
    each job's film equals that job rendered alone by a watertight context."""
    jobs = [(scenes.cornell_box(seed=1), scenes.cornell_settings(48, 40, 3)),
            (scenes.sphere_field(3, 9, 10, seed=21, n_lights=3, light_size=1.5, light_height=5.0),
             scenes.RenderSettings(width=40, height=30, spp=2, max_depth=6, seed=77)),
            (cases.lens_scene("many_blades"), scenes.RenderSettings(width=32, height=24, spp=2, max_depth=5, seed=3))]
    with BatchRenderer(triangle_test="watertight") as b:
        for sc, st in jobs:
            b.add_job(sc, st)
        b.run("persistent")
        pers = [b.film(j) for j in range(len(jobs))]
        b.run("loop")
        loop = [b.film(j) for j in range(len(jobs))]
        b.run("plain")
        plain = [b.film(j) for j in range(len(jobs))]
    for (sc, st), (lf, lc), (pf, pc), (sf, scn) in zip(jobs, loop, plain, pers):
        with wt_tracer(sc, st) as t:
            assert t.reset_accumulation()
            for s in range(st.spp):
                assert t.render_tile(RenderTile(0, 0, st.width, st.height, s), 0)
            g, cnt, _ = t.film()
        assert np.array_equal(lc, cnt) and np.array_equal(pc, cnt) and np.array_equal(scn, cnt)
        assert np.array_equal(bits(lf), bits(g)) and np.array_equal(bits(pf), bits(g))
        assert np.array_equal(bits(sf), bits(g))
