"""Failure handling on the GPU, in the forms that fault, trap or hang nothing.

* The persistent batch kernel's grid barrier waits with a bound; a run given a
  bound of one ~128 ns sleep runs out of it at once.  Every block then leaves
  at its next barrier, the call returns VKPTC_TIMEOUT, and the next run of the
  same batch renders films identical to the plain mode.
* A set cancel flag stops vkptc_render before its first tile with
  VKPTC_CANCELLED and the film untouched (the reference's stop checks,
  src/pathtracer/ScalarCpuPathTracer.Render.cpp:166-169, 208-212).
* Malformed scene data is treated as the reference treats it: triangles whose
  vertex indices or instance ranges fall outside the arrays are dropped by the
  accelerator build (src/pathtracer/CpuBvhAccelerator.cpp:173-247), an
  out-of-range material index is clamped to the last material
  (src/pathtracer/ScalarCpuPathTracer.cpp:1058, 1171); arrays the ABI cannot
  read (a null pointer with a non-zero count), and instance ranges of more
  triangles than the wide BVH's leaf references reach (2^28 - 8), are
  VKPTC_INVALID_ARGUMENT.
"""
import ctypes

import numpy as np
import pytest

import oracle
from vkpathtracer_b200 import native, scenes
from vkpathtracer_b200.tracer import BatchRenderer, CudaPathTracer, RenderTile, scene_view

pytestmark = pytest.mark.gpu


def _two_jobs():
    return [(scenes.cornell_box(seed=1), scenes.RenderSettings(width=48, height=40, spp=3, max_depth=8, seed=1234)),
            (scenes.sphere_field(2, 8, 10, seed=3, n_lights=2, light_size=1.0, light_height=4.0),
             scenes.RenderSettings(width=32, height=24, spp=4, max_depth=6, seed=9))]


def test_persistent_barrier_timeout_returns_timeout_and_the_batch_stays_usable():
    with BatchRenderer(device=0) as b:
        for sc, st in _two_jobs():
            b.add_job(sc, st)
        b.run("plain")
        plain = [b.film(j) for j in range(2)]
        with pytest.raises(native.VkptcError) as e:
            b.run("persistent", barrier_spins=1)
        assert e.value.code == native.TIMEOUT, e.value
        assert "barrier" in str(e.value)
        # the same batch object, the default bound: a complete, identical render
        b.run("persistent")
        for j in range(2):
            f, c = b.film(j)
            assert np.array_equal(f, plain[j][0]) and np.array_equal(c, plain[j][1])
        # and the graph-replayed loop driver after it
        b.run("loop")
        for j in range(2):
            f, c = b.film(j)
            assert np.array_equal(f, plain[j][0]) and np.array_equal(c, plain[j][1])


def test_cancel_flag_stops_render_before_any_tile():
    sc = scenes.cornell_box(seed=1)
    st = scenes.cornell_settings(32, 24, 1)
    with CudaPathTracer() as t:
        assert t.configure(st) and t.load_scene_snapshot(sc) and t.build_or_update_acceleration()
        assert t.reset_accumulation()
        lib = native.load()
        tiles = (native.Tile * 2)(native.Tile(0, 0, 16, 24, 0, 0, 0), native.Tile(16, 0, 16, 24, 0, 1, 0))
        flag = ctypes.c_int32(1)
        rc = lib.vkptc_render(t._ctx, tiles, 2, 0, ctypes.byref(flag))
        assert rc == native.CANCELLED
        assert "cancel" in t.status().last_error
        f, c, _ = t.film()
        assert int(c.sum()) == 0 and not np.any(f)
        # cleared flag: both tiles render
        flag.value = 0
        assert lib.vkptc_render(t._ctx, tiles, 2, 0, ctypes.byref(flag)) == native.OK
        _, c, _ = t.film()
        assert int(c.sum()) == 32 * 24


def _malformed_scene():
    """The box room plus three defects: triangles indexing past the vertex
    array, an instance whose triangle range runs past the index array, and an
    instance whose material index is past the material table."""
    sc = scenes.cornell_box(seed=1)
    nv = sc.vertices.shape[0]
    nt = sc.indices.shape[0]
    bad = np.array([[0, 1, nv + 5], [nv, 2, 3]], np.uint32)
    idx = np.concatenate([sc.indices, bad]).astype(np.uint32)
    inst = sc.instances.astype(np.uint32).copy()
    inst[-1, 2] = sc.materials.shape[0] + 40            # material index out of range: clamped
    extra = np.array([[nt, 2, 0],                        # the two bad triangles: dropped
                      [nt + 1, 9, 0]], np.uint32)        # range past the index array: dropped
    return scenes.Scene(sc.vertices, idx, np.concatenate([inst, extra]), sc.materials, sc.lights, sc.environment,
                        sc.camera, "malformed_box")


@pytest.mark.parametrize("build", ["device", "host"])
def test_malformed_scene_is_treated_as_the_reference_treats_it(build):
    sc = _malformed_scene()
    st = scenes.RenderSettings(width=40, height=32, spp=2, max_depth=6, seed=77)
    o = oracle.load("auto")
    rays = scenes.primary_rays(sc.camera, 48, 40)
    rp, rt, _, _ = o.intersect(sc, rays, threads=8)
    ref = o.render(sc, st, threads=8)
    with CudaPathTracer(build=build) as t:
        assert t.configure(st) and t.load_scene_snapshot(sc) and t.build_or_update_acceleration()
        assert t.accel_info()["primitive_count"] == scenes.cornell_box(seed=1).triangle_count
        p, tt = t.trace_rays(rays)
        assert t.reset_accumulation()
        t.render_frame(0, st.spp)
        f, c, _ = t.film()
    assert np.array_equal(p, rp) and np.array_equal(tt.view(np.uint32), rt.view(np.uint32))
    assert np.array_equal(c, ref["count"])
    rel = float(np.sqrt(np.mean((f - ref["sum"]) ** 2)) / (np.mean(ref["sum"]) + 1e-12))
    assert rel < 1e-3, rel


def test_unreadable_scene_arrays_are_invalid_argument():
    sc = scenes.cornell_box(seed=1)
    with CudaPathTracer() as t:
        assert t.configure(scenes.cornell_settings(16, 16, 1))
        v, keep = scene_view(sc)
        v.vertices = None                      # vertex_count stays non-zero
        rc = native.load().vkptc_load_scene(t._ctx, ctypes.byref(v))
        assert rc == native.INVALID_ARGUMENT
        assert "null" in t._err()
        v, keep = scene_view(sc)
        v.instances = None
        assert native.load().vkptc_load_scene(t._ctx, ctypes.byref(v)) == native.INVALID_ARGUMENT
        # instance ranges adding up to more triangles than a wide-BVH leaf can reference
        # (checked before any index is read)
        big = scenes.Scene(sc.vertices, sc.indices, np.array([[0, 1 << 27, 0], [0, 1 << 27, 0]], np.uint32),
                           sc.materials, sc.lights, sc.environment, sc.camera, "too_many_triangles")
        v, keep = scene_view(big)
        assert native.load().vkptc_load_scene(t._ctx, ctypes.byref(v)) == native.INVALID_ARGUMENT
        assert "2^28" in t._err()
        # a well-formed scene afterwards loads and builds
        assert t.load_scene_snapshot(sc) and t.build_or_update_acceleration()
