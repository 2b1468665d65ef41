"""The accelerator built on the device (the default) against the host build
(the parity mode, a restatement of the reference's ParallelBvhBuilder pinned
to it by the golden fixtures).

* Reference traversal tree: every device array the traversal reads -- wide
  nodes, triangle records, tie records, shading records -- is bit-identical to
  the host build's, on scenes that reach every branch of the builder (a root
  leaf, a root small enough for the per-thread builder, level-synchronous
  levels, invalid and zero-count instances, no triangles).
* SAH traversal tree: the device's own binned-SAH tree; tie and shading
  records equal the host's, and closest-hit ids and distances equal the
  reference tree's on every ray.
* Non-finite vertices send the build to the host path (same arrays).
"""
import numpy as np
import pytest

from tests.golden import cases
from vkpathtracer_b200 import native, scenes
from vkpathtracer_b200.tracer import CudaPathTracer

pytestmark = pytest.mark.gpu

ARRAYS = {"wide": native.ACCEL_WIDE_NODES, "tris": native.ACCEL_TRIANGLES, "tie": native.ACCEL_TIE_NODES,
          "shade": native.ACCEL_SHADING}


def built(sc, build, bvh="reference"):
    t = CudaPathTracer(bvh=bvh, build=build)
    assert t.configure(scenes.RenderSettings(width=8, height=8, spp=1)).ok
    assert t.load_scene_snapshot(sc).ok
    assert t.build_or_update_acceleration().ok
    return t


def arrays(t):
    out = {k: t.read_accel(v) for k, v in ARRAYS.items()}
    info = t.accel_info()
    info.pop("build_ms")
    return out, info


def tiny_scene(n_tris, seed=0, extra_instances=()):
    rs = np.random.RandomState(seed)
    v = rs.uniform(-1, 1, (3 * n_tris, 3)).astype(np.float32)
    idx = np.arange(3 * n_tris, dtype=np.uint32).reshape(-1, 3)
    inst = [(0, n_tris, 0)] + list(extra_instances)
    mats = np.array([scenes.material()])
    return scenes.Scene(v, idx, np.array(inst, np.uint32), mats, np.zeros((0, 16), np.float32)).contiguous()


def scene_cases():
    yield "box", scenes.cornell_box(seed=1)
    yield "field", scenes.sphere_field(3, 9, 10, seed=21, n_lights=3, light_size=1.5, light_height=5.0)
    yield "sphere", cases._sphere()
    yield "sdf", scenes.sdf_gallery()
    yield "root_leaf", tiny_scene(3)
    yield "root_small", tiny_scene(40)
    yield "two_levels", tiny_scene(300, seed=2)
    # invalid triangles (index past the end), an instance past the index array, a zero-count instance
    bad = tiny_scene(200, seed=3, extra_instances=[(190, 20, 0), (5000, 3, 0), (10, 0, 0)])
    bad.indices[7] = (0, 1, 10 ** 6)
    yield "invalid_and_empty_instances", bad
    # the reference's own scene documents: dynamic-transform instances with local geometry
    for name in ("cornell_native", "tessellation_sphere_levels", "material_shader_physics_showcase"):
        yield name, cases.scene_from_arrays(cases.load_scene_fixture(name))


@pytest.mark.parametrize("name,sc", list(scene_cases()))
def test_device_build_equals_host_build(name, sc):
    a, ia = arrays(built(sc, "device"))
    b, ib = arrays(built(sc, "host"))
    assert ia == ib, (ia, ib)
    for k in ARRAYS:
        assert a[k].size == b[k].size, k
        assert np.array_equal(a[k], b[k]), k


def test_scene_without_triangles():
    sc = scenes.sdf_complexity()
    t = built(sc, "device")
    assert t.accel_info()["primitive_count"] == 0
    for k in ARRAYS:
        assert t.read_accel(ARRAYS[k]).size == 0


def test_full_frame_scene_device_build_equals_host_build():
    """2,064,418 triangles: the level-synchronous path at full size."""
    sc = scenes.sphere_grid()
    td = built(sc, "device")
    th = built(sc, "host")
    a, ia = arrays(td)
    b, ib = arrays(th)
    print("device build", td.accel_info()["build_ms"], "ms; host build", th.accel_info()["build_ms"], "ms")
    assert ia == ib
    for k in ARRAYS:
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("name,sc", [c for c in scene_cases() if c[0] in ("box", "field", "sphere", "two_levels")])
def test_device_sah_tree_gives_reference_hits(name, sc):
    rays = np.concatenate([scenes.primary_rays(sc.camera, 96, 64),
                           scenes.random_rays(20000, 1.0, seed=5)]).astype(np.float32)
    ts = built(sc, "device", bvh="sah")
    tr = built(sc, "host", bvh="reference")
    sa, sb = arrays(ts)[0], arrays(tr)[0]
    assert np.array_equal(sa["tie"], sb["tie"]) and np.array_equal(sa["shade"], sb["shade"])
    p1, t1 = ts.trace_rays(rays)
    p2, t2 = tr.trace_rays(rays)
    assert np.array_equal(p1, p2)
    assert np.array_equal(t1.view(np.uint32), t2.view(np.uint32))
    a1, _ = ts.trace_rays(rays, mode=native.QUERY_ANY)
    a2, _ = tr.trace_rays(rays, mode=native.QUERY_ANY)
    assert np.array_equal(a1, a2)


def test_nonfinite_vertex_falls_back_to_host_build():
    sc = tiny_scene(100, seed=4)
    sc.vertices[5, 1] = np.nan
    a, ia = arrays(built(sc, "device"))
    b, ib = arrays(built(sc, "host"))
    assert ia == ib
    for k in ARRAYS:
        assert np.array_equal(a[k], b[k]), k
