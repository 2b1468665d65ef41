"""Camera and scene deltas on the device (IPathTracer::update_camera,
update_camera_state, update_scene_delta; src/pathtracer/PathTracer.h:1102-1141,
ApplyCameraState and ApplySceneDeltaUpdate, src/pathtracer/PathTracer.cpp:343-483).

* A delta applied to a loaded (and built) context renders exactly what a
  context loaded fresh with the changed scene renders: films, sample counts
  and the accelerator's shading records bit-identical, in both build modes and
  with either traversal tree.
* Every index is checked before anything changes; a rejected delta leaves the
  film and the shading records as they were.
* The thin-lens shapes (polygonal iris, anamorphic squeeze) against the oracle.
"""
import numpy as np
import pytest

import oracle
from tests.golden import cases
from tests.test_gpu_parity import BIT_EXACT_FRAC, RMSE_REL_TOL, SIGMA3_FAIL_FRAC, film_report
from vkpathtracer_b200 import native, scenes
from vkpathtracer_b200.tracer import CudaPathTracer

pytestmark = pytest.mark.gpu

ST = scenes.RenderSettings(width=64, height=48, spp=2, max_depth=6, seed=17)


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def tracer(sc, st=ST, build_now=True, **kw):
    t = CudaPathTracer(**kw)
    assert t.configure(st)
    assert t.load_scene_snapshot(sc)
    if build_now:
        assert t.build_or_update_acceleration()
    return t


def film(t, st=ST):
    assert t.reset_accumulation()
    t.render_frame(0, st.spp)
    s, c, _ = t.film()
    return s.copy(), c.copy()


def assert_same(a, b):
    fa, fb = film(a), film(b)
    assert np.array_equal(fa[1], fb[1])
    assert np.array_equal(bits(fa[0]), bits(fb[0]))
    sa, sb = a.read_accel(native.ACCEL_SHADING), b.read_accel(native.ACCEL_SHADING)
    assert np.array_equal(sa, sb)
    assert a.read_counters()["samples"] == b.read_counters()["samples"]


def field():
    return scenes.sphere_field(3, 9, 10, seed=21, n_lights=3, light_size=1.5, light_height=5.0)


def moved_camera(c):
    return scenes.Camera((c.position[0] + 0.4, c.position[1] + 0.3, c.position[2] - 0.2), c.target, c.up,
                         c.fov_deg * 0.85, 0.08, 6.0, 7, 12.0, 0.42, 1.15)


# ---------------------------------------------------------------- lens shapes
@pytest.mark.parametrize("variant", list(cases.LENS_VARIANTS))
def test_lens_shapes_match_oracle(variant):
    sc = cases.lens_scene(variant)
    st = scenes.RenderSettings(width=48, height=40, spp=4, max_depth=5, seed=5)
    ref = oracle.load("auto").render(sc, st, threads=8, per_sample=True)
    t = tracer(sc, st)
    g, cnt = film(t, st)
    rep = film_report(g, ref["sum"], ref["samples"], st.spp)
    print(variant, rep)
    assert np.array_equal(cnt, ref["count"])
    assert rep["rmse_rel"] < RMSE_REL_TOL
    assert rep["sigma3_fail"] < SIGMA3_FAIL_FRAC
    assert rep["bit_exact"] >= BIT_EXACT_FRAC


# ---------------------------------------------------------------- camera
@pytest.mark.parametrize("build", ["device", "host"])
def test_camera_update_equals_fresh_load(build):
    sc = field()
    cam = moved_camera(sc.camera)
    a = tracer(sc, build=build)
    film(a)   # rendered with the old camera first
    a.update_camera_state(cam)
    got = a.get_camera()
    for k in ("position", "target", "up"):
        assert np.array_equal(np.float32(getattr(got, k)), np.float32(getattr(cam, k))), k
    assert (got.iris_blade_count, np.float32(got.iris_roundness), np.float32(got.anamorphic_squeeze)) == \
        (7, np.float32(0.42), np.float32(1.15))
    sc2 = field()
    sc2.camera = cam
    assert_same(a, tracer(sc2, build=build))


def test_update_camera_keeps_the_lens():
    """update_camera changes position, target, up and field of view only
    (ScalarCpuPathTracer::update_camera, src/pathtracer/ScalarCpuPathTracer.cpp:522-533)."""
    sc = field()
    cam = moved_camera(sc.camera)
    a = tracer(sc)
    a.update_camera_state(cam)
    a.update_camera((1.0, 3.0, 9.0), (0.0, 0.5, 0.0), (0.0, 1.0, 0.0), 50.0)
    sc2 = field()
    sc2.camera = scenes.Camera((1.0, 3.0, 9.0), (0.0, 0.5, 0.0), (0.0, 1.0, 0.0), 50.0, cam.aperture_radius,
                               cam.focus_distance, cam.iris_blade_count, cam.iris_rotation_degrees,
                               cam.iris_roundness, cam.anamorphic_squeeze)
    assert_same(a, tracer(sc2))


# ---------------------------------------------------------------- scene deltas
def delta_and_expected(sc):
    """A delta over materials (one becomes transmissive, one gains an effect),
    lights (a negative radius, clamped as on load), instance materials (one
    instance updated twice: the last wins) and the environment colour, and the
    scene it produces."""
    mats = {}
    glass = sc.materials[2].copy()
    glass[7], glass[9], glass[10] = 5.0, 1.5, 1.0
    mats[2] = glass
    fx = sc.materials[4].copy()
    fx[0:3] = (0.2, 0.7, 0.3)
    fx[15] = 3.0
    mats[4] = fx
    lights = {}
    l0 = sc.lights[0].copy()
    l0[7] = -1.0
    lights[0] = l0
    l2 = sc.lights[2].copy()
    l2[3:6] = (1.0, 0.7, 0.5)
    l2[6] *= 1.8
    lights[2] = l2
    inst = [(1, 3), (5, 0), (1, 7), (6, int(sc.instances[6, 2]))]
    env = (0.03, 0.05, 0.09)
    out = scenes.Scene(sc.vertices.copy(), sc.indices.copy(), sc.instances.copy(), sc.materials.copy(),
                       sc.lights.copy(), env, sc.camera, "expected")
    for k, v in mats.items():
        out.materials[k] = v
    for k, v in lights.items():
        out.lights[k] = v
    for i, m in inst:
        out.instances[i, 2] = m
    return dict(materials=mats, lights=lights, instance_materials=inst, environment=env), out.contiguous()


@pytest.mark.parametrize("build,bvh", [("device", "reference"), ("device", "sah"), ("host", "reference")])
def test_scene_delta_equals_fresh_load(build, bvh):
    sc = field()
    delta, expected = delta_and_expected(sc)
    a = tracer(sc, build=build, bvh=bvh)
    film(a)
    a.update_scene_delta(**delta)
    assert_same(a, tracer(expected, build=build, bvh=bvh))


def test_scene_delta_before_build_and_after_rebuild():
    sc = field()
    delta, expected = delta_and_expected(sc)
    fresh = tracer(expected)
    early = tracer(sc, build_now=False)
    early.update_scene_delta(**delta)
    assert early.build_or_update_acceleration()
    assert_same(early, fresh)
    late = tracer(sc)
    late.update_scene_delta(**delta)
    assert late.build_or_update_acceleration()   # the instance table kept the new materials
    assert_same(late, fresh)


@pytest.mark.parametrize("bad", [
    dict(materials={13: np.zeros(16, np.float32)}),
    dict(lights={3: np.zeros(16, np.float32)}),
    dict(instance_materials={13: 0}),
    dict(instance_materials={0: 13}),
    dict(materials={0: np.ones(16, np.float32)}, instance_materials={99: 0}),   # checked before anything applies
    dict(),                                                                   # nothing changes
    dict(instance_materials={0: 0}),                                          # already that material
])
def test_rejected_scene_delta_changes_nothing(bad):
    sc = field()
    a = tracer(sc)
    before = film(a)
    shade = a.read_accel(native.ACCEL_SHADING)
    with pytest.raises(native.VkptcError) as e:
        a.update_scene_delta(**bad)
    assert e.value.code == native.INVALID_ARGUMENT
    after = film(a)
    assert np.array_equal(bits(before[0]), bits(after[0]))
    assert np.array_equal(shade, a.read_accel(native.ACCEL_SHADING))


def test_updates_need_a_scene():
    t = CudaPathTracer()
    assert t.configure(ST)
    with pytest.raises(native.VkptcError) as e:
        t.update_scene_delta(environment=(1.0, 1.0, 1.0))
    assert e.value.code == native.NOT_READY
    with pytest.raises(native.VkptcError) as e:
        t.update_camera_state(scenes.Camera())
    assert e.value.code == native.NOT_READY


def test_instance_material_delta_survives_transform_refit():
    """The refit of a dynamic-transform instance rewrites its shading records
    from the instance table, which holds the delta's material."""
    d = cases.load_scene_fixture("cornell_native")
    sc = cases.scene_from_arrays(d)
    dyn = [i for i in range(sc.instances.shape[0])
           if sc.instance_local[i, 0] & 1 and sc.instance_local[i, 2] and sc.instance_local[i, 4]]
    assert dyn
    i = dyn[0]
    m = (int(sc.instances[i, 2]) + 1) % sc.materials.shape[0]
    upd = [{"instance": i, "translation": tuple(sc.instance_transforms[i, 0:3] + np.float32(0.05)),
            "rotation": (0.0, 0.2588190, 0.0, 0.9659258), "scale": tuple(sc.instance_transforms[i, 7:10])}]
    d_st = scenes.RenderSettings(width=48, height=36, spp=2, max_depth=6, seed=3)
    a = tracer(sc, d_st)
    a.update_scene_delta(instance_materials={i: m})
    a.update_instance_transforms(upd)
    sc2 = cases.scene_from_arrays(d)
    sc2.instances[i, 2] = m
    b = tracer(sc2, d_st)
    b.update_instance_transforms(upd)
    assert np.array_equal(a.read_accel(native.ACCEL_SHADING), b.read_accel(native.ACCEL_SHADING))
    fa, fb = film(a, d_st), film(b, d_st)
    assert np.array_equal(bits(fa[0]), bits(fb[0]))
