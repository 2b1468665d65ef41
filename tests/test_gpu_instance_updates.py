"""Instance transform updates (apply_instance_transform_update) refitted on
the device, against the reference's CPU accelerator refit (the oracle applies
the same updates after its build): the updated instances' primitives are
recomputed from their local geometry and both trees are refitted with their
topology unchanged, so films equal the reference's after the same update."""
import numpy as np
import pytest

import oracle
from tests.golden import cases
from vkpathtracer_b200 import native
from vkpathtracer_b200.tracer import CudaPathTracer

pytestmark = pytest.mark.gpu

RMSE_REL_TOL = 1e-3
SIGMA3_FAIL_FRAC = 3e-3
BIT_EXACT_FRAC = 0.97
SCENES = ["cornell_native", "tessellation_sphere_levels", "material_shader_physics_showcase"]


def make_updates(sc, step=1.0, count=3):
    return cases.transform_updates(sc, step, count)


def tracer(sc, st, bvh="reference", build="device"):
    t = CudaPathTracer(bvh=bvh, build=build)
    assert t.configure(st).ok and t.load_scene_snapshot(sc).ok and t.build_or_update_acceleration().ok
    return t


def report(g, ref_sum, ref_samples, spp):
    mean = ref_sum / spp
    rmse = float(np.sqrt(np.mean((g / spp - mean) ** 2)) / (np.mean(mean) + 1e-12))
    sd = np.std(ref_samples, axis=0) / np.sqrt(spp)
    fail = float(np.mean(np.abs(g / spp - mean) > 3 * sd + 1e-6))
    exact = float(np.mean(np.all(g.view(np.uint32) == ref_sum.view(np.uint32), axis=-1)))
    return rmse, fail, exact


@pytest.mark.parametrize("bvh", ["reference", "sah"])
@pytest.mark.parametrize("name", SCENES)
def test_refit_matches_reference_refit(name, bvh):
    d = cases.load_scene_fixture(name)
    sc, st = cases.scene_from_arrays(d), cases.settings_from_arrays(d)
    ups = make_updates(sc)
    ref = oracle.load("auto").render(sc, st, per_sample=True, updates=ups)
    with tracer(sc, st, bvh) as t:
        t.update_instance_transforms(ups, check_only=True)
        t.update_instance_transforms(ups)
        t.render_frame(0, st.spp)
        g, cnt, _ = t.film()
    rmse, fail, exact = report(g, ref["sum"], ref["samples"], st.spp)
    print(name, bvh, "rmse", rmse, "3sigma", fail, "bit-exact", exact)
    assert np.array_equal(cnt, ref["count"])
    assert rmse < RMSE_REL_TOL and fail < SIGMA3_FAIL_FRAC and exact >= BIT_EXACT_FRAC


def test_successive_updates_equal_the_last_one():
    """Primitives depend only on the latest transform and every node is
    refitted from them, so two updates equal one with the final transforms."""
    d = cases.load_scene_fixture("cornell_native")
    sc, st = cases.scene_from_arrays(d), cases.settings_from_arrays(d)
    first, last = make_updates(sc, step=2.0), make_updates(sc, step=0.5)
    with tracer(sc, st) as t:
        t.update_instance_transforms(first)
        t.update_instance_transforms(last)
        t.render_frame(0, st.spp)
        a, _, _ = t.film()
        arrays_a = [t.read_accel(k) for k in range(4)]
    with tracer(sc, st) as t:
        t.update_instance_transforms(last)
        t.render_frame(0, st.spp)
        b, _, _ = t.film()
        arrays_b = [t.read_accel(k) for k in range(4)]
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    for x, y in zip(arrays_a, arrays_b):
        assert np.array_equal(x, y)


def test_refit_keeps_topology_and_differs_from_rebuild():
    """A refit is not a rebuild: same node count, the tree of the original
    positions with new bounds (the reference's behaviour)."""
    d = cases.load_scene_fixture("material_shader_physics_showcase")
    sc, st = cases.scene_from_arrays(d), cases.settings_from_arrays(d)
    ups = make_updates(sc, count=8)
    with tracer(sc, st) as t:
        before = t.accel_info()
        t.update_instance_transforms(ups)
        after = t.accel_info()
        refit_nodes = t.read_accel(native.ACCEL_WIDE_NODES)
    assert before["wide_node_count"] == after["wide_node_count"]
    moved = cases.scene_from_arrays(d)
    for u in ups:
        moved.instance_transforms[u["instance"]] = list(u["translation"]) + list(u["rotation"]) + list(u["scale"])
    with tracer(moved, st) as t:
        rebuilt = t.read_accel(native.ACCEL_WIDE_NODES)
    assert refit_nodes.size != rebuilt.size or not np.array_equal(refit_nodes, rebuilt)


def test_rejected_updates():
    d = cases.load_scene_fixture("cornell_native")
    sc, st = cases.scene_from_arrays(d), cases.settings_from_arrays(d)
    with tracer(sc, st) as t:
        with pytest.raises(native.VkptcError) as e:
            t.update_instance_transforms([{"instance": 10 ** 6}])
        assert e.value.code == native.INVALID_ARGUMENT
    d2 = cases.load_scene_fixture("glass_lab")   # no dynamic instances
    sc2 = cases.scene_from_arrays(d2)
    with tracer(sc2, cases.settings_from_arrays(d2)) as t:
        with pytest.raises(native.VkptcError) as e:
            t.update_instance_transforms([{"instance": 0}])
        assert e.value.code == native.UNSUPPORTED
    with tracer(sc, st, build="host") as t:
        with pytest.raises(native.VkptcError) as e:
            t.update_instance_transforms(make_updates(sc))
        assert e.value.code == native.UNSUPPORTED


def test_dynamic_field_refit_matches_reference():
    """Many instances of one local mesh (rotated, scaled), all moved."""
    from vkpathtracer_b200 import scenes
    sc = scenes.dynamic_sphere_field(grid=8)
    st = scenes.RenderSettings(width=96, height=64, spp=4, max_depth=6, seed=11)
    ups = cases.transform_updates(sc, count=64)
    ref = oracle.load("auto").render(sc, st, per_sample=True, updates=ups)
    with tracer(sc, st, "sah") as t:
        t.update_instance_transforms(ups)
        t.render_frame(0, st.spp)
        g, cnt, _ = t.film()
    rmse, fail, exact = report(g, ref["sum"], ref["samples"], st.spp)
    print("dynamic field rmse", rmse, "3sigma", fail, "bit-exact", exact)
    assert np.array_equal(cnt, ref["count"])
    assert rmse < RMSE_REL_TOL and fail < SIGMA3_FAIL_FRAC and exact >= BIT_EXACT_FRAC
