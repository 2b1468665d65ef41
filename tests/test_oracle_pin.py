"""Pins the CPU restatement (oracle/port.cpp) to the reference.

Against the golden fixtures (outputs of the reference's own CPU tracer,
made by tests/golden/make_golden.py) everywhere, and against the live
reference oracle (oracle/_ref/libvkptref.so) where it was built, over a
material/light set that walks every branch of the integrator.
"""
import hashlib

import numpy as np
import pytest

import oracle
from tests.golden import cases
from vkpathtracer_b200 import scenes


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.fixture(scope="module")
def port():
    return oracle.load("port")


@pytest.mark.parametrize("name", ["box", "field", "sdf", "lens"])
def test_port_film_matches_reference_golden(port, name):
    d = cases.load_fixture(name)
    scene, st = cases.scene_from_arrays(d), cases.settings_from_arrays(d)
    r = port.render(scene, st, per_sample=True)
    assert np.array_equal(bits(r["sum"]), bits(d["film_sum"]))
    assert np.array_equal(r["count"], d["film_count"])
    assert np.array_equal(bits(r["samples"]), bits(d["samples"]))
    c = r["counters"]
    got = np.array([c["samples"], c["rays"], c["triangle_tests"], c["triangle_hits"], c["bvh_node_visits"],
                    c["bvh_leaf_visits"], c["shadow_tests"]], np.uint64)
    assert np.array_equal(got, d["counters"])
    if "sdf_counters" in d:
        sdf = np.array([c["sdf_tests"], c["sdf_steps"], c["sdf_hits"], c["sdf_misses"]], np.uint64)
        assert np.array_equal(sdf, d["sdf_counters"])


@pytest.mark.parametrize("name", ["box", "field", "sphere"])
def test_port_bvh_matches_reference_golden(port, name):
    d = cases.load_fixture(name)
    nodes, prim = port.build_bvh(cases.scene_from_arrays(d))
    h = np.frombuffer(hashlib.sha256(nodes.tobytes() + prim.tobytes()).digest(), np.uint8)
    assert nodes.shape[0] == int(d["bvh_node_count"][0])
    assert np.array_equal(h, d["bvh_nodes_sha256"])


@pytest.mark.parametrize("name", ["box", "field", "sphere"])
def test_port_hits_match_reference_golden(port, name):
    d = cases.load_fixture(name)
    p, t, stats, _ = port.intersect(cases.scene_from_arrays(d), d["rays"], threads=2, stats=True)
    assert np.array_equal(p, d["hit_prim"])
    assert np.array_equal(bits(t), bits(d["hit_t"]))
    assert np.array_equal(stats, d["ray_stats"])


def material_zoo_scene():
    """Every material class the integrator branches on, spot and sphere lights."""
    sc = scenes.cornell_box(seed=9)
    mats = sc.materials.copy()
    extra = [
        scenes.material(albedo=(0.9, 0.6, 0.3), roughness=0.3, model=4, metallic=0.9),        # metal
        scenes.material(albedo=(0.8, 0.9, 1.0), roughness=0.05, model=5, ior=1.45, transmission=0.9, alpha=0.7),
        scenes.material(albedo=(0.5, 0.2, 0.2), roughness=0.4, model=7, clearcoat=0.6),       # clearcoat
        scenes.material(albedo=(0.3, 0.5, 0.2), roughness=0.6, model=6, sheen=0.8),           # sheen
        scenes.material(albedo=(0.7, 0.7, 0.2), roughness=0.9, model=8),                      # toon
        scenes.material(albedo=(0.9, 0.9, 0.9), roughness=0.0, model=2),                      # mirror
        scenes.material(albedo=(0.2, 0.2, 0.2), emissive=(2.0, 1.0, 0.5), roughness=0.7, model=1),
    ]
    base = mats.shape[0]
    mats = np.concatenate([mats, np.array(extra)])
    inst = sc.instances.copy()
    # walls 0..4 keep diffuse; boxes get metal / transmissive; floor clearcoat etc.
    inst[5, 2] = base + 0
    inst[6, 2] = base + 1
    inst[0, 2] = base + 2
    inst[3, 2] = base + 3
    inst[4, 2] = base + 4
    inst[2, 2] = base + 5
    inst[1, 2] = base + 6
    lights = np.concatenate([sc.lights,
                             scenes.point_light((0.2, 0.8, 0.1), (3.0, 3.0, 3.0), 0.05, radius=0.05)[None],
                             scenes.point_light((-0.3, 0.9, -0.2), (1.0, 2.0, 4.0), 0.2, radius=0.0,
                                                direction=(0.3, -1.0, 0.1), spot_inner_cos=0.9,
                                                spot_outer_cos=0.7)[None]])
    return scenes.Scene(sc.vertices, sc.indices, inst, mats, lights, (0.05, 0.04, 0.03), sc.camera, "zoo").contiguous()


@pytest.mark.skipif(not oracle.have_reference(), reason="reference oracle not built here")
@pytest.mark.parametrize("nee,mis", [(True, True), (True, False), (False, False)])
def test_port_matches_live_reference_material_zoo(port, nee, mis):
    ref = oracle.load("reference")
    sc = material_zoo_scene()
    st = scenes.RenderSettings(width=40, height=32, spp=2, max_depth=7, seed=99, enable_nee=nee, enable_mis=mis)
    a = ref.render(sc, st)
    b = port.render(sc, st)
    assert np.array_equal(bits(a["sum"]), bits(b["sum"]))
    assert np.array_equal(a["count"], b["count"])
    for k in ("samples", "rays", "triangle_tests", "triangle_hits", "bvh_node_visits", "bvh_leaf_visits",
              "shadow_tests"):
        assert a["counters"][k] == b["counters"][k], k


@pytest.mark.skipif(not oracle.have_reference(), reason="reference oracle not built here")
@pytest.mark.parametrize("nee,mis", [(True, True), (False, False)])
def test_port_matches_live_reference_material_effects(port, nee, mis):
    """Procedural material effects 1..19 (apply_material_effect) in the trace
    loop and in next-event estimation."""
    ref = oracle.load("reference")
    sc = scenes.effect_gallery()
    st = scenes.RenderSettings(width=48, height=40, spp=2, max_depth=6, seed=5, enable_nee=nee, enable_mis=mis)
    a = ref.render(sc, st)
    b = port.render(sc, st)
    assert np.array_equal(bits(a["sum"]), bits(b["sum"]))
    assert np.array_equal(a["count"], b["count"])
    assert a["counters"]["rays"] == b["counters"]["rays"]


SDF_SCENES = {"gallery": lambda: scenes.sdf_gallery(), "glass": lambda: scenes.sdf_gallery(glass=True),
              "complexity": lambda: scenes.sdf_complexity()}


@pytest.mark.skipif(not oracle.have_reference(), reason="reference oracle not built here")
@pytest.mark.parametrize("variant", list(SDF_SCENES))
@pytest.mark.parametrize("nee,mis", [(True, True), (False, False)])
def test_port_matches_live_reference_sdf_primitives(port, variant, nee, mis):
    """SDF primitives (intersect_scene's loop after the triangles): analytic
    sphere, sphere-traced box / rounded box / plane / torus / capsule with
    rotations and scales, a transmissive SDF in the shadow loop, and a scene
    with no triangles."""
    ref = oracle.load("reference")
    sc = SDF_SCENES[variant]()
    st = scenes.RenderSettings(width=48, height=36, spp=2, max_depth=6, seed=9, enable_nee=nee, enable_mis=mis)
    a = ref.render(sc, st)
    b = port.render(sc, st)
    assert np.array_equal(bits(a["sum"]), bits(b["sum"]))
    assert np.array_equal(a["count"], b["count"])
    for k in ("samples", "rays", "shadow_tests", "sdf_tests", "sdf_steps", "sdf_hits", "sdf_misses",
              "triangle_tests", "bvh_node_visits"):
        assert a["counters"][k] == b["counters"][k], k
    assert a["counters"]["sdf_hits"] > 0


def test_lens_golden_uses_the_lens_shape(port):
    """The lens fixture's film depends on the iris and the squeeze: the same
    render with a round, unsqueezed lens differs."""
    d = cases.load_fixture("lens")
    scene, st = cases.scene_from_arrays(d), cases.settings_from_arrays(d)
    assert scene.camera.iris_blade_count == 7 and scene.camera.anamorphic_squeeze == np.float32(1.15)
    scene.camera.iris_blade_count, scene.camera.anamorphic_squeeze = 0, 1.0
    r = port.render(scene, st)
    assert not np.array_equal(bits(r["sum"]), bits(d["film_sum"]))


@pytest.mark.skipif(not oracle.have_reference(), reason="reference oracle not built here")
@pytest.mark.parametrize("variant", list(cases.LENS_VARIANTS))
def test_port_matches_live_reference_lens_shapes(port, variant):
    """ScalarCpuPathTracer::camera_rays' polygonal aperture and anamorphic
    squeeze, including its clamps (src/pathtracer/ScalarCpuPathTracer.Render.cpp:88-116)."""
    ref = oracle.load("reference")
    sc = cases.lens_scene(variant)
    st = scenes.RenderSettings(width=32, height=24, spp=3, max_depth=4, seed=5)
    a = ref.render(sc, st)
    b = port.render(sc, st)
    assert np.array_equal(bits(a["sum"]), bits(b["sum"]))
    assert np.array_equal(a["count"], b["count"])


@pytest.mark.skipif(not oracle.have_reference(), reason="reference oracle not built here")
def test_port_matches_live_reference_environment_map(port):
    """Escaping paths sample the equirectangular map (SampleSceneEnvironment)."""
    ref = oracle.load("reference")
    sc = scenes.sky_scene()
    st = scenes.RenderSettings(width=48, height=32, spp=2, max_depth=5, seed=3)
    a = ref.render(sc, st)
    b = port.render(sc, st)
    assert np.array_equal(bits(a["sum"]), bits(b["sum"]))
    plain = scenes.sky_scene()
    plain.env_map = None
    c = ref.render(plain, st)
    assert not np.array_equal(a["sum"], c["sum"])   # the map is actually used


@pytest.mark.skipif(not oracle.have_reference(), reason="reference oracle not built here")
def test_port_matches_live_reference_pixel_list_and_threads(port):
    ref = oracle.load("reference")
    sc = scenes.cornell_box(seed=3)
    st = scenes.cornell_settings(32, 24, 2)
    px = np.arange(0, 32 * 24, 5, dtype=np.uint32)
    a = ref.render(sc, st, pixels=px, threads=3)
    b = port.render(sc, st, pixels=px, threads=2)
    assert np.array_equal(bits(a["sum"]), bits(b["sum"]))
    full = ref.render(sc, st, threads=4)
    c = port.render(sc, st, threads=1)
    assert np.array_equal(bits(full["sum"]), bits(c["sum"]))


@pytest.mark.skipif(not oracle.have_reference(), reason="reference oracle not built here")
def test_port_matches_live_reference_ray_query_with_parallel_axes(port):
    """Rays with |d_axis| <= 1e-4 exercise the reference's parallel-axis slab rule."""
    ref = oracle.load("reference")
    sc = scenes.displaced_sphere(resolution=48, seed=5)
    rng = np.random.default_rng(1)
    n = 3000
    o = rng.uniform(-30, 30, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d[: n // 3, 1] = rng.uniform(-1e-4, 1e-4, n // 3)      # near-parallel to the xz plane
    d[n // 3: 2 * n // 3, 0] = 0.0
    d /= np.linalg.norm(d, axis=1, keepdims=True).astype(np.float32)
    rays = np.ascontiguousarray(np.concatenate([o, d.astype(np.float32)], 1), np.float32)
    pa, ta, sa, _ = ref.intersect(sc, rays, threads=2, stats=True)
    pb, tb, sb, _ = port.intersect(sc, rays, threads=2, stats=True)
    assert np.array_equal(pa, pb)
    assert np.array_equal(bits(ta), bits(tb))
    assert np.array_equal(sa, sb)


@pytest.mark.parametrize("name", cases.SCENE_DOCUMENTS)
def test_port_film_matches_reference_scene_documents(port, name):
    """The reference's own scene files (converted by its SceneDocument loader
    and BuildSceneDataFromDocument): dynamic-transform instances flattened
    through their local geometry and transforms, SDF primitives, transmissive
    and emissive materials; films, per-sample radiance and counters equal the
    reference's."""
    d = cases.load_scene_fixture(name)
    scene, st = cases.scene_from_arrays(d), cases.settings_from_arrays(d)
    r = port.render(scene, st, per_sample=True, threads=4)
    assert np.array_equal(bits(r["sum"]), bits(d["film_sum"]))
    assert np.array_equal(r["count"], d["film_count"])
    assert np.array_equal(bits(r["samples"]), bits(d["samples"]))
    c = r["counters"]
    got = np.array([c["samples"], c["rays"], c["triangle_tests"], c["triangle_hits"], c["bvh_node_visits"],
                    c["bvh_leaf_visits"], c["shadow_tests"]], np.uint64)
    assert np.array_equal(got, d["counters"])
    sdf = np.array([c["sdf_tests"], c["sdf_steps"], c["sdf_hits"], c["sdf_misses"]], np.uint64)
    assert np.array_equal(sdf, d["sdf_counters"])


@pytest.mark.skipif(not oracle.have_reference(), reason="reference oracle not built here")
def test_port_film_resolve_matches_reference(port):
    """ApplyFilmResolve: exposure, white balance (ColorTemperatureToRgb), every
    tone map, gamma and linear output, with and without the clamp; NaN and
    infinite pixels."""
    ref = oracle.load("reference")
    rs = np.random.RandomState(0)
    hdr = (rs.exponential(0.7, (48, 64, 3)) * (rs.rand(48, 64, 1) < 0.98)).astype(np.float32)
    hdr[3, 5, 1], hdr[7, 9, 0] = np.nan, np.inf
    for tm in ("linear", "reinhard", "filmic", "aces"):
        for ot in ("gamma", "linear"):
            for kelvin in (6500.0, 3200.0, 9000.0):
                for clamp in (True, False):
                    kw = dict(exposure=1.3, white_balance_kelvin=kelvin, tone_map=tm, output_transform=ot,
                              gamma=2.2, clamp_output=clamp)
                    assert np.array_equal(ref.apply_film_resolve(hdr, **kw), port.apply_film_resolve(hdr, **kw)), kw


@pytest.mark.skipif(not oracle.have_reference(), reason="reference oracle not built here")
@pytest.mark.parametrize("name", ["cornell_native", "tessellation_sphere_levels", "material_shader_physics_showcase"])
def test_port_instance_refit_matches_reference(port, name):
    """apply_instance_transform_update of the CPU accelerator after the build:
    the port's refit gives the reference's film."""
    ref = oracle.load("reference")
    d = cases.load_scene_fixture(name)
    scene, st = cases.scene_from_arrays(d), cases.settings_from_arrays(d)
    ups = cases.transform_updates(scene)
    a = ref.render(scene, st, updates=ups)
    b = port.render(scene, st, updates=ups)
    assert np.array_equal(bits(a["sum"]), bits(b["sum"]))
    assert a["counters"]["rays"] == b["counters"]["rays"]
    assert not np.array_equal(bits(a["sum"]), bits(d["film_sum"]))
