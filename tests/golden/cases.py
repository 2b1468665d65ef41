"""Small parity cases shared by the golden fixtures and the parity tests.

Each case: (scene factory, render-settings factory or None, ray factory or None).
Sizes are chosen so the CPU oracle finishes each in well under a second.
"""
import numpy as np

from vkpathtracer_b200 import scenes


def _box():
    return scenes.cornell_box(seed=1)


def _box_settings():
    return scenes.RenderSettings(width=48, height=40, spp=3, max_depth=8, seed=1234, enable_nee=True, enable_mis=True)


def _box_rays(scene):
    prim = scenes.primary_rays(scene.camera, 64, 48)
    rnd = scenes.random_rays(2048, 0.45, seed=11)
    rnd[:, 1] += 0.5   # origins inside the room
    return np.ascontiguousarray(np.concatenate([prim, rnd]))


def _field():
    return scenes.sphere_field(3, 9, 10, seed=21, n_lights=3, light_size=1.5, light_height=5.0)


def _field_settings():
    return scenes.RenderSettings(width=40, height=30, spp=2, max_depth=6, seed=77, enable_nee=True, enable_mis=True)


def _field_rays(scene):
    return scenes.primary_rays(scene.camera, 48, 36)


def _sphere():
    return scenes.displaced_sphere(resolution=64, amplitude=0.05, octaves=8, seed=2, scale=16.0)


def _sphere_rays(scene):
    return scenes.ray_query_rays(scene, primary_side=48, random_count=4096, scale=16.0, seed=3)


def _sdf():
    return scenes.sdf_gallery()


def _sdf_settings():
    return scenes.RenderSettings(width=48, height=36, spp=2, max_depth=6, seed=4321, enable_nee=True, enable_mis=True)


def _lens():
    """The Cornell box through a thin lens with the iris and squeeze of the
    reference's shallow depth-of-field scene document (7 blades rotated 12
    degrees, roundness 0.42, anamorphic squeeze 1.15)."""
    sc = scenes.cornell_box(seed=1)
    c = sc.camera
    c.aperture_radius, c.focus_distance = 0.1, 1.5
    c.iris_blade_count, c.iris_rotation_degrees, c.iris_roundness, c.anamorphic_squeeze = 7, 12.0, 0.42, 1.15
    return sc


# Lens shapes (blades, rotation degrees, roundness, squeeze) that reach each
# branch and clamp of ScalarCpuPathTracer::camera_rays' thin-lens sampling.
LENS_VARIANTS = {
    "pentagon_sharp": (5, -30.0, 0.0, 1.0),
    "many_blades": (64, 400.0, 0.5, 0.7),
    "too_many_blades": (200, 3.0, 0.2, 2.0),        # clamped to 64
    "two_blades": (2, 0.0, 0.0, 1.3),               # below 3: round
    "round_enough": (6, 0.0, 0.9995, 1.0),          # roundness >= 0.999: round
    "nan_roundness": (6, 10.0, float("nan"), 1.0),  # clamp01(NaN) = 0
    "tiny_squeeze": (0, 0.0, 1.0, 0.001),           # at least 0.01
    "inf_squeeze": (8, 0.0, 0.3, float("inf")),     # non-finite: 1
}


def lens_scene(variant):
    """The Cornell box through a thin lens of LENS_VARIANTS[variant]."""
    sc = scenes.cornell_box(seed=1)
    c = sc.camera
    c.aperture_radius, c.focus_distance = 0.12, 1.4
    c.iris_blade_count, c.iris_rotation_degrees, c.iris_roundness, c.anamorphic_squeeze = LENS_VARIANTS[variant]
    return sc


def _lens_settings():
    return scenes.RenderSettings(width=48, height=40, spp=4, max_depth=6, seed=99, enable_nee=True, enable_mis=True)


CASES = {
    "box": (_box, _box_settings, _box_rays),
    "lens": (_lens, _lens_settings, None),
    "field": (_field, _field_settings, _field_rays),
    "sphere": (_sphere, None, _sphere_rays),
    "sdf": (_sdf, _sdf_settings, None),
}


# ---- fixture (de)serialisation: the fixtures carry their exact inputs
def scene_to_arrays(scene):
    c = scene.camera
    out = {
        "vertices": scene.vertices, "indices": scene.indices, "instances": scene.instances,
        "materials": scene.materials, "lights": scene.lights,
        "environment": np.array(scene.environment, np.float32),
        "camera": np.array(list(c.position) + list(c.target) + list(c.up) +
                           [c.fov_deg, c.aperture_radius, c.focus_distance], np.float32),
        "camera_lens": np.array([c.iris_blade_count, c.iris_rotation_degrees, c.iris_roundness,
                                 c.anamorphic_squeeze], np.float32),
    }
    if scene.sdf is not None:
        out["sdf"] = np.ascontiguousarray(scene.sdf, np.float32)
    if scene.instance_local is not None:
        out["instance_local"] = np.ascontiguousarray(scene.instance_local, np.uint32)
        out["instance_transforms"] = np.ascontiguousarray(scene.instance_transforms, np.float32)
        out["local_vertices"] = np.ascontiguousarray(scene.local_vertices, np.float32)
        out["local_indices"] = np.ascontiguousarray(scene.local_indices, np.uint32)
    if scene.env_map is not None:
        out["env_map"] = np.ascontiguousarray(scene.env_map, np.float32)
        out["env_scale"] = np.array(scene.env_scale, np.float32)
    return out


def scene_from_arrays(d):
    cam = d["camera"].astype(np.float64)
    camera = scenes.Camera(tuple(cam[0:3]), tuple(cam[3:6]), tuple(cam[6:9]), float(cam[9]), float(cam[10]),
                           float(cam[11]))
    if "camera_lens" in d:
        lens = d["camera_lens"].astype(np.float64)
        camera.iris_blade_count = int(lens[0])
        camera.iris_rotation_degrees, camera.iris_roundness, camera.anamorphic_squeeze = (float(x) for x in lens[1:])
    return scenes.Scene(d["vertices"], d["indices"], d["instances"], d["materials"], d["lights"],
                        tuple(float(x) for x in d["environment"]), camera, "fixture",
                        env_map=d.get("env_map"),
                        env_scale=tuple(float(x) for x in d["env_scale"]) if "env_scale" in d else (0.0, 0.0, 0.0),
                        sdf=d.get("sdf"), instance_local=d.get("instance_local"),
                        instance_transforms=d.get("instance_transforms"), local_vertices=d.get("local_vertices"),
                        local_indices=d.get("local_indices")).contiguous()


def settings_to_arrays(st):
    return {"settings": np.array([st.width, st.height, st.spp, st.max_depth, st.seed, int(st.enable_nee),
                                  int(st.enable_mis), st.russian_roulette_start_depth], np.uint64),
            "settings_rr": np.array([st.russian_roulette_min_survival, st.russian_roulette_max_survival], np.float32)}


def settings_from_arrays(d):
    a = [int(x) for x in d["settings"]]
    rr = d["settings_rr"]
    return scenes.RenderSettings(width=a[0], height=a[1], spp=a[2], max_depth=a[3], seed=a[4],
                                 enable_nee=bool(a[5]), enable_mis=bool(a[6]), russian_roulette_start_depth=a[7],
                                 russian_roulette_min_survival=float(rr[0]),
                                 russian_roulette_max_survival=float(rr[1]))


def load_fixture(name):
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), f"{name}.npz")
    return dict(np.load(path))


# ---- the reference's own scene documents, converted by its SceneDocument loader and
# BuildSceneDataFromDocument (tests/golden/make_scene_fixtures.py)
SCENE_DOCUMENTS = ["cornell_native", "glass_lab", "material_gauntlet", "mirror_room", "neon_room", "shadow_study",
                   "sdf_complexity", "tessellation_sphere_levels", "ecs_lifecycle_scripting_demo",
                   "particle_benchmark_simple", "material_shader_physics_showcase"]


def scene_document_settings():
    return scenes.RenderSettings(width=64, height=48, spp=4, max_depth=8, seed=4321, enable_nee=True, enable_mis=True)


def load_scene_fixture(name):
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "scenes", f"{name}.npz")
    return dict(np.load(path))


def transform_updates(scene, step=1.0, count=3):
    """Instance transform updates for the first `count` dynamic-transform
    instances with local geometry: a shift, a rotation about y, a 5 % scale."""
    import math
    il = scene.instance_local
    dyn = [i for i in range(scene.instances.shape[0]) if il[i, 0] & 1 and il[i, 2] and il[i, 4]]
    ups = []
    for k, i in enumerate(dyn[:count]):
        t = scene.instance_transforms[i]
        a = (0.3 + 0.2 * k) * step
        ups.append({"instance": i, "translation": (t[0] + 0.05 * (k + 1) * step, t[1] + 0.02 * step, t[2] - 0.03),
                    "rotation": (0.0, math.sin(a / 2), 0.0, math.cos(a / 2)), "scale": tuple(t[7:10] * 1.05)})
    return ups
