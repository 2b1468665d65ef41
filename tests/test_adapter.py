"""The C++ drop-in: CudaPathTracer (vkpathtracer_b200/host) is a real
vkpt::pathtracer::IPathTracer compiled against the reference's own headers.
oracle/_ref/adapter_check runs it next to the reference's ScalarCpuPathTracer
through that interface with ptbench's render loop and compares the films.
The binary is built where the reference sources exist (oracle/Makefile
`adapter`) and travels with the other built files."""
import os
import subprocess

import numpy as np
import pytest

from tests.conftest import cuda_available
from vkpathtracer_b200 import scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "adapter_check")
needs_bin = pytest.mark.skipif(not os.path.exists(BIN), reason="adapter_check not built (needs the reference sources)")


def write_scene(path, sc, st):
    with open(path, "wb") as f:
        np.array([sc.vertices.shape[0], sc.indices.size, sc.instances.shape[0], sc.materials.shape[0],
                  sc.lights.shape[0]], np.uint32).tofile(f)
        sc.vertices.astype(np.float32).tofile(f)
        sc.indices.astype(np.uint32).tofile(f)
        sc.instances.astype(np.uint32).tofile(f)
        sc.materials.astype(np.float32).tofile(f)
        sc.lights.astype(np.float32).tofile(f)
        np.array(sc.environment, np.float32).tofile(f)
        c = sc.camera
        np.array(list(c.position) + list(c.target) + list(c.up) + [c.fov_deg, c.aperture_radius, c.focus_distance],
                 np.float32).tofile(f)
        np.array([st.width, st.height, st.spp, st.max_depth, int(st.enable_nee), int(st.enable_mis),
                  st.russian_roulette_start_depth], np.uint32).tofile(f)
        np.array([st.seed], np.uint64).tofile(f)
        np.array([st.russian_roulette_min_survival, st.russian_roulette_max_survival], np.float32).tofile(f)
        sdf = sc.sdf if sc.sdf is not None else np.zeros((0, 16), np.float32)
        np.array([sdf.shape[0]], np.uint32).tofile(f)
        sdf.astype(np.float32).tofile(f)
        if sc.instance_local is not None:   # dynamic-transform instances
            lv = np.asarray(sc.local_vertices, np.float32).reshape(-1, 3)
            li = np.asarray(sc.local_indices, np.uint32).reshape(-1)
            np.array([sc.instances.shape[0], lv.shape[0], li.size], np.uint32).tofile(f)
            np.asarray(sc.instance_local, np.uint32).tofile(f)
            np.asarray(sc.instance_transforms, np.float32).tofile(f)
            lv.tofile(f)
            li.tofile(f)


@needs_bin
@pytest.mark.skipif(cuda_available(), reason="checks the no-device path")
def test_adapter_without_device_reports_unsupported():
    r = subprocess.run([BIN, "nodevice"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr


@needs_bin
@pytest.mark.gpu
@pytest.mark.parametrize("which", ["box", "field", "sdf"])
def test_adapter_matches_reference_through_ipathtracer(tmp_path, which):
    if which == "box":
        sc, st = scenes.cornell_box(seed=1), scenes.cornell_settings(64, 48, 3)
    elif which == "sdf":
        sc, st = scenes.sdf_gallery(), scenes.RenderSettings(width=64, height=48, spp=2, max_depth=6, seed=8)
    else:
        sc = scenes.sphere_field(4, 12, 14, seed=5, n_lights=4, light_size=2.0, light_height=6.0)
        st = scenes.RenderSettings(width=64, height=40, spp=2, max_depth=8, seed=31)
    path = os.path.join(tmp_path, "scene.bin")
    write_scene(path, sc, st)
    r = subprocess.run([BIN, path], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr



REFERENCE_SCENES = ["cornell_native", "glass_lab", "tessellation_sphere_levels", "material_shader_physics_showcase",
                    "sdf_complexity", "mirror_room"]


@needs_bin
@pytest.mark.gpu
@pytest.mark.parametrize("name", REFERENCE_SCENES)
def test_adapter_renders_reference_scene_documents(tmp_path, name):
    """The reference's own scene files as its SceneDocument loader and
    BuildSceneDataFromDocument convert them (fixtures made by
    tests/golden/make_scene_fixtures.py), dynamic-transform instances and SDF
    primitives included, rendered through IPathTracer by both tracers: the
    snapshot ptbench's `run --scene <file>.json` hands the cuda backend."""
    from tests.golden import cases
    d = cases.load_scene_fixture(name)
    sc = cases.scene_from_arrays(d)
    st = scenes.RenderSettings(width=64, height=48, spp=2, max_depth=8, seed=1234)
    path = os.path.join(tmp_path, "scene.bin")
    write_scene(path, sc, st)
    r = subprocess.run([BIN, path], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
