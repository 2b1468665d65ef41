"""Converts the reference's own scene documents into snapshot fixtures.

Run where the reference sources are present (the reference oracle
oracle/_ref/libvkptref.so compiles its SceneDocument loader and
BuildSceneDataFromDocument, src/pathtracer/SceneConversion.cpp):

    python tests/golden/make_scene_fixtures.py [name ...]

Each fixture tests/golden/scenes/<name>.npz holds the converted
PathTracerSceneSnapshot (triangles, dynamic-transform instances with their
local geometry, SDF primitives, materials, lights, camera) and the reference
CPU tracer's film of it at cases.scene_document_settings() (per-sample
radiance and counters).  Scene documents that reference model files absent
from the reference checkout are not converted.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from tests.golden import cases  # noqa: E402

SCENE_DIR = os.path.join(oracle.REFERENCE_DIR, "assets", "scenes")


def main():
    oracle.build_ref()
    ref = oracle.load("reference")
    names = sys.argv[1:] or cases.SCENE_DOCUMENTS
    os.makedirs(os.path.join(HERE, "scenes"), exist_ok=True)
    for name in names:
        scene = ref.convert_scene_json(os.path.join(SCENE_DIR, f"{name}.json"))
        out = cases.scene_to_arrays(scene)
        st = cases.scene_document_settings()
        out.update(cases.settings_to_arrays(st))
        r = ref.render(scene, st, per_sample=True, threads=8)
        out["film_sum"] = r["sum"]
        out["film_count"] = r["count"]
        out["samples"] = r["samples"]
        c = r["counters"]
        out["counters"] = np.array([c["samples"], c["rays"], c["triangle_tests"], c["triangle_hits"],
                                    c["bvh_node_visits"], c["bvh_leaf_visits"], c["shadow_tests"]], np.uint64)
        out["sdf_counters"] = np.array([c["sdf_tests"], c["sdf_steps"], c["sdf_hits"], c["sdf_misses"]], np.uint64)
        path = os.path.join(HERE, "scenes", f"{name}.npz")
        np.savez_compressed(path, **out)
        print(name, scene.triangle_count, "triangles", os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
