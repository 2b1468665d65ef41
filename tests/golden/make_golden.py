"""Regenerates the golden fixtures of tests/golden from the REFERENCE itself.

Run in a container that has the reference sources (the reference oracle
oracle/_ref/libvkptref.so is built from them by oracle/Makefile):

    python tests/golden/make_golden.py [case ...]     (default: every case)

Each fixture is a small .npz: the inputs are regenerated from the seeded
scene generators at test time, the outputs come from the reference's own
ScalarCpuPathTracer / CpuBvhAccelerator / ParallelBvhBuilder.
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from tests.golden import cases  # noqa: E402


def main():
    oracle.build_ref()
    ref = oracle.load("reference")
    only = set(sys.argv[1:])
    for name, (scene_fn, settings_fn, rays_fn) in cases.CASES.items():
        if only and name not in only:
            continue
        scene = scene_fn()
        out = cases.scene_to_arrays(scene)
        nodes, prim = ref.build_bvh(scene)
        out["bvh_nodes_sha256"] = np.frombuffer(hashlib.sha256(nodes.tobytes() + prim.tobytes()).digest(), np.uint8)
        out["bvh_node_count"] = np.array([nodes.shape[0]], np.int64)
        if settings_fn is not None:
            st = settings_fn()
            out.update(cases.settings_to_arrays(st))
            r = ref.render(scene, st, per_sample=True)
            out["film_sum"] = r["sum"]
            out["film_count"] = r["count"]
            out["samples"] = r["samples"]
            c = r["counters"]
            out["counters"] = np.array([c["samples"], c["rays"], c["triangle_tests"], c["triangle_hits"],
                                        c["bvh_node_visits"], c["bvh_leaf_visits"], c["shadow_tests"]], np.uint64)
            if scene.sdf is not None:
                out["sdf_counters"] = np.array([c["sdf_tests"], c["sdf_steps"], c["sdf_hits"], c["sdf_misses"]],
                                               np.uint64)
        if rays_fn is not None:
            rays = rays_fn(scene)
            out["rays"] = rays
            p, t, stats, _ = ref.intersect(scene, rays, threads=4, stats=True)
            out["hit_prim"] = p
            out["hit_t"] = t
            out["ray_stats"] = stats
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(name, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
