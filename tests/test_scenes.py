"""Seeded generators: deterministic, with the workload sizes the benchmarks quote."""
import numpy as np

from vkpathtracer_b200 import scenes


def test_generators_are_deterministic():
    a, b = scenes.cornell_box(1), scenes.cornell_box(1)
    assert np.array_equal(a.vertices, b.vertices) and np.array_equal(a.materials, b.materials)
    assert a.triangle_count == 36
    r1 = scenes.random_rays(1000, 24.0, 3)
    r2 = scenes.random_rays(1000, 24.0, 3)
    assert np.array_equal(r1, r2)
    assert np.allclose(np.linalg.norm(r1[:, 3:], axis=1), 1.0, atol=1e-6)


def test_ray_query_sizes():
    # 2 * (n - 1) * n triangles for an n x n grid sphere: 1,046,904 at n = 724.
    sc = scenes.displaced_sphere(resolution=32)
    assert sc.triangle_count == 2 * 31 * 32
    assert 2 * 723 * 724 == 1_046_904
    rays = scenes.ray_query_rays(sc, primary_side=16, random_count=100)
    assert rays.shape == (16 * 16 + 100, 6) and rays.dtype == np.float32


def test_sphere_grid_size_and_material_mix():
    sc = scenes.sphere_field(8, 15, 18, seed=4)
    assert sc.triangle_count == 64 * 504 + 2 + 16 * 2
    models = sc.materials[: 64, 7]
    rough = sc.materials[: 64, 6]
    assert (models == 2).sum() > 0 and (models == 3).sum() > 0 and (models == 0).sum() > 0
    assert np.all(rough[models == 2] == 0.0)
    assert sc.lights.shape == (16, 16)


def test_batch_jobs_ranges():
    jobs = scenes.batch_jobs(count=6, max_triangles=20_000, max_side=256)
    for j in jobs:
        assert 128 <= j.settings.width <= 256 and j.settings.width == j.settings.height
        assert j.settings.spp in (4, 8, 16, 32, 64) and j.settings.max_depth in (4, 8, 16)
