"""The FP64 CPU adjoint (oracle/adjoint.cpp) against its own central
differences: forward-mode derivatives of the estimator equal the
flip-excluding finite differences (same uniforms, unperturbed roulette).
CPU only; it validates the checker the GPU adjoint tests use."""
import numpy as np

import oracle
from vkpathtracer_b200 import scenes
from vkpathtracer_b200.tracer import material_params


def problem(width=32, height=32, spp=4):
    A = oracle.load_adjoint()
    sc = scenes.inverse_box_scene()
    st = scenes.inverse_settings(width, height, spp)
    p_true = material_params(sc.materials)
    _, _, img = A.run(sc, st, p_true, None, spp, [], threads=4)
    rs = np.random.RandomState(0)
    p = p_true.copy()
    p[5:21, :3] = rs.uniform(0.1, 0.8, (16, 3))
    p[5:21, 3] = rs.uniform(0.1, 0.8, 16)
    return A, sc, st, p, img.astype(np.float32)


def test_primal_image_is_close_to_reference_render():
    A, sc, st, p, _ = problem()
    o = oracle.load("auto").render(sc, st)
    ref = o["sum"] / np.maximum(o["count"], 1)[..., None]
    _, _, img = A.run(sc, st, material_params(sc.materials), None, st.spp, [], threads=4)
    # double vs float primal: the same paths almost everywhere
    close = np.abs(img - ref) <= 1e-4 * np.maximum(1.0, np.abs(ref))
    assert close.mean() > 0.97


def test_forward_mode_matches_finite_differences():
    A, sc, st, p, target = problem()
    idx = np.array([(5 + k) * 7 + j for k in range(16) for j in range(4)])
    loss, g, _ = A.run(sc, st, p, target, st.spp, idx, threads=4)
    assert loss > 0
    fd, flips = A.finite_difference(sc, st, p, target, st.spp, idx, 1e-3, threads=4)
    alb = idx % 7 != 3
    # albedo: no decision depends on it; agreement to rounding
    assert np.allclose(g[alb], fd[alb], rtol=1e-6, atol=1e-12)
    assert flips[alb].sum() == 0
    # roughness: equal wherever no path flipped (to the O(h^2) truncation of central differences)
    clean = ~alb & (flips == 0)
    assert np.allclose(g[clean], fd[clean], rtol=1e-3, atol=1e-9)


def test_roulette_params_change_only_the_roulette():
    A, sc, st, p, target = problem(24, 24, 4)
    l0, _, img0 = A.run(sc, st, p, target, st.spp, [], threads=2)
    l1, _, img1 = A.run(sc, st, p, target, st.spp, [], threads=2, rr_params=p)
    assert l0 == l1 and np.array_equal(img0, img1)
