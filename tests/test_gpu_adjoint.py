"""Differentiable rendering: the GPU forward/backward pair (vkptc_forward /
vkptc_backward) on the inverse-rendering box scene (room + 16 boxes, 64
parameters: per-box RGB albedo and roughness).

* The forward's image is bit-identical to the renderer's film resolve (same
  paths, same sample order).
* The backward agrees with the FP64 CPU adjoint (oracle/adjoint.cpp, forward
  mode in double) and with central finite differences (h = 1e-3, common
  random numbers, the unperturbed roulette) taken through the GPU forward,
  leaving out the paths whose discrete decisions flip under the perturbation
  (their boundary terms are outside the estimator).
* The gradient is deterministic; gradient descent lowers the loss.
"""
import numpy as np
import pytest

import oracle
from vkpathtracer_b200 import native, scenes
from vkpathtracer_b200.tracer import CudaPathTracer, material_params

pytestmark = pytest.mark.gpu

OBJ = slice(5, 21)                 # the 16 box materials of inverse_box_scene
GRAD_REL_TOL = 1e-2                # gradient relative error bound
H = 1e-3                           # finite-difference step


def param_index():
    return np.array([(5 + k) * 7 + j for k in range(16) for j in range(4)], np.int64)


def setup(width, height, spp, bvh="reference", scene=None):
    sc = scene if scene is not None else scenes.inverse_box_scene()
    st = scenes.inverse_settings(width, height, spp)
    t = CudaPathTracer(bvh=bvh)
    assert t.configure(st).ok
    assert t.load_scene_snapshot(sc).ok
    assert t.build_or_update_acceleration().ok
    return t, sc, st


def start_params(sc, seed=0):
    rs = np.random.RandomState(seed)
    p = material_params(sc.materials).copy()
    p[OBJ, :3] = rs.uniform(0.1, 0.8, (16, 3))
    p[OBJ, 3] = rs.uniform(0.1, 0.8, 16)
    return p


def rel_err(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("bvh", ["reference", "sah"])
def test_forward_image_equals_renderer_film(bvh):
    t, sc, st = setup(64, 48, 4, bvh)
    t.reset_accumulation()
    t.render_frame(0, 4)
    film = t.resolve_hdr()
    t.adjoint_setup(4)
    loss, img = t.forward(material_params(sc.materials), image=True)
    assert loss == 0.0
    assert np.array_equal(np.ascontiguousarray(img).view(np.uint32),
                          np.ascontiguousarray(film.reshape(img.shape)).view(np.uint32))
    t.close()


def test_loss_is_fp64_mse_of_image():
    t, sc, st = setup(40, 32, 4)
    p = material_params(sc.materials)
    t.adjoint_setup(4)
    _, img = t.forward(p, image=True)
    target = (img * 0.8 + 0.01).astype(np.float32)
    t.adjoint_setup(4, target)
    loss, img2 = t.forward(p, image=True)
    assert np.array_equal(img, img2)
    ref = np.mean((img.astype(np.float64) - target.astype(np.float64)) ** 2)
    assert abs(loss - ref) <= 1e-6 * ref
    t.close()


@pytest.fixture(scope="module")
def problem():
    """48x48, 8 spp: target at the scene's own parameters, start point perturbed."""
    t, sc, st = setup(48, 48, 8)
    t.adjoint_setup(8)
    _, target = t.forward(material_params(sc.materials), image=True)
    t.adjoint_setup(8, target)
    p = start_params(sc)
    loss = t.forward(p)
    grad = t.backward()
    yield t, sc, st, target, p, loss, grad
    t.close()


def test_backward_matches_fp64_adjoint(problem):
    t, sc, st, target, p, loss, grad = problem
    idx = param_index()
    o_loss, o_grad, o_img = oracle.load_adjoint().run(sc, st, p, target, 8, idx, threads=8)
    g = grad.reshape(-1)[idx]
    assert abs(loss - o_loss) <= 1e-3 * o_loss, (loss, o_loss)
    alb = np.arange(64) % 4 != 3
    e_alb, e_rough, e_all = rel_err(g[alb], o_grad[alb]), rel_err(g[~alb], o_grad[~alb]), rel_err(g, o_grad)
    print(f"rel err vs FP64 adjoint: albedo {e_alb:.2e} roughness {e_rough:.2e} all {e_all:.2e}")
    assert e_alb <= GRAD_REL_TOL
    assert e_rough <= GRAD_REL_TOL
    assert e_all <= GRAD_REL_TOL


def test_full_size_backward_matches_fp64_adjoint():
    """128x128, 32 spp, depth 6, all 64 box parameters (the inverse-rendering workload)."""
    import os
    t, sc, st = setup(128, 128, 32)
    t.adjoint_setup(32)
    _, target = t.forward(material_params(sc.materials), image=True)
    t.adjoint_setup(32, target)
    p = start_params(sc, seed=11)
    loss = t.forward(p)
    g = t.backward().reshape(-1)[param_index()]
    o_loss, o_grad, _ = oracle.load_adjoint().run(sc, st, p, target, 32, param_index(),
                                                  threads=os.cpu_count() or 1)
    e = rel_err(g, o_grad)
    print(f"full size: loss {loss:.6e} (fp64 {o_loss:.6e}), gradient rel err {e:.2e}")
    assert abs(loss - o_loss) <= 1e-3 * o_loss
    assert e <= GRAD_REL_TOL
    t.close()


def fd_check(t, p, spp, idx):
    """Central differences through the GPU forward with the roulette of p,
    linearised loss, flipped paths left out; returns (fd, adjoint on the same
    paths, flips)."""
    _, img = t.forward(p, image=True)
    rgb0, sig0 = t.adjoint_samples()
    target = t._fd_target
    npx = img.shape[0] * img.shape[1]
    finite = np.isfinite(rgb0).all(axis=-1)
    cnt = np.maximum(finite.sum(axis=0), 1)
    w = 2.0 * (img.astype(np.float64) - target) / (3.0 * npx) / cnt[..., None]
    fd, adj, flips = [], [], []
    flat = p.reshape(-1)
    for i in idx:
        pp, pm = flat.copy(), flat.copy()
        pp[i] += H
        pm[i] -= H
        t.forward(pp.reshape(p.shape), rr_params=p)
        rp, sp = t.adjoint_samples()
        t.forward(pm.reshape(p.shape), rr_params=p)
        rm, sm = t.adjoint_samples()
        keep = (sp == sig0) & (sm == sig0) & finite
        flips.append(int((~keep & finite).sum()))
        d = (rp.astype(np.float64) - rm) / (2 * H)
        fd.append(float(np.sum(np.where(keep[..., None], d, 0.0) * w[None])))
        t.forward(p)
        g = t.backward(path_weight=keep.astype(np.float32))
        adj.append(float(g.reshape(-1)[i]))
    return np.array(fd), np.array(adj), np.array(flips)


def test_backward_matches_central_finite_differences(problem):
    t, sc, st, target, p, loss, grad = problem
    t._fd_target = target.astype(np.float64)
    idx = param_index()[::3]    # 22 of the 64 parameters, albedo and roughness of every box
    fd, adj, flips = fd_check(t, p, 8, idx)
    g_all = grad.reshape(-1)[idx]
    for i, a, b, c, f in zip(idx, adj, fd, g_all, flips):
        print(f"param {i:4d} adjoint {a:+.6e} fd {b:+.6e} (all paths {c:+.6e}, flips {f})")
    assert rel_err(adj, fd) <= GRAD_REL_TOL
    big = np.abs(fd) > 0.05 * np.abs(fd).max()
    assert np.all(np.abs(adj[big] - fd[big]) <= GRAD_REL_TOL * np.abs(fd[big]) + 1e-7)
    # roulette and albedo never flip a path; only roughness moves directions
    assert all(f == 0 for i, f in zip(idx, flips) if i % 7 != 3)
    t.forward(p)


def test_backward_is_deterministic(problem):
    t, sc, st, target, p, loss, grad = problem
    t.forward(p)
    g1 = t.backward()
    g2 = t.backward()
    assert np.array_equal(g1, g2)
    assert np.array_equal(g1, grad)


def test_decorrelated_backward_replays_the_chosen_frame(problem):
    t, sc, st, target, p, loss, grad = problem
    # replaying the forward's own frame reproduces the ordinary backward exactly
    t.adjoint_setup(8, target, frame=0, decorrelated=True, backward_frame=0)
    assert t.forward(p) == loss
    assert np.array_equal(t.backward(), grad)
    # another frame: independent samples (the shared-sample covariance term
    # of the ordinary gradient is absent, so the two differ)
    t.adjoint_frames(0, 12345)
    t.forward(p)
    g2 = t.backward()
    assert np.all(np.isfinite(g2))
    assert not np.array_equal(g2, grad)
    assert np.abs(g2.reshape(-1)[param_index()]).max() > 0
    t.adjoint_setup(8, target)
    t.forward(p)


def test_recorded_forward_gives_the_replayed_gradient(problem):
    """An ordinary forward writes its paths' vertex records and the backward
    skips the replay; a decorrelated setup whose backward frame is the
    forward's replays the same paths.  Both gradients, with and without path
    weights, are bit-identical, and a weighted backward leaves the records
    for the next one untouched."""
    t, sc, st, target, p, loss, grad = problem
    w = np.random.default_rng(3).uniform(0.0, 2.0, st.width * st.height * 8).astype(np.float32)
    w[::7] = 0.0
    t.adjoint_setup(8, target)
    t.forward(p)
    rec_plain = t.backward()
    rec_weighted = t.backward(path_weight=w)
    assert np.array_equal(t.backward(), rec_plain)
    t.adjoint_setup(8, target, frame=0, decorrelated=True, backward_frame=0)
    t.forward(p)
    assert np.array_equal(t.backward(), rec_plain)
    assert np.array_equal(t.backward(path_weight=w), rec_weighted)
    assert np.array_equal(rec_plain, grad)
    assert not np.array_equal(rec_weighted, rec_plain)
    t.adjoint_setup(8, target)
    t.forward(p)


def test_gradient_descent_lowers_loss():
    t, sc, st = setup(32, 32, 8)
    t.adjoint_setup(8)
    p_true = material_params(sc.materials)
    _, target = t.forward(p_true, image=True)
    t.adjoint_setup(8, target)
    p = start_params(sc, seed=3)
    mask = np.zeros_like(p, bool)
    mask[OBJ, :4] = True
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    first = None
    for k in range(1, 61):
        loss = t.forward(p)
        first = loss if first is None else first
        g = t.backward()
        m = 0.9 * m + 0.1 * g
        v = 0.999 * v + 0.001 * g * g
        step = 0.02 * (m / (1 - 0.9 ** k)) / (np.sqrt(v / (1 - 0.999 ** k)) + 1e-8)
        p = np.where(mask, np.clip(p - step, 0.02, 1.0), p)
    last = t.forward(p)
    print(f"loss {first:.4e} -> {last:.4e}")
    assert last < 0.5 * first
    t.close()


def test_unsupported_material_is_rejected():
    sc = scenes.inverse_box_scene()
    sc.materials[6, 8] = 0.9     # metallic box
    t, _, _ = setup(16, 16, 1, scene=sc)
    with pytest.raises(native.VkptcError) as e:
        t.adjoint_setup(1)
    assert e.value.code == native.UNSUPPORTED
    t.close()


def test_procedural_effect_is_rejected():
    sc = scenes.inverse_box_scene()
    sc.materials[7, 15] = 4.0     # veined box
    t, _, _ = setup(16, 16, 1, scene=sc)
    with pytest.raises(native.VkptcError) as e:
        t.adjoint_setup(1)
    assert e.value.code == native.UNSUPPORTED
    t.close()


def test_sdf_scene_is_rejected():
    sc = scenes.inverse_box_scene()
    sc.sdf = scenes.sdf_primitive("sphere", (0.0, 0.3, 0.0), (0.1, 0.1, 0.1), material=6, radius=1.0)[None]
    t, _, _ = setup(16, 16, 1, scene=sc)
    with pytest.raises(native.VkptcError) as e:
        t.adjoint_setup(1)
    assert e.value.code == native.UNSUPPORTED
    t.close()


def test_backward_before_forward_is_not_ready():
    t, sc, st = setup(16, 16, 1)
    t.adjoint_setup(1)
    with pytest.raises(native.VkptcError) as e:
        t.backward()
    assert e.value.code == native.NOT_READY
    t.close()
