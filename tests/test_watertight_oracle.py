"""The watertight triangle test of the oracle port (Woop, Benthin and Wald,
"Watertight Ray/Triangle Intersection", JCGT 2(1), 2013), an extension: the
reference traverses with Moller-Trumbore only, so this restatement is
validated here, on the CPU, against an FP64 evaluation, and its agreement with
the reference's Moller-Trumbore is reported, not required.

* Against FP64: on every ray whose FP64 closest hit is unambiguous (the hit
  point at least 1e-6 inside its triangle, the next surface at least 1e-5
  farther, relatively), the same primitive and t within 2e-6 relative; on every
  ray that clears every triangle by 1e-6, a miss.
* Watertight: rays from points inside a closed mesh aimed at every vertex and
  at points on every edge all hit it (Moller-Trumbore's misses are printed).
"""
import numpy as np
import pytest

import oracle
from vkpathtracer_b200 import scenes


@pytest.fixture(scope="module")
def port():
    return oracle.load("port")


def closed_mesh(resolution=32):
    return scenes.displaced_sphere(resolution=resolution, amplitude=0.05, octaves=4, seed=7, scale=16.0,
                                   weld_poles=True)


def fp64_closest(sc, rays, chunk=256):
    """Brute-force FP64 closest hit over every triangle: (prim, t, inside margin,
    relative gap to the next surface, near-miss margin of a miss)."""
    v = sc.vertices.astype(np.float64)
    tri = sc.indices.reshape(-1, 3).astype(np.int64)
    a, b, c = v[tri[:, 0]], v[tri[:, 1]], v[tri[:, 2]]
    e1, e2 = b - a, c - a
    n = rays.shape[0]
    prim = np.full(n, -1, np.int64)
    t_out = np.full(n, np.inf)
    margin = np.zeros(n)
    gap = np.full(n, np.inf)
    for s0 in range(0, n, chunk):
        r = rays[s0:s0 + chunk].astype(np.float64)
        o, d = r[:, None, 0:3], r[:, None, 3:6]
        h = np.cross(d, e2[None])
        det = np.einsum("ijk,jk->ij", h, e1)
        with np.errstate(divide="ignore", invalid="ignore"):
            inv = 1.0 / det
            s = o - a[None]
            u = np.einsum("ijk,ijk->ij", s, h) * inv
            q = np.cross(s, e1[None])
            w = np.einsum("ijk,ijk->ij", np.broadcast_to(d, q.shape), q) * inv
            t = np.einsum("jk,ijk->ij", e2, q) * inv
        bary = np.minimum(np.minimum(u, w), 1.0 - u - w)
        bary = np.where(np.isfinite(bary) & (det != 0.0), bary, -np.inf)
        front = np.isfinite(t) & (t > 1e-4)
        hit = front & (bary >= 0.0)
        tt = np.where(hit, t, np.inf)
        k = np.argmin(tt, axis=1)
        rows = np.arange(r.shape[0])
        t1 = tt[rows, k]
        tt2 = tt.copy()
        tt2[rows, k] = np.inf
        # the nearest other surface the ray comes close to (hit or near miss)
        near = np.where(front & (bary >= -1e-6), t, np.inf)
        near[rows, k] = np.inf
        has = np.isfinite(t1)
        prim[s0:s0 + chunk] = np.where(has, k, -1)
        t_out[s0:s0 + chunk] = t1
        margin[s0:s0 + chunk] = np.where(has, bary[rows, k], np.max(np.where(front, bary, -np.inf), axis=1))
        gap[s0:s0 + chunk] = np.where(has, (near.min(axis=1) - t1) / t1, np.inf)
    return prim, t_out, margin, gap


def test_watertight_port_matches_fp64(port):
    sc = closed_mesh(24)
    rays = np.concatenate([scenes.primary_rays(sc.camera, 40, 40), scenes.random_rays(1500, 1.2, seed=9) * 1.0])
    rays[1600:, 0:3] *= 16.0   # origins spread inside and around the mesh
    rays = np.ascontiguousarray(rays, np.float32)
    with port.triangle_test("watertight"):
        p, t, _, _ = port.intersect(sc, rays, threads=4, stats=True)
    fp, ft, margin, gap = fp64_closest(sc, rays)
    clear_hit = (fp >= 0) & (margin > 1e-6) & (gap > 1e-5)
    clear_miss = (fp < 0) & (margin < -1e-6)
    print("rays", rays.shape[0], "unambiguous hits", int(clear_hit.sum()), "unambiguous misses", int(clear_miss.sum()))
    assert clear_hit.sum() > 1000 and clear_miss.sum() > 100
    assert np.array_equal(p[clear_hit].astype(np.int64), fp[clear_hit])
    rel = np.abs(t[clear_hit].astype(np.float64) - ft[clear_hit]) / ft[clear_hit]
    print("max relative t error", float(rel.max()))
    assert rel.max() < 2e-6
    assert np.all(p[clear_miss] == 0xFFFFFFFF)


def test_watertight_port_has_no_leaks_where_mt_may(port):
    sc = closed_mesh(32)
    origins = [(0.0, 0.0, 0.0), (3.1, -2.7, 1.9), (-6.5, 4.25, -2.0), (0.5, 9.0, 0.25)]
    rays = scenes.edge_probe_rays(sc, origins)
    with port.triangle_test("watertight"):
        p_wt, _, _, _ = port.intersect(sc, rays, threads=8)
    p_mt, _, _, _ = port.intersect(sc, rays, threads=8)
    leaks_wt = int(np.sum(p_wt == 0xFFFFFFFF))
    leaks_mt = int(np.sum(p_mt == 0xFFFFFFFF))
    print(f"{rays.shape[0]} rays at vertices and edges: watertight misses {leaks_wt}, Moller-Trumbore misses {leaks_mt}")
    assert leaks_wt == 0


def test_watertight_agreement_with_reference_mt_reported(port):
    """Reported, not required: the share of rays whose watertight closest hit
    is the reference Moller-Trumbore's (they differ on near-edge rays and
    where the reference's |det| < 1e-4 cull rejects a triangle)."""
    sc = closed_mesh(48)
    rays = scenes.ray_query_rays(sc, primary_side=96, random_count=8192, scale=16.0, seed=3)
    p_mt, _, _, _ = port.intersect(sc, rays, threads=8)
    with port.triangle_test("watertight"):
        p_wt, _, _, _ = port.intersect(sc, rays, threads=8)
    agree = float(np.mean(p_mt == p_wt))
    print(f"watertight vs reference Moller-Trumbore: {agree:.6f} of {rays.shape[0]} closest-hit ids agree")
    assert agree > 0.99


def test_reference_oracle_refuses_the_watertight_test():
    if not oracle.have_reference():
        pytest.skip("reference oracle not built here")
    ref = oracle.load("reference")
    with pytest.raises(RuntimeError):
        with ref.triangle_test("watertight"):
            pass
