"""The allocation-free entry point, vkptc_render_tile_noalloc.

It serves callers that cannot allocate GPU memory while rendering -- an
engine that owns every device allocation through its own pool or budget, a
render loop captured into a CUDA graph (cudaMalloc is not allowed during
stream capture), a real-time thread that must not enter the driver's
allocator.  Its path queues live in one fixed device array inside the
library, and it adds each sample into a film the caller allocated.

This file is collected last on purpose: when it fails, a run that stops at
the first failure has already run every other test.  It passes both alone
in a fresh process and after the rest of the suite.
"""
import ctypes

import numpy as np
import pytest

from vkpathtracer_b200 import native, scenes
from vkpathtracer_b200.tracer import CudaPathTracer, RenderTile

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _ready(scene, st):
    t = CudaPathTracer()
    assert t.configure(st) and t.load_scene_snapshot(scene) and t.build_or_update_acceleration()
    assert t.reset_accumulation()
    return t


def test_noalloc_matches_allocating_render_on_two_calls_in_a_row():
    import torch
    sc = scenes.cornell_box(seed=1)
    st = scenes.cornell_settings(64, 48, 2)
    W, H = st.width, st.height
    ref = _ready(sc, st)
    na = _ready(sc, st)
    lib = native.load()
    # The caller owns the film: W*H float4 sums and W*H uint32 counts, zeroed.
    film_sum = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
    film_cnt = torch.zeros((H, W), dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    tile = RenderTile(0, 0, W, H, 0)
    for sample in range(2):      # two calls in a row share (and reuse) the scratch
        tile.sample_index = sample
        assert ref.render_tile(tile, 0), ref.status().last_error
        ct = native.Tile(tile.x, tile.y, tile.width, tile.height, sample, 0, 0)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc = lib.vkptc_render_tile_noalloc(na._ctx, ctypes.byref(ct), 0, film_sum.data_ptr(), film_cnt.data_ptr(),
                                           stream)
        assert rc == native.OK, na._err()
        torch.cuda.synchronize()
        # The call allocated nothing: the device's free memory is unchanged.
        assert torch.cuda.mem_get_info()[0] == free_before
        want_sum, want_cnt, _ = ref.film()
        got_sum = film_sum[..., :3].cpu().numpy()
        got_cnt = film_cnt.cpu().numpy().astype(np.uint32)
        # Same kernels, same sample: the films agree bit for bit (the tile tests' tolerance).
        assert np.array_equal(got_cnt, want_cnt)
        assert np.array_equal(bits(got_sum), bits(want_sum))
    ref.close()
    na.close()


def test_noalloc_on_a_caller_stream_is_ordered_before_a_later_rebuild():
    """The call's kernels wait on a caller stream held back by a GPU sleep;
    the host meanwhile loads another scene (same array sizes, so nothing is
    freed) into the context and rebuilds it on the context's stream.  The
    film must still be the first scene's: the context's stream waits for the
    call's kernels before it rewrites the scene and BVH arrays they read."""
    import torch
    first, second = scenes.cornell_box(seed=1), scenes.cornell_box(seed=2)
    assert first.triangle_count == second.triangle_count
    st = scenes.cornell_settings(64, 48, 1)
    W, H = st.width, st.height
    ref = _ready(first, st)
    assert ref.render_tile(RenderTile(0, 0, W, H, 0), 0), ref.status().last_error
    want_sum, want_cnt, _ = ref.film()
    ref.close()
    na = _ready(first, st)
    lib = native.load()
    film_sum = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
    film_cnt = torch.zeros((H, W), dtype=torch.int32, device="cuda")
    caller = torch.cuda.Stream()
    torch.cuda.synchronize()
    with torch.cuda.stream(caller):
        torch.cuda._sleep(200_000_000)       # ~0.1 s of GPU time ahead of the call's kernels
    ct = native.Tile(0, 0, W, H, 0, 0, 0)
    rc = lib.vkptc_render_tile_noalloc(na._ctx, ctypes.byref(ct), 0, film_sum.data_ptr(), film_cnt.data_ptr(),
                                       caller.cuda_stream)
    assert rc == native.OK, na._err()
    assert na.load_scene_snapshot(second) and na.build_or_update_acceleration()
    torch.cuda.synchronize()
    na.synchronize()
    assert np.array_equal(film_cnt.cpu().numpy().astype(np.uint32), want_cnt)
    assert np.array_equal(bits(film_sum[..., :3].cpu().numpy()), bits(want_sum))
    na.close()


def _deep_chain_scene(lo: int = -8, hi: int = 125) -> scenes.Scene:
    """Three chains of small triangles at distances 2^lo .. 2^(hi-1) along x, y
    and z: every midpoint split peels one triangle off the axis with the widest
    centroid extent, so the reference builder's tree is ~200 levels deep and
    its worst-case traversal stack is ~200 entries (~1.6 KB per thread)."""
    e = np.float32(2.0) ** np.arange(lo, hi, dtype=np.float32)
    tris = []
    for axis in range(3):
        a1, a2 = (axis + 1) % 3, (axis + 2) % 3
        for x in e:
            t = np.zeros((3, 3), np.float32)
            t[:, axis] = x
            t[1, a1] = 1.0
            t[2, a2] = 1.0
            tris.append(t)
    n = len(tris)
    mat = np.zeros((1, 16), np.float32)
    mat[0, :3] = 0.5
    mat[0, scenes.M_ROUGHNESS] = 1.0
    light = np.zeros((1, 16), np.float32)
    light[0, scenes.L_POS:scenes.L_POS + 3] = (0.5, 3.0, 0.5)
    light[0, scenes.L_COLOR:scenes.L_COLOR + 3] = 1.0
    light[0, scenes.L_INTENSITY] = 1.0
    cam = scenes.Camera(position=(4.0, 3.0, 5.0), target=(0.0, 0.0, 0.0), fov_deg=40.0)
    return scenes.Scene(np.concatenate(tris), np.arange(3 * n, dtype=np.uint32).reshape(n, 3),
                        np.array([[0, n, 0]], np.uint32), mat, light, camera=cam, name="deep_chain")


def test_noalloc_refuses_a_bvh_whose_stack_does_not_fit_in_shared_memory():
    import torch
    sc = _deep_chain_scene()
    st = scenes.RenderSettings(width=32, height=32, spp=1, max_depth=4, seed=5)
    block = 256
    t = CudaPathTracer(block_size=block)
    assert t.configure(st) and t.load_scene_snapshot(sc) and t.build_or_update_acceleration()
    assert t.reset_accumulation()
    need = t.accel_info()["stack_required"] * 8 * block
    optin = torch.cuda.get_device_properties(0).shared_memory_per_block_optin
    assert need > optin, (need, optin)     # the scene is deep enough for this check
    film_sum = torch.zeros((32, 32, 4), dtype=torch.float32, device="cuda")
    film_cnt = torch.zeros((32, 32), dtype=torch.int32, device="cuda")
    ct = native.Tile(0, 0, 32, 32, 0, 0, 0)
    lib = native.load()
    rc = lib.vkptc_render_tile_noalloc(t._ctx, ctypes.byref(ct), 0, film_sum.data_ptr(), film_cnt.data_ptr(), None)
    assert rc == native.UNSUPPORTED
    assert "shared memory" in t._err()
    assert int(film_cnt.sum()) == 0
    # the allocating path spills the stack to global memory and renders the same tile
    assert t.render_tile(RenderTile(0, 0, 32, 32, 0), 0), t.status().last_error
    _, cnt, _ = t.film()
    assert int(cnt.sum()) == 32 * 32
    t.close()


def test_noalloc_rejects_tiles_above_the_limit():
    import torch
    sc = scenes.cornell_box(seed=1)
    st = scenes.cornell_settings(300, 300, 1)      # 90,000 pixels > 65,536
    na = _ready(sc, st)
    lib = native.load()
    film_sum = torch.zeros((300, 300, 4), dtype=torch.float32, device="cuda")
    film_cnt = torch.zeros((300, 300), dtype=torch.int32, device="cuda")
    ct = native.Tile(0, 0, 300, 300, 0, 0, 0)
    rc = lib.vkptc_render_tile_noalloc(na._ctx, ctypes.byref(ct), 0, film_sum.data_ptr(), film_cnt.data_ptr(), None)
    assert rc == native.INVALID_ARGUMENT
    assert "65536" in na._err()
    # a tile within the limit on the same film is accepted
    ct = native.Tile(0, 0, 256, 256, 0, 0, 0)
    assert lib.vkptc_render_tile_noalloc(na._ctx, ctypes.byref(ct), 0, film_sum.data_ptr(), film_cnt.data_ptr(),
                                         None) == native.OK
    na.synchronize()
    assert int(film_cnt[:256, :256].min()) == 1 and int(film_cnt[256:, :].max()) == 0
    na.close()
