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
        rc = lib.vkptc_render_tile_noalloc(na._ctx, ctypes.byref(ct), 0, film_sum.data_ptr(), film_cnt.data_ptr(),
                                           stream)
        assert rc == native.OK, na._err()
        torch.cuda.synchronize()
        want_sum, want_cnt, _ = ref.film()
        got_sum = film_sum[..., :3].cpu().numpy()
        got_cnt = film_cnt.cpu().numpy().astype(np.uint32)
        # Same kernels, same sample: the films agree bit for bit (the tile tests' tolerance).
        assert np.array_equal(got_cnt, want_cnt)
        assert np.array_equal(bits(got_sum), bits(want_sum))
    ref.close()
    na.close()


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
