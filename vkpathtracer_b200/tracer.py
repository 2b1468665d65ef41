"""CudaPathTracer: the reference's IPathTracer contract over libvkpt_cuda.

Method names, argument meaning and error behaviour follow
`vkpt::pathtracer::IPathTracer` (src/pathtracer/PathTracer.h:1069-1184):
configure / load_scene_snapshot / build_or_update_acceleration return a Status;
reset_accumulation / render_tile / render_tiles return bool and record
status().last_error; resolve_hdr returns the averaged film; read_counters
returns SampleCounters.  trace_rays is the batched form of
IRayAccelerator::intersect (src/pathtracer/PathTracer.h:1001-1036).
"""
from __future__ import annotations

import ctypes
import dataclasses
import threading
from typing import Iterable, Optional, Sequence

import numpy as np

from . import native
from .scenes import Camera, RenderSettings, Scene


@dataclasses.dataclass
class Status:
    code: int
    message: str = ""

    @property
    def ok(self) -> bool:
        return self.code == native.OK

    def __bool__(self) -> bool:
        return self.ok


@dataclasses.dataclass
class RenderTile:
    """Mirror of RenderTile (src/pathtracer/PathTracer.h:914-922)."""
    x: int = 0
    y: int = 0
    width: int = 0
    height: int = 0
    sample_index: int = 0
    tile_id: int = 0
    gpu_id: int = 0


@dataclasses.dataclass
class PathTracerStatus:
    backend: str
    lifecycle: str
    scene_loaded: bool
    accel_valid: bool
    ready_to_render: bool
    current_sample: int
    last_sample_us: int
    total_samples: int
    accumulation_gen: int
    last_error: str


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def settings_c(settings: RenderSettings) -> "native.RenderSettingsC":
    s = native.RenderSettingsC()
    s.width, s.height, s.spp, s.max_depth = settings.width, settings.height, settings.spp, settings.max_depth
    s.seed = settings.seed
    s.enable_nee, s.enable_mis = int(settings.enable_nee), int(settings.enable_mis)
    s.deterministic = int(settings.deterministic)
    s.rr_start_depth = settings.russian_roulette_start_depth
    s.rr_min_survival = settings.russian_roulette_min_survival
    s.rr_max_survival = settings.russian_roulette_max_survival
    s.camera_aperture_radius = settings.camera_aperture_radius
    s.camera_focus_distance = settings.camera_focus_distance
    s.firefly_clamp = settings.firefly_clamp
    return s


def set_lens(v, camera) -> None:
    """The camera's lens shape into a vkptc_scene_view (camera_lens_set = 1)."""
    v.camera_lens_set = 1
    v.camera_iris_blade_count = int(camera.iris_blade_count)
    v.camera_iris_rotation_degrees = float(camera.iris_rotation_degrees)
    v.camera_iris_roundness = float(camera.iris_roundness)
    v.camera_anamorphic_squeeze = float(camera.anamorphic_squeeze)


def scene_view(scene: Scene):
    """POD view of a Scene; returns (view, arrays to keep alive during the call)."""
    v = native.SceneView()
    keep = (np.ascontiguousarray(scene.vertices, np.float32), np.ascontiguousarray(scene.indices, np.uint32),
            np.ascontiguousarray(scene.instances, np.uint32), np.ascontiguousarray(scene.materials, np.float32),
            np.ascontiguousarray(scene.lights, np.float32))
    v.vertices, v.vertex_count = _ptr(keep[0]), keep[0].shape[0]
    v.indices, v.index_count = _ptr(keep[1]), keep[1].size
    v.instances, v.instance_count = _ptr(keep[2]), keep[2].shape[0]
    v.materials, v.material_count = _ptr(keep[3]), keep[3].shape[0]
    v.lights, v.light_count = (_ptr(keep[4]) if keep[4].size else None), keep[4].shape[0]
    v.environment[:] = scene.environment
    c = scene.camera
    v.camera_position[:] = c.position
    v.camera_target[:] = c.target
    v.camera_up[:] = c.up
    v.camera_fov_deg = c.fov_deg
    v.camera_aperture_radius = c.aperture_radius
    v.camera_focus_distance = c.focus_distance
    set_lens(v, c)
    if scene.env_map is not None:
        env = np.ascontiguousarray(scene.env_map, np.float32)
        keep = keep + (env,)
        v.environment_map = _ptr(env)
        v.environment_map_height, v.environment_map_width = env.shape[0], env.shape[1]
        v.environment_map_scale[:] = scene.env_scale
    if scene.sdf is not None and len(scene.sdf):
        sdf = np.ascontiguousarray(scene.sdf, np.float32).reshape(-1, 16)
        keep = keep + (sdf,)
        v.sdf_primitives, v.sdf_count = _ptr(sdf), sdf.shape[0]
    if scene.instance_local is not None:
        il = np.ascontiguousarray(scene.instance_local, np.uint32).reshape(-1, 5)
        it = np.ascontiguousarray(scene.instance_transforms, np.float32).reshape(-1, 10)
        lv = np.ascontiguousarray(scene.local_vertices, np.float32).reshape(-1, 3)
        li = np.ascontiguousarray(scene.local_indices, np.uint32).reshape(-1)
        keep = keep + (il, it, lv, li)
        v.instance_local, v.instance_transforms = _ptr(il), _ptr(it)
        v.local_vertices, v.local_vertex_count = (_ptr(lv) if lv.size else None), lv.shape[0]
        v.local_indices, v.local_index_count = (_ptr(li) if li.size else None), li.size
    return v, keep


class CudaPathTracer:
    """One GPU render context.  Not re-entrant: drive it from one thread."""

    backend_name = "cuda-wavefront"

    def __init__(self, device: int = 0, block_size: int = 0, stack_depth: int = 0, math_mode: int = 0,
                 collect_stats: bool = False, wave_paths: int = 0, stage_timing: bool = False,
                 steps: int = 0, bvh: str = "reference", build: str = "device", triangle_test: str = "mt"):
        """triangle_test: "mt" (the reference's Moller-Trumbore, hit ids bit-exact
        against it) or "watertight" (Woop, Benthin and Wald; device build only)."""
        self._lib = native.load()
        cfg = native.Config()
        cfg.device = device
        cfg.block_size = block_size
        cfg.stack_depth = stack_depth
        cfg.math_mode = math_mode
        cfg.collect_stats = int(collect_stats)
        cfg.wave_paths = wave_paths
        cfg.stage_timing = int(stage_timing)
        cfg.steps = steps
        cfg.bvh_mode = native.BVH_SAH if bvh == "sah" else native.BVH_REFERENCE
        cfg.build_mode = native.BUILD_HOST if build == "host" else native.BUILD_DEVICE
        cfg.triangle_test = {"mt": native.TRIANGLE_MT, "watertight": native.TRIANGLE_WATERTIGHT}[triangle_test]
        handle = ctypes.c_void_p()
        rc = self._lib.vkptc_create(ctypes.byref(cfg), ctypes.byref(handle))
        if rc != native.OK:
            raise native.VkptcError(rc, "vkptc_create failed (no CUDA device?)")
        self._ctx = handle
        self._settings: Optional[RenderSettings] = None
        self._keep = None
        self._material_count = 0

    # ------------------------------------------------------------ plumbing
    def _err(self) -> str:
        return self._lib.vkptc_last_error(self._ctx).decode()

    def _status(self, rc: int) -> Status:
        return Status(rc, "" if rc == native.OK else self._err())

    def _check(self, rc: int):
        if rc != native.OK:
            raise native.VkptcError(rc, self._err())

    def close(self):
        if getattr(self, "_ctx", None):
            self._lib.vkptc_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------ lifecycle
    def configure(self, settings: RenderSettings) -> Status:
        s = settings_c(settings)
        st = self._status(self._lib.vkptc_configure(self._ctx, ctypes.byref(s)))
        if st.ok:
            self._settings = settings
        return st

    def load_scene_snapshot(self, scene: Scene) -> Status:
        v, keep = scene_view(scene)
        st = self._status(self._lib.vkptc_load_scene(self._ctx, ctypes.byref(v)))
        if st.ok:
            self._material_count = max(1, int(np.asarray(scene.materials).reshape(-1, 16).shape[0]))
        return st

    def build_or_update_acceleration(self) -> Status:
        return self._status(self._lib.vkptc_build_acceleration(self._ctx))

    def load_bvh(self, nodes: np.ndarray, prim_indices: np.ndarray) -> Status:
        """Adopts an externally built binary BVH (ParallelBvhBuilder layout, 10 words per node)."""
        nodes = np.ascontiguousarray(nodes, np.uint32).reshape(-1, 10)
        prim = np.ascontiguousarray(prim_indices, np.uint32)
        b = native.BvhView(_ptr(nodes), nodes.shape[0], _ptr(prim), prim.size)
        return self._status(self._lib.vkptc_load_bvh(self._ctx, ctypes.byref(b)))

    def read_bandwidth(self, nbytes: int, reps: int) -> float:
        """GB/s of 16-byte reads (cached in L2 only) streaming `reps` times over a
        device buffer of `nbytes`: L2 bandwidth for a buffer well under the L2
        size, HBM read bandwidth for one far above it."""
        g = ctypes.c_double(0.0)
        self._check(self._lib.vkptc_measure_read_bandwidth(self._ctx, nbytes, reps, ctypes.byref(g)))
        return float(g.value)

    def accel_info(self) -> dict:
        a = native.AccelInfo()
        self._check(self._lib.vkptc_get_accel_info(self._ctx, ctypes.byref(a)))
        return a.as_dict()

    def update_instance_transforms(self, updates, check_only: bool = False):
        """Instance transform updates ({"instance", "translation", "rotation",
        "scale", "flags"}), refitted on the device (apply_instance_transform_update)."""
        arr = (native.InstanceUpdate * max(1, len(updates)))()
        for k, u in enumerate(updates):
            arr[k].instance_index = u["instance"]
            arr[k].flags = u.get("flags", 0)
            arr[k].translation[:] = u.get("translation", (0.0, 0.0, 0.0))
            arr[k].rotation[:] = u.get("rotation", (0.0, 0.0, 0.0, 1.0))
            arr[k].scale[:] = u.get("scale", (1.0, 1.0, 1.0))
        fn = self._lib.vkptc_check_instance_transforms if check_only else self._lib.vkptc_update_instance_transforms
        self._check(fn(self._ctx, ctypes.cast(arr, ctypes.c_void_p), len(updates)))

    def get_camera(self) -> Camera:
        """The loaded scene's camera (ExtractCameraState)."""
        c = native.CameraC()
        self._check(self._lib.vkptc_get_camera(self._ctx, ctypes.byref(c)))
        return Camera(tuple(c.position), tuple(c.target), tuple(c.up), c.fov_deg, c.aperture_radius, c.focus_distance,
                      c.iris_blade_count, c.iris_rotation_degrees, c.iris_roundness, c.anamorphic_squeeze)

    def update_camera_state(self, camera: Camera) -> None:
        """IPathTracer::update_camera_state: the whole camera replaced; no
        rebuild, the film is kept (reset_accumulation clears it)."""
        c = native.CameraC()
        c.position[:], c.target[:], c.up[:] = camera.position, camera.target, camera.up
        c.fov_deg, c.aperture_radius, c.focus_distance = camera.fov_deg, camera.aperture_radius, camera.focus_distance
        c.iris_blade_count, c.iris_rotation_degrees = int(camera.iris_blade_count), camera.iris_rotation_degrees
        c.iris_roundness, c.anamorphic_squeeze = camera.iris_roundness, camera.anamorphic_squeeze
        self._check(self._lib.vkptc_update_camera(self._ctx, ctypes.byref(c)))

    def update_camera(self, position, target, up, fov_deg: float) -> None:
        """IPathTracer::update_camera: position, target, up and field of view
        changed, the rest of the camera kept."""
        cam = self.get_camera()
        cam.position, cam.target, cam.up, cam.fov_deg = tuple(position), tuple(target), tuple(up), float(fov_deg)
        self.update_camera_state(cam)

    def update_scene_delta(self, materials=None, lights=None, instance_materials=None, environment=None) -> None:
        """IPathTracer::update_scene_delta (ApplySceneDeltaUpdate): materials and
        lights as {index: 16-float record}, instance_materials as
        {instance index: material index} (or sequences of (index, value) pairs,
        applied in order), environment an rgb colour or None."""
        def pairs(x):
            return list(x.items()) if isinstance(x, dict) else list(x or ())

        materials, lights, inst = pairs(materials), pairs(lights), pairs(instance_materials)
        mi = np.array([k for k, _ in materials], np.uint32)
        mw = np.ascontiguousarray(np.array([v for _, v in materials], np.float32).reshape(-1, 16))
        li = np.array([k for k, _ in lights], np.uint32)
        lw = np.ascontiguousarray(np.array([v for _, v in lights], np.float32).reshape(-1, 16))
        ii = np.array([k for k, _ in inst], np.uint32)
        im = np.array([v for _, v in inst], np.uint32)
        d = native.SceneDelta()
        d.material_indices, d.materials, d.material_count = _ptr(mi), _ptr(mw), mi.size
        d.light_indices, d.lights, d.light_count = _ptr(li), _ptr(lw), li.size
        d.instance_indices, d.instance_material_indices, d.instance_material_count = _ptr(ii), _ptr(im), ii.size
        if environment is not None:
            d.environment_changed = 1
            d.environment[:] = environment
        self._check(self._lib.vkptc_update_scene_delta(self._ctx, ctypes.byref(d)))

    @staticmethod
    def film_resolve(exposure: float = 1.0, white_balance_kelvin: float = 6500.0, tone_map: str = "linear",
                     output_transform: str = "gamma", gamma: float = 2.2, clamp_output: bool = True):
        """FilmResolveSettings (the reference's defaults)."""
        r = native.FilmResolve()
        r.exposure, r.white_balance_kelvin = exposure, white_balance_kelvin
        r.tone_map, r.output_transform = native.TONE_MAPS[tone_map], native.OUTPUT_TRANSFORMS[output_transform]
        r.gamma, r.clamp_output = gamma, int(clamp_output)
        return r

    def resolve_ldr(self, **settings) -> np.ndarray:
        """ApplyFilmResolve(resolve_hdr()) on the device: (H, W, 4) uint8."""
        st = self._settings
        out = np.zeros((st.height, st.width, 4), np.uint8)
        rs = self.film_resolve(**settings)
        self._check(self._lib.vkptc_resolve_ldr(self._ctx, ctypes.byref(rs), out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def request_film_readback(self, **settings) -> int:
        tok = ctypes.c_uint64(0)
        rs = self.film_resolve(**settings)
        self._check(self._lib.vkptc_request_ldr_readback(self._ctx, ctypes.byref(rs), ctypes.byref(tok)))
        return int(tok.value)

    def poll_film(self, token: int):
        """(state, image or None); state is native.READBACK_*; never blocks."""
        st = self._settings
        out = np.zeros((st.height, st.width, 4), np.uint8)
        state = ctypes.c_uint32(0)
        self._lib.vkptc_poll_ldr_readback(self._ctx, token, out.ctypes.data_as(ctypes.c_void_p), ctypes.byref(state))
        return int(state.value), (out if state.value == native.READBACK_READY else None)

    def read_accel(self, what: int) -> np.ndarray:
        """One device array of the accelerator (native.ACCEL_*) as raw uint32 words."""
        n = ctypes.c_uint64(0)
        self._check(self._lib.vkptc_read_accel(self._ctx, what, None, 0, ctypes.byref(n)))
        out = np.zeros(n.value // 4, np.uint32)
        if n.value:
            self._check(self._lib.vkptc_read_accel(self._ctx, what, out.ctypes.data_as(ctypes.c_void_p), n.value,
                                                   ctypes.byref(n)))
        return out

    def reset_accumulation(self) -> bool:
        return self._lib.vkptc_reset(self._ctx) == native.OK

    def shutdown(self):
        self._lib.vkptc_shutdown(self._ctx)
        self._settings = None

    # ------------------------------------------------------------ rendering
    def supports_tile_rendering(self) -> bool:
        return True

    def supports_tile_batching(self) -> bool:
        return True

    def render_tile(self, tile: RenderTile, frame_index: int = 0) -> bool:
        return self.render_tiles([tile], frame_index)

    def render_tile_cancellable(self, tile: RenderTile, frame_index: int, stop: Optional[threading.Event]) -> bool:
        return self.render_tiles([tile], frame_index, stop)

    def render_tiles(self, tiles: Sequence[RenderTile], frame_index: int = 0,
                     stop: Optional[threading.Event] = None) -> bool:
        if stop is not None and stop.is_set():
            return False
        arr = (native.Tile * max(1, len(tiles)))()
        for i, t in enumerate(tiles):
            arr[i] = native.Tile(t.x, t.y, t.width, t.height, t.sample_index, t.tile_id, t.gpu_id)
        flag = ctypes.c_int32(0)
        rc = self._lib.vkptc_render(self._ctx, arr, len(tiles), frame_index, ctypes.byref(flag))
        return rc == native.OK

    def render_frame(self, first_sample: int, sample_count: int, frame_index: int = 0, sync: bool = True):
        """Renders full-frame samples [first, first+count) (batched render_tile calls)."""
        self._check(self._lib.vkptc_render_frame(self._ctx, first_sample, sample_count, frame_index))
        if sync:
            self.synchronize()

    def synchronize(self):
        self._check(self._lib.vkptc_synchronize(self._ctx))

    def set_stream(self, stream_handle: int):
        """Enqueue all further work on this cudaStream_t (0 = the context's own stream)."""
        self._check(self._lib.vkptc_set_stream(self._ctx, stream_handle or None))

    STAGES = ("raygen", "extend", "shade", "shadow", "accumulate")

    def read_stage_times(self) -> dict:
        """{stage: (ms, launches)} since the last read (needs stage_timing=True)."""
        ms = (ctypes.c_double * 5)()
        n = (ctypes.c_uint64 * 5)()
        self._check(self._lib.vkptc_read_stage_times(self._ctx, ms, n))
        return {k: (ms[i], int(n[i])) for i, k in enumerate(self.STAGES)}

    # ------------------------------------------------------------ film
    def film(self):
        """Raw film: (sum (H,W,3) float32, count (H,W) uint32, invalid (H,W) float32)."""
        st = self._settings
        W, H = st.width, st.height
        s = np.zeros((H, W, 3), np.float32)
        c = np.zeros((H, W), np.uint32)
        inv = np.zeros((H, W), np.float32)
        self._check(self._lib.vkptc_read_film(self._ctx, _ptr(s), _ptr(c), _ptr(inv)))
        return s, c, inv

    def resolve_hdr(self) -> np.ndarray:
        st = self._settings
        out = np.zeros((st.height, st.width, 3), np.float32)
        self._check(self._lib.vkptc_resolve_hdr(self._ctx, _ptr(out)))
        return out

    def replace_film_history(self, film_sum: np.ndarray, count: np.ndarray, invalid: Optional[np.ndarray] = None) -> bool:
        s = np.ascontiguousarray(film_sum, np.float32)
        c = np.ascontiguousarray(count, np.uint32)
        i = None if invalid is None else np.ascontiguousarray(invalid, np.float32)
        return self._lib.vkptc_write_film(self._ctx, _ptr(s), _ptr(c), _ptr(i)) == native.OK

    def read_counters(self) -> dict:
        c = native.Counters()
        self._check(self._lib.vkptc_read_counters(self._ctx, ctypes.byref(c)))
        return c.as_dict()

    def traversal_stats(self) -> dict:
        """Wide-BVH work split by query kind (needs collect_stats=True)."""
        a = (ctypes.c_uint64 * 8)()
        self._check(self._lib.vkptc_read_traversal_stats(self._ctx, a))
        keys = ("rays", "nodes", "leaves", "tris", "shadow_rays", "shadow_nodes", "shadow_leaves", "shadow_tris")
        return {k: int(a[i]) for i, k in enumerate(keys)}

    def extension_counters(self) -> dict:
        s = self.traversal_stats()
        return {"rays": s["rays"], "nodes": s["nodes"], "tris": s["tris"], "leaves": s["leaves"]}

    def status(self) -> PathTracerStatus:
        s = native.TracerStatusC()
        self._lib.vkptc_get_status(self._ctx, ctypes.byref(s))
        return PathTracerStatus("cuda-wavefront", native.LIFECYCLE_NAMES[s.lifecycle], bool(s.scene_loaded),
                                bool(s.accel_valid), bool(s.ready_to_render), int(s.current_sample),
                                int(s.last_sample_us), int(s.total_samples), int(s.accumulation_gen), self._err())

    # ------------------------------------------------------------ ray queries
    def trace_rays(self, rays: np.ndarray, mode: int = native.QUERY_CLOSEST, tmax: Optional[np.ndarray] = None):
        """rays (N,6) float32 on the host -> (prim uint32, t float32)."""
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        n = rays.shape[0]
        prim = np.zeros(n, np.uint32)
        t = np.zeros(n, np.float32)
        tm = None if tmax is None else np.ascontiguousarray(tmax, np.float32)
        self._check(self._lib.vkptc_trace_rays(self._ctx, _ptr(rays), _ptr(tm), n, mode, _ptr(prim), _ptr(t)))
        return prim, t

    def trace_rays_device(self, d_rays: int, d_tmax: int, n: int, mode: int, d_prim: int, d_t: int, stream: int = 0):
        """Device-pointer variant (e.g. torch tensors' data_ptr()); enqueued, not synchronised."""
        self._check(self._lib.vkptc_trace_rays_device(self._ctx, d_rays, d_tmax or None, n, mode, d_prim,
                                                      d_t or None, stream or None))


    # ------------------------------------------------ differentiable rendering
    def adjoint_setup(self, spp: int, target: Optional[np.ndarray] = None, frame: int = 0, first_sample: int = 0,
                      decorrelated: bool = False, backward_frame: int = 0):
        """Prepares vkptc_forward / vkptc_backward: spp samples per pixel, MSE
        loss against target (H, W, 3) float32, or no target.  decorrelated:
        the backward replays the paths of backward_frame instead of the
        forward's (an unbiased gradient of the expected image's loss)."""
        d = native.AdjointDesc()
        d.spp, d.first_sample, d.frame = spp, first_sample, frame
        d.backward_frame = backward_frame
        d.flags = native.ADJ_DECORRELATED if decorrelated else 0
        tg = None if target is None else np.ascontiguousarray(target, np.float32).reshape(-1)
        self._check(self._lib.vkptc_adjoint_setup(self._ctx, ctypes.byref(d), _ptr(tg), 0 if tg is None else tg.size))
        self._adj_spp = spp

    def forward(self, params: np.ndarray, rr_params: Optional[np.ndarray] = None, image: bool = False):
        """params: (materials, 7) albedo rgb, roughness, emission rgb.  Returns
        the loss (FP64), and the (H, W, 3) image when image=True."""
        p = np.ascontiguousarray(params, np.float32).reshape(-1)
        rp = None if rr_params is None else np.ascontiguousarray(rr_params, np.float32).reshape(-1)
        if rp is not None and rp.size != p.size:
            raise ValueError("rr_params must have the shape of params")
        loss = ctypes.c_double(0.0)
        img = np.zeros((self._settings.height, self._settings.width, 3), np.float32) if image else None
        self._check(self._lib.vkptc_forward(self._ctx, _ptr(p), p.size, _ptr(rp), ctypes.byref(loss), _ptr(img)))
        return (loss.value, img) if image else loss.value

    def backward(self, path_weight: Optional[np.ndarray] = None) -> np.ndarray:
        """dL/dparams of the last forward, shape (materials, 7).  path_weight
        (optional, one float per path) scales each path's contribution."""
        n = self._material_count * native.ADJ_PARAMS_PER_MATERIAL
        g = np.zeros(n, np.float32)
        if path_weight is None:
            self._check(self._lib.vkptc_backward(self._ctx, _ptr(g), n))
        else:
            pw = np.ascontiguousarray(path_weight, np.float32).reshape(-1)
            if pw.size != self._settings.width * self._settings.height * self._adj_spp:
                raise ValueError("path_weight must hold one float per path")
            self._check(self._lib.vkptc_backward_weighted(self._ctx, _ptr(pw), _ptr(g), n))
        return g.reshape(-1, native.ADJ_PARAMS_PER_MATERIAL)

    def adjoint_frames(self, frame: int, backward_frame: int = 0):
        """New RNG frames for the next forward (and a decorrelated backward)."""
        self._check(self._lib.vkptc_adjoint_set_frames(self._ctx, frame, backward_frame))

    def adjoint_samples(self):
        """(rgb (spp, H, W, 3), signature (spp, H, W) uint32) of the last forward."""
        W, H, n = self._settings.width, self._settings.height, self._adj_spp
        rgb = np.zeros((n, H, W, 3), np.float32)
        sig = np.zeros((n, H, W), np.uint32)
        self._check(self._lib.vkptc_adjoint_read_samples(self._ctx, _ptr(rgb), _ptr(sig)))
        return rgb, sig

    def adjoint_stats(self) -> dict:
        st = native.AdjointStats()
        self._check(self._lib.vkptc_adjoint_get_stats(self._ctx, ctypes.byref(st)))
        return st.as_dict()


def material_params(materials: np.ndarray) -> np.ndarray:
    """The 7 differentiable parameters of each material row (16 floats):
    albedo rgb, roughness, emission rgb."""
    m = np.asarray(materials, np.float32).reshape(-1, 16)
    return np.ascontiguousarray(np.concatenate([m[:, 0:3], m[:, 6:7], m[:, 3:6]], axis=1))


class BatchRenderer:
    """Many render jobs (scene + settings each) rendered together.

    run("plain") renders every job one frame (sample) per launch sequence;
    run("persistent") renders all of them in one persistent launch fed by a
    device work queue, replayed from a CUDA graph.  Films are bit-identical.
    """

    def __init__(self, device: int = 0, math_mode: int = 0, collect_stats: bool = False, bvh: str = "reference",
                 stage_timing: bool = False, build: str = "device", triangle_test: str = "mt"):
        """triangle_test "watertight": every job traverses with the watertight
        test, in every driver."""
        self._lib = native.load()
        cfg = native.Config()
        cfg.device = device
        cfg.math_mode = math_mode
        cfg.collect_stats = int(collect_stats)
        cfg.stage_timing = int(stage_timing)
        cfg.bvh_mode = native.BVH_SAH if bvh == "sah" else native.BVH_REFERENCE
        cfg.build_mode = native.BUILD_HOST if build == "host" else native.BUILD_DEVICE
        cfg.triangle_test = {"mt": native.TRIANGLE_MT, "watertight": native.TRIANGLE_WATERTIGHT}[triangle_test]
        h = ctypes.c_void_p()
        rc = self._lib.vkptc_batch_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc != native.OK:
            raise native.VkptcError(rc, "vkptc_batch_create failed")
        self._b = h
        self.settings = []

    def _err(self):
        return self._lib.vkptc_batch_last_error(self._b).decode()

    def close(self):
        if getattr(self, "_b", None):
            self._lib.vkptc_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add_job(self, scene: Scene, settings: RenderSettings) -> int:
        v, keep = scene_view(scene)
        s = settings_c(settings)
        jid = ctypes.c_uint32()
        rc = self._lib.vkptc_batch_add_job(self._b, ctypes.byref(v), ctypes.byref(s), ctypes.byref(jid))
        if rc != native.OK:
            raise native.VkptcError(rc, self._err())
        self.settings.append(settings)
        return int(jid.value)

    def run(self, mode: str = "persistent", pool_paths: int = 0, block_size: int = 0, stack_depth: int = 0,
            steps: int = 0, sample_limit: int = 0, use_graph: bool = True, occupancy: int = 0,
            barrier_spins: int = 0) -> dict:
        t = native.BatchTuning(pool_paths, block_size, stack_depth, steps, sample_limit, int(use_graph), occupancy,
                               barrier_spins)
        modes = {"plain": native.BATCH_PLAIN, "persistent": native.BATCH_PERSISTENT, "loop": native.BATCH_LOOP}
        if mode not in modes:
            raise ValueError(f"mode must be one of {sorted(modes)}")
        m = modes[mode]
        rc = self._lib.vkptc_batch_run(self._b, m, ctypes.byref(t))
        if rc != native.OK:
            raise native.VkptcError(rc, self._err())
        st = native.BatchStats()
        self._lib.vkptc_batch_get_stats(self._b, ctypes.byref(st))
        return st.as_dict()

    def read_films(self, sums, counts=None):
        """Every job's film into caller-owned arrays (sums[j]: (H, W, 3) float32,
        counts[j]: (H, W) uint32 or None), one wait for all copies."""
        n = len(self.settings)
        ps = (ctypes.c_void_p * max(1, n))(*[s.ctypes.data if s is not None else None for s in sums])
        pc = None
        if counts is not None:
            pc = (ctypes.c_void_p * max(1, n))(*[c.ctypes.data if c is not None else None for c in counts])
        rc = self._lib.vkptc_batch_read_films(self._b, ps, pc)
        if rc != native.OK:
            raise native.VkptcError(rc, self._err())

    def film(self, job: int):
        st = self.settings[job]
        s = np.zeros((st.height, st.width, 3), np.float32)
        c = np.zeros((st.height, st.width), np.uint32)
        rc = self._lib.vkptc_batch_read_film(self._b, job, _ptr(s), _ptr(c))
        if rc != native.OK:
            raise native.VkptcError(rc, self._err())
        return s, c
