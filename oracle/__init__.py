"""CPU oracle for the render hot path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / --impl
reference legs may import this package, and only as the checker or the CPU
baseline.  The product package (vkpathtracer_b200) never imports it.

The FP64 adjoint (oracle/adjoint.cpp -> oracle/_build/libvkptadj.so,
oracle/vkpt_adjoint.h) is the checker of the GPU forward/backward pair;
load_adjoint() returns it.

Two interchangeable implementations of oracle/vkpt_oracle.h:
  "reference"  oracle/_ref/libvkptref.so   -- the reference's own CPU tracer,
               compiled from its unmodified sources by oracle/Makefile.
  "port"       oracle/_build/libvkptport.so -- restatement (oracle/port.cpp),
               pinned bit-for-bit to "reference" by tests/test_oracle_pin.py.
"""
from __future__ import annotations

import contextlib
import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libvkptref.so")
# The reference's AVX2 build (timing only: its leaf size and arithmetic differ from the parity build).
REF_AVX2_LIB = os.path.join(HERE, "_ref_avx2", "libvkptref.so")
PORT_LIB = os.path.join(HERE, "_build", "libvkptport.so")
ADJ_LIB = os.path.join(HERE, "_build", "libvkptadj.so")
# The reference checkout (read-only); VKPT_REFERENCE_DIR overrides the default location.
REFERENCE_DIR = os.environ.get("VKPT_REFERENCE_DIR", "/root/reference")
REFERENCE_SRC = os.path.join(REFERENCE_DIR, "src")


class VkoScene(ctypes.Structure):
    _fields_ = [
        ("vertices", ctypes.c_void_p), ("vertex_count", ctypes.c_uint32),
        ("indices", ctypes.c_void_p), ("index_count", ctypes.c_uint32),
        ("instances", ctypes.c_void_p), ("instance_count", ctypes.c_uint32),
        ("materials", ctypes.c_void_p), ("material_count", ctypes.c_uint32),
        ("lights", ctypes.c_void_p), ("light_count", ctypes.c_uint32),
        ("environment", ctypes.c_float * 3),
        ("camera_position", ctypes.c_float * 3),
        ("camera_target", ctypes.c_float * 3),
        ("camera_up", ctypes.c_float * 3),
        ("camera_fov_deg", ctypes.c_float),
        ("camera_aperture_radius", ctypes.c_float),
        ("camera_focus_distance", ctypes.c_float),
        ("environment_map", ctypes.c_void_p),
        ("environment_map_width", ctypes.c_uint32),
        ("environment_map_height", ctypes.c_uint32),
        ("environment_map_scale", ctypes.c_float * 3),
        ("sdf_primitives", ctypes.c_void_p),
        ("sdf_count", ctypes.c_uint32),
        ("instance_local", ctypes.c_void_p),
        ("instance_transforms", ctypes.c_void_p),
        ("local_vertices", ctypes.c_void_p),
        ("local_vertex_count", ctypes.c_uint32),
        ("local_indices", ctypes.c_void_p),
        ("local_index_count", ctypes.c_uint32),
        ("camera_lens_set", ctypes.c_uint32),
        ("camera_iris_blade_count", ctypes.c_uint32),
        ("camera_iris_rotation_degrees", ctypes.c_float),
        ("camera_iris_roundness", ctypes.c_float),
        ("camera_anamorphic_squeeze", ctypes.c_float),
    ]


class VkoSettings(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("max_depth", ctypes.c_uint32),
        ("enable_nee", ctypes.c_uint32), ("enable_mis", ctypes.c_uint32), ("rr_start", ctypes.c_uint32),
        ("rr_min", ctypes.c_float), ("rr_max", ctypes.c_float), ("seed", ctypes.c_uint64),
        ("firefly_clamp", ctypes.c_float), ("_pad", ctypes.c_uint32),
    ]


class VkoCounters(ctypes.Structure):
    _fields_ = [
        ("samples", ctypes.c_uint64), ("rays", ctypes.c_uint64), ("triangle_tests", ctypes.c_uint64),
        ("triangle_hits", ctypes.c_uint64), ("bvh_node_visits", ctypes.c_uint64),
        ("bvh_leaf_visits", ctypes.c_uint64), ("shadow_tests", ctypes.c_uint64),
        ("render_ms", ctypes.c_double),
        ("sdf_tests", ctypes.c_uint64), ("sdf_steps", ctypes.c_uint64), ("sdf_hits", ctypes.c_uint64),
        ("sdf_misses", ctypes.c_uint64),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class VkoJob(ctypes.Structure):
    _fields_ = [("scene", ctypes.POINTER(VkoScene)), ("settings", ctypes.POINTER(VkoSettings)),
                ("pixels", ctypes.c_void_p), ("pixel_count", ctypes.c_uint32), ("first_sample", ctypes.c_uint32),
                ("n_samples", ctypes.c_uint32), ("reserved", ctypes.c_uint32), ("film_sum", ctypes.c_void_p),
                ("film_count", ctypes.c_void_p), ("film_m2", ctypes.c_void_p), ("counters", VkoCounters)]


class VkoInstanceUpdate(ctypes.Structure):
    _fields_ = [("instance_index", ctypes.c_uint32), ("flags", ctypes.c_uint32), ("translation", ctypes.c_float * 3),
                ("rotation", ctypes.c_float * 4), ("scale", ctypes.c_float * 3)]


def instance_updates(updates, struct=VkoInstanceUpdate):
    """[{"instance", "translation", "rotation", "scale", "flags"}] -> ctypes array."""
    arr = (struct * max(1, len(updates)))()
    for k, u in enumerate(updates):
        arr[k].instance_index = u["instance"]
        arr[k].flags = u.get("flags", 0)
        arr[k].translation[:] = u.get("translation", (0.0, 0.0, 0.0))
        arr[k].rotation[:] = u.get("rotation", (0.0, 0.0, 0.0, 1.0))
        arr[k].scale[:] = u.get("scale", (1.0, 1.0, 1.0))
    return arr


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def build_port(quiet: bool = True) -> str:
    """Compile the restatement with g++ (no reference sources needed)."""
    os.makedirs(os.path.join(HERE, "_build"), exist_ok=True)
    src = os.path.join(HERE, "port.cpp")
    deps = [src] + [os.path.join(HERE, f) for f in ("vkpt_oracle.h", "worker_pool.h")]
    if (not os.path.exists(PORT_LIB)) or os.path.getmtime(PORT_LIB) < max(os.path.getmtime(d) for d in deps):
        cmd = ["g++", "-std=c++20", "-O2", "-fPIC", "-shared", "-o", PORT_LIB, src, "-lpthread"]
        subprocess.run(cmd, check=True, capture_output=quiet)
    return PORT_LIB


def build_ref(quiet: bool = True) -> Optional[str]:
    """Compile the reference oracle where the reference sources exist; else None."""
    if not os.path.isdir(REFERENCE_SRC):
        return REF_LIB if os.path.exists(REF_LIB) else None
    subprocess.run(["make", "-C", HERE, "ref", f"REF={REFERENCE_SRC}", "-j8"], check=True,
                   capture_output=quiet)
    subprocess.run(["make", "-C", HERE, "ref_avx2", f"REF={REFERENCE_SRC}", "-j8"], check=True,
                   capture_output=quiet)
    # The C++ IPathTracer adapter checker links the library; build it when the library exists.
    lib = os.path.join(os.path.dirname(HERE), "vkpathtracer_b200", "_lib", "libvkpt_cuda.so")
    if os.path.exists(lib):
        subprocess.run(["make", "-C", HERE, "adapter", f"REF={REFERENCE_SRC}"], check=True, capture_output=quiet)
    return REF_LIB


class Oracle:
    def __init__(self, path: str):
        self.path = path
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.vko_render.restype = ctypes.c_int
        L.vko_render.argtypes = [ctypes.POINTER(VkoScene), ctypes.POINTER(VkoSettings), ctypes.c_uint32,
                                 ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint32,
                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                 ctypes.POINTER(VkoCounters)]
        L.vko_build_bvh.restype = ctypes.c_int
        L.vko_build_bvh.argtypes = [ctypes.POINTER(VkoScene), ctypes.c_uint32, ctypes.c_int,
                                    ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32), ctypes.c_void_p]
        L.vko_intersect.restype = ctypes.c_int
        L.vko_intersect.argtypes = [ctypes.POINTER(VkoScene), ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.POINTER(ctypes.c_double)]
        L.vko_render_jobs.restype = ctypes.c_int
        L.vko_render_jobs.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32,
                                      ctypes.POINTER(ctypes.c_double)]
        L.vko_last_error.restype = ctypes.c_char_p
        L.vko_impl_name.restype = ctypes.c_char_p
        L.vko_set_triangle_test.restype = ctypes.c_int
        L.vko_set_triangle_test.argtypes = [ctypes.c_uint32]
        self.kind = L.vko_impl_name().decode()

    @contextlib.contextmanager
    def triangle_test(self, mode: str):
        """Traverse with "mt" (the reference's Moller-Trumbore) or "watertight"
        (port only) inside the block; Moller-Trumbore again afterwards."""
        self._check(self.lib.vko_set_triangle_test({"mt": 0, "watertight": 1}[mode]))
        try:
            yield self
        finally:
            self.lib.vko_set_triangle_test(0)

    # -- helpers
    @staticmethod
    def make_scene(scene):
        keep = (scene.vertices, scene.indices, scene.instances, scene.materials, scene.lights)
        s = VkoScene()
        s.vertices, s.vertex_count = _ptr(scene.vertices), scene.vertices.shape[0]
        s.indices, s.index_count = _ptr(scene.indices), scene.indices.size
        s.instances, s.instance_count = _ptr(scene.instances), scene.instances.shape[0]
        s.materials, s.material_count = _ptr(scene.materials), scene.materials.shape[0]
        s.lights, s.light_count = (_ptr(scene.lights) if scene.lights.size else None), scene.lights.shape[0]
        s.environment[:] = scene.environment
        c = scene.camera
        s.camera_position[:] = c.position
        s.camera_target[:] = c.target
        s.camera_up[:] = c.up
        s.camera_fov_deg = c.fov_deg
        s.camera_aperture_radius = c.aperture_radius
        s.camera_focus_distance = c.focus_distance
        s.camera_lens_set = 1
        s.camera_iris_blade_count = int(getattr(c, "iris_blade_count", 0))
        s.camera_iris_rotation_degrees = float(getattr(c, "iris_rotation_degrees", 0.0))
        s.camera_iris_roundness = float(getattr(c, "iris_roundness", 1.0))
        s.camera_anamorphic_squeeze = float(getattr(c, "anamorphic_squeeze", 1.0))
        env = getattr(scene, "env_map", None)
        if env is not None:
            env = np.ascontiguousarray(env, np.float32)
            keep = keep + (env,)
            s.environment_map = _ptr(env)
            s.environment_map_height, s.environment_map_width = env.shape[0], env.shape[1]
            s.environment_map_scale[:] = scene.env_scale
        sdf = getattr(scene, "sdf", None)
        if sdf is not None and len(sdf):
            sdf = np.ascontiguousarray(sdf, np.float32).reshape(-1, 16)
            keep = keep + (sdf,)
            s.sdf_primitives, s.sdf_count = _ptr(sdf), sdf.shape[0]
        if getattr(scene, "instance_local", None) is not None:
            il = np.ascontiguousarray(scene.instance_local, np.uint32).reshape(-1, 5)
            it = np.ascontiguousarray(scene.instance_transforms, np.float32).reshape(-1, 10)
            lv = np.ascontiguousarray(scene.local_vertices, np.float32).reshape(-1, 3)
            li = np.ascontiguousarray(scene.local_indices, np.uint32).reshape(-1)
            keep = keep + (il, it, lv, li)
            s.instance_local, s.instance_transforms = _ptr(il), _ptr(it)
            s.local_vertices, s.local_vertex_count = (_ptr(lv) if lv.size else None), lv.shape[0]
            s.local_indices, s.local_index_count = (_ptr(li) if li.size else None), li.size
        return s, keep

    @staticmethod
    def make_settings(st):
        s = VkoSettings()
        s.width, s.height, s.max_depth = st.width, st.height, st.max_depth
        s.enable_nee, s.enable_mis = int(st.enable_nee), int(st.enable_mis)
        s.rr_start = st.russian_roulette_start_depth
        s.rr_min, s.rr_max = st.russian_roulette_min_survival, st.russian_roulette_max_survival
        s.seed = st.seed
        s.firefly_clamp = st.firefly_clamp
        return s

    def _check(self, rc: int):
        if rc != 0:
            raise RuntimeError(f"oracle ({self.kind}) failed: {self.lib.vko_last_error().decode()}")

    # -- API
    def render(self, scene, settings, first_sample: int = 0, n_samples: Optional[int] = None,
               threads: int = 1, pixels: Optional[np.ndarray] = None, per_sample: bool = False,
               updates=None):
        """Returns dict(sum=(H,W,3), count=(H,W), invalid=(H,W), samples=(n,H,W,3)|None, counters).
        updates: instance transform updates applied after the build (one tracer, full frame)."""
        n = settings.spp if n_samples is None else n_samples
        W, H = settings.width, settings.height
        sc, keep = self.make_scene(scene)
        st = self.make_settings(settings)
        film = np.zeros((H, W, 3), np.float32)
        count = np.zeros((H, W), np.uint32)
        invalid = np.zeros((H, W), np.float32)
        samples = np.zeros((n, H, W, 3), np.float32) if per_sample else None
        px = None if pixels is None else np.ascontiguousarray(pixels, dtype=np.uint32)
        ctr = VkoCounters()
        if updates:
            ups = instance_updates(updates)
            self.lib.vko_set_instance_updates(ups, len(updates))
        try:
            rc = self.lib.vko_render(ctypes.byref(sc), ctypes.byref(st), first_sample, n, threads,
                                     _ptr(px), 0 if px is None else px.size, _ptr(film), _ptr(count),
                                     _ptr(invalid), _ptr(samples), ctypes.byref(ctr))
        finally:
            if updates:
                self.lib.vko_set_instance_updates(None, 0)
        del keep
        self._check(rc)
        return {"sum": film, "count": count, "invalid": invalid, "samples": samples,
                "counters": ctr.as_dict()}

    def render_jobs(self, jobs, threads: int = 1):
        """Many jobs on one pool of `threads` workers (vko_render_jobs).
        jobs: [(scene, settings, pixels)] with pixels a 1-D array of distinct
        y*W+x indices; every sample of each listed pixel is rendered.
        Returns ([dict(sum=(n,3), count=(n,), m2=(n,3), counters)], render_ms)."""
        recs = (VkoJob * max(1, len(jobs)))()
        keep, outs = [], []
        for k, (scene, settings, pixels) in enumerate(jobs):
            sc, kp = self.make_scene(scene)
            st = self.make_settings(settings)
            px = np.ascontiguousarray(pixels, dtype=np.uint32).reshape(-1)
            out = {"sum": np.zeros((px.size, 3), np.float32), "count": np.zeros(px.size, np.uint32),
                   "m2": np.zeros((px.size, 3), np.float32)}
            keep.append((sc, st, kp, px))
            outs.append(out)
            r = recs[k]
            r.scene, r.settings = ctypes.pointer(sc), ctypes.pointer(st)
            r.pixels, r.pixel_count = _ptr(px), px.size
            r.first_sample, r.n_samples = 0, settings.spp
            r.film_sum, r.film_count, r.film_m2 = _ptr(out["sum"]), _ptr(out["count"]), _ptr(out["m2"])
        ms = ctypes.c_double(0.0)
        rc = self.lib.vko_render_jobs(ctypes.cast(recs, ctypes.c_void_p), len(jobs), max(1, threads),
                                      ctypes.byref(ms))
        self._check(rc)
        for k, out in enumerate(outs):
            out["counters"] = recs[k].counters.as_dict()
        del keep
        return outs, ms.value

    def apply_film_resolve(self, hdr: np.ndarray, exposure: float = 1.0, white_balance_kelvin: float = 6500.0,
                           tone_map: str = "linear", output_transform: str = "gamma", gamma: float = 2.2,
                           clamp_output: bool = True) -> np.ndarray:
        """ApplyFilmResolve of an (H, W, 3) HDR film -> (H, W, 4) uint8."""
        hdr = np.ascontiguousarray(hdr, np.float32)
        h, w = hdr.shape[0], hdr.shape[1]

        class Resolve(ctypes.Structure):
            _fields_ = [("exposure", ctypes.c_float), ("white_balance_kelvin", ctypes.c_float),
                        ("tone_map", ctypes.c_uint32), ("output_transform", ctypes.c_uint32),
                        ("gamma", ctypes.c_float), ("clamp_output", ctypes.c_uint32)]
        rs = Resolve(exposure, white_balance_kelvin, {"linear": 0, "reinhard": 1, "filmic": 2, "aces": 3}[tone_map],
                     {"gamma": 0, "linear": 1}[output_transform], gamma, int(clamp_output))
        out = np.zeros((h, w, 4), np.uint8)
        self.lib.vko_apply_film_resolve.restype = ctypes.c_int
        self._check(self.lib.vko_apply_film_resolve(_ptr(hdr), w, h, ctypes.byref(rs), _ptr(out)))
        return out

    def convert_scene_json(self, path: str):
        """Reference only: a scene document converted by the reference's own
        SceneDocument loader and BuildSceneDataFromDocument, as a Scene."""
        import tempfile
        from vkpathtracer_b200 import scenes
        if self.kind != "reference":
            raise RuntimeError("scene documents are converted by the reference oracle only")
        self.lib.vko_convert_scene_json.restype = ctypes.c_int
        self.lib.vko_convert_scene_json.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
        with tempfile.TemporaryDirectory() as d:
            out = os.path.join(d, "snapshot.bin")
            self._check(self.lib.vko_convert_scene_json(path.encode(), out.encode()))
            return scenes.load_snapshot_dump(out, os.path.splitext(os.path.basename(path))[0])

    def build_bvh(self, scene, leaf_threshold: int = 4, deterministic: bool = True):
        sc, keep = self.make_scene(scene)
        n = scene.triangle_count
        nodes = np.zeros((max(1, 2 * n - 1), 10), np.uint32)
        prim = np.zeros(max(1, n), np.uint32)
        cnt = ctypes.c_uint32(0)
        rc = self.lib.vko_build_bvh(ctypes.byref(sc), leaf_threshold, int(deterministic), _ptr(nodes),
                                    ctypes.byref(cnt), _ptr(prim))
        del keep
        self._check(rc)
        return nodes[:cnt.value].copy(), prim[:n].copy()

    def intersect(self, scene, rays: np.ndarray, threads: int = 1, stats: bool = False):
        """Closest-hit: returns (prim uint32 [0xFFFFFFFF = miss], t float32, stats|None, ms)."""
        sc, keep = self.make_scene(scene)
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
        n = rays.shape[0]
        prim = np.zeros(n, np.uint32)
        t = np.zeros(n, np.float32)
        st = np.zeros(4, np.uint64) if stats else None
        ms = ctypes.c_double(0.0)
        rc = self.lib.vko_intersect(ctypes.byref(sc), _ptr(rays), n, threads, _ptr(prim), _ptr(t), _ptr(st),
                                    ctypes.byref(ms))
        del keep
        self._check(rc)
        return prim, t, st, ms.value


_CACHE = {}


def load(kind: str = "auto") -> Oracle:
    """kind: "reference", "port", "auto" (reference when built, else port) or
    "reference_avx2" (the reference's AVX2 build: CPU timing only)."""
    if kind == "auto":
        kind = "reference" if os.path.exists(REF_LIB) else "port"
    if kind in _CACHE:
        return _CACHE[kind]
    if kind == "reference":
        if not os.path.exists(REF_LIB):
            raise FileNotFoundError("reference oracle not built (oracle/_ref/libvkptref.so)")
        o = Oracle(REF_LIB)
    elif kind == "reference_avx2":
        if not os.path.exists(REF_AVX2_LIB):
            raise FileNotFoundError("reference AVX2 build missing (oracle/_ref_avx2/libvkptref.so)")
        o = Oracle(REF_AVX2_LIB)
    elif kind == "port":
        o = Oracle(build_port())
    else:
        raise ValueError(kind)
    _CACHE[kind] = o
    return o


def have_reference() -> bool:
    return os.path.exists(REF_LIB)


def have_reference_avx2() -> bool:
    return os.path.exists(REF_AVX2_LIB)


def build_adjoint(quiet: bool = True) -> str:
    """Compile the FP64 adjoint with g++ (no reference sources needed)."""
    os.makedirs(os.path.join(HERE, "_build"), exist_ok=True)
    deps = [os.path.join(HERE, f) for f in ("adjoint.cpp", "vkpt_adjoint.h", "vkpt_oracle.h")]
    if (not os.path.exists(ADJ_LIB)) or os.path.getmtime(ADJ_LIB) < max(os.path.getmtime(d) for d in deps):
        cmd = ["g++", "-std=c++20", "-O2", "-fPIC", "-shared", "-o", ADJ_LIB, deps[0], "-lpthread"]
        subprocess.run(cmd, check=True, capture_output=quiet)
    return ADJ_LIB


class VkoAdjointRequest(ctypes.Structure):
    _fields_ = [("params", ctypes.c_void_p), ("param_count", ctypes.c_uint32), ("spp", ctypes.c_uint32),
                ("first_sample", ctypes.c_uint32), ("frame", ctypes.c_uint32), ("target", ctypes.c_void_p),
                ("grad_index", ctypes.c_void_p), ("grad_count", ctypes.c_uint32), ("threads", ctypes.c_uint32),
                ("rr_params", ctypes.c_void_p)]


class AdjointOracle:
    """FP64 forward-mode adjoint of the render path (checker only)."""

    def __init__(self, path: str):
        self.lib = ctypes.CDLL(path)
        self.lib.vko_adjoint.restype = ctypes.c_int
        self.lib.vko_adjoint.argtypes = [ctypes.POINTER(VkoScene), ctypes.POINTER(VkoSettings),
                                         ctypes.POINTER(VkoAdjointRequest), ctypes.POINTER(ctypes.c_double),
                                         ctypes.c_void_p, ctypes.c_void_p]
        self.lib.vko_adjoint_last_error.restype = ctypes.c_char_p
        self.lib.vko_adjoint_fd.restype = ctypes.c_int
        self.lib.vko_adjoint_fd.argtypes = [ctypes.POINTER(VkoScene), ctypes.POINTER(VkoSettings),
                                            ctypes.POINTER(VkoAdjointRequest), ctypes.c_double, ctypes.c_void_p,
                                            ctypes.c_void_p]

    def finite_difference(self, scene, settings, params: np.ndarray, target: np.ndarray, spp: int, grad_index,
                          h: float = 1e-3, threads: int = 1, frame: int = 0, first_sample: int = 0):
        """Flip-excluding central differences (see vko_adjoint_fd): returns (fd, flips)."""
        sc, keep = Oracle.make_scene(scene)
        st = Oracle.make_settings(settings)
        p = np.ascontiguousarray(params, np.float32).reshape(-1)
        tg = np.ascontiguousarray(target, np.float32).reshape(-1)
        gi = np.ascontiguousarray(grad_index, np.uint32).reshape(-1)
        fd = np.zeros(max(1, gi.size), np.float64)
        flips = np.zeros(max(1, gi.size), np.uint64)
        rq = VkoAdjointRequest(_ptr(p), p.size, spp, first_sample, frame, _ptr(tg), _ptr(gi), gi.size, threads, None)
        rc = self.lib.vko_adjoint_fd(ctypes.byref(sc), ctypes.byref(st), ctypes.byref(rq), h, _ptr(fd), _ptr(flips))
        del keep
        if rc != 0:
            raise RuntimeError(f"adjoint oracle failed: {self.lib.vko_adjoint_last_error().decode()}")
        return fd[:gi.size], flips[:gi.size]

    def run(self, scene, settings, params: np.ndarray, target: Optional[np.ndarray], spp: int,
            grad_index, threads: int = 1, frame: int = 0, first_sample: int = 0,
            rr_params: Optional[np.ndarray] = None):
        """Returns (loss, grad[len(grad_index)], image (H, W, 3) float64)."""
        sc, keep = Oracle.make_scene(scene)
        st = Oracle.make_settings(settings)
        p = np.ascontiguousarray(params, np.float32).reshape(-1)
        tg = None if target is None else np.ascontiguousarray(target, np.float32).reshape(-1)
        gi = np.ascontiguousarray(grad_index, np.uint32).reshape(-1)
        grad = np.zeros(max(1, gi.size), np.float64)
        img = np.zeros((settings.height, settings.width, 3), np.float64)
        rp = None if rr_params is None else np.ascontiguousarray(rr_params, np.float32).reshape(-1)
        if rp is not None and rp.size != p.size:
            raise ValueError("rr_params must have the shape of params")
        rq = VkoAdjointRequest(_ptr(p), p.size, spp, first_sample, frame, _ptr(tg), _ptr(gi) if gi.size else None,
                               gi.size, threads, _ptr(rp))
        loss = ctypes.c_double(0.0)
        rc = self.lib.vko_adjoint(ctypes.byref(sc), ctypes.byref(st), ctypes.byref(rq), ctypes.byref(loss),
                                  _ptr(grad), _ptr(img))
        del keep
        if rc != 0:
            raise RuntimeError(f"adjoint oracle failed: {self.lib.vko_adjoint_last_error().decode()}")
        return loss.value, grad[:gi.size], img


def load_adjoint() -> AdjointOracle:
    if "adjoint" not in _CACHE:
        _CACHE["adjoint"] = AdjointOracle(build_adjoint())
    return _CACHE["adjoint"]
