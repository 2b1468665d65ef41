"""Seeded synthetic scenes and ray sets for the render hot path.

Every workload is generated here from a documented splitmix64 stream, so the
CUDA path, the CPU oracle and the benchmark see bit-identical float32 inputs.
There is no dataset: the reference's own fixtures are binary LFS assets, so
each workload is procedural with the shapes, sizes and value ranges of the
benchmark configurations:

  cornell_box()          closed box scene (36 triangles), 256x256, 16 spp, depth 8
  displaced_sphere()     1,046,904-triangle value-noise sphere + 8,388,608 query rays
  sphere_grid()          64x64 displaced spheres (~2M triangles), 1920x1080, 64 spp, depth 16
  batch_jobs()           64 uneven render jobs for the persistent batched renderer
  inverse_box_scene()    the box room with 16 boxes and a 64-parameter material vector
  effect_gallery()       the box room with one box per procedural material effect (1..19)
  sky_scene()            displaced spheres under an equirectangular sky map

Scene records use the reference's standard GPU word maps
(src/gpu/VulkanGpuPathTracer.cpp:323-338 for materials, :381-396 for lights),
so a packed buffer from the reference's Vulkan backend is accepted unchanged.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

import numpy as np

MASK64 = (1 << 64) - 1

# Material word offsets (16 floats per material).
M_ALBEDO, M_EMISSIVE, M_ROUGHNESS, M_MODEL, M_METALLIC, M_IOR = 0, 3, 6, 7, 8, 9
M_TRANSMISSION, M_CLEARCOAT, M_SHEEN, M_ANISO, M_ALPHA, M_EFFECT = 10, 11, 12, 13, 14, 15
# Light word offsets (16 floats per light).
L_POS, L_COLOR, L_INTENSITY, L_RADIUS, L_DIR, L_INNER, L_OUTER = 0, 3, 6, 7, 8, 11, 12


def splitmix64(x: int) -> int:
    """One splitmix64 step on a Python int (same constants as the reference RNG)."""
    x = (x + 0x9E3779B97F4A7C15) & MASK64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & MASK64
    return x ^ (x >> 31)


def splitmix64_np(x: np.ndarray) -> np.ndarray:
    """Vectorised splitmix64 over a uint64 array (wrapping arithmetic)."""
    x = x.astype(np.uint64, copy=True)
    with np.errstate(over="ignore"):
        x += np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


class Stream:
    """Generator stream: state_{k+1} = splitmix64(state_k); uniform = top 24 bits / 2^24."""

    def __init__(self, seed: int):
        self.state = splitmix64(seed & MASK64)

    def next_u64(self) -> int:
        self.state = splitmix64(self.state)
        return self.state

    def uniform(self, lo: float = 0.0, hi: float = 1.0) -> float:
        u = (self.next_u64() >> 40) * (1.0 / 16777216.0)
        return lo + (hi - lo) * u

    def randint(self, lo: int, hi: int) -> int:
        """Integer in [lo, hi]."""
        return lo + int(self.uniform() * (hi - lo + 1)) if hi > lo else lo

    def uniform_np(self, n: int) -> np.ndarray:
        """n uniforms in [0,1) as float64, from a counter-keyed block of this stream."""
        base = self.next_u64()
        keys = np.arange(n, dtype=np.uint64) + np.uint64(base)
        return (splitmix64_np(keys) >> np.uint64(40)).astype(np.float64) * (1.0 / 16777216.0)


@dataclasses.dataclass
class Camera:
    position: tuple = (0.0, 0.0, 0.0)
    target: tuple = (0.0, 0.0, -1.0)
    up: tuple = (0.0, 1.0, 0.0)
    fov_deg: float = 60.0
    aperture_radius: float = 0.0
    focus_distance: float = 0.0
    # thin-lens shape (PathTracerSceneSnapshot camera_iris_* / camera_anamorphic_squeeze)
    iris_blade_count: int = 0
    iris_rotation_degrees: float = 0.0
    iris_roundness: float = 1.0
    anamorphic_squeeze: float = 1.0


@dataclasses.dataclass
class Scene:
    """Flattened scene in the layout of the reference's PathTracerSceneSnapshot."""
    vertices: np.ndarray            # (V,3) float32
    indices: np.ndarray             # (T,3) uint32
    instances: np.ndarray           # (I,3) uint32: first_triangle, triangle_count, material_index
    materials: np.ndarray           # (M,16) float32
    lights: np.ndarray              # (L,16) float32
    environment: tuple = (0.0, 0.0, 0.0)
    camera: Camera = dataclasses.field(default_factory=Camera)
    name: str = "scene"
    env_map: Optional[np.ndarray] = None   # (H, W, 3) float32 equirectangular map, row 0 toward +y
    env_scale: tuple = (0.0, 0.0, 0.0)     # texel multiplier (all <= 1e-6 means 1)
    sdf: Optional[np.ndarray] = None       # (N, 16) float32 SDF primitive records (sdf_primitive)
    # dynamic-transform instances (all None when the scene has none)
    instance_local: Optional[np.ndarray] = None        # (I, 5) uint32: flags, local first/count vertex, first/count index
    instance_transforms: Optional[np.ndarray] = None   # (I, 10) float32: translation3, quaternion xyzw, scale3
    local_vertices: Optional[np.ndarray] = None        # (V', 3) float32
    local_indices: Optional[np.ndarray] = None         # (K,) uint32

    @property
    def triangle_count(self) -> int:
        return int(self.indices.shape[0])

    def contiguous(self) -> "Scene":
        self.vertices = np.ascontiguousarray(self.vertices, dtype=np.float32)
        self.indices = np.ascontiguousarray(self.indices, dtype=np.uint32)
        self.instances = np.ascontiguousarray(self.instances, dtype=np.uint32).reshape(-1, 3)
        self.materials = np.ascontiguousarray(self.materials, dtype=np.float32).reshape(-1, 16)
        self.lights = np.ascontiguousarray(self.lights, dtype=np.float32).reshape(-1, 16)
        return self


@dataclasses.dataclass
class RenderSettings:
    """Mirror of the reference's RenderSettings (src/pathtracer/PathTracer.h:134-178)."""
    width: int = 256
    height: int = 256
    spp: int = 8
    max_depth: int = 6
    seed: int = 0x12345678
    enable_nee: bool = True
    enable_mis: bool = True
    deterministic: bool = True
    russian_roulette_start_depth: int = 3
    russian_roulette_min_survival: float = 0.1
    russian_roulette_max_survival: float = 0.99
    camera_aperture_radius: float = 0.0
    camera_focus_distance: float = 0.0
    # Extension absent from the reference: per-channel clamp of each sample's
    # radiance before accumulation (0 = off, the reference's behaviour).
    firefly_clamp: float = 0.0


def material(albedo=(1.0, 1.0, 1.0), emissive=(0.0, 0.0, 0.0), roughness=1.0, model=0,
             metallic=0.0, ior=1.5, transmission=0.0, clearcoat=0.0, sheen=0.0,
             anisotropy=0.0, alpha=1.0, effect=0, double_sided=False) -> np.ndarray:
    m = np.zeros(16, dtype=np.float32)
    m[0:3] = albedo
    m[3:6] = emissive
    m[M_ROUGHNESS] = roughness
    m[M_MODEL] = float(model)
    m[M_METALLIC] = metallic
    m[M_IOR] = ior
    m[M_TRANSMISSION] = transmission
    m[M_CLEARCOAT] = clearcoat
    m[M_SHEEN] = sheen
    m[M_ANISO] = anisotropy
    m[M_ALPHA] = alpha
    m[M_EFFECT] = float((effect & 1023) | (1024 if double_sided else 0))
    return m


def point_light(position, color, intensity, radius=0.0, direction=(0.0, -1.0, 0.0),
                spot_inner_cos=-1.0, spot_outer_cos=-1.0) -> np.ndarray:
    l = np.zeros(16, dtype=np.float32)
    l[0:3] = position
    l[3:6] = color
    l[L_INTENSITY] = intensity
    l[L_RADIUS] = max(0.0, radius)
    l[8:11] = direction
    l[L_INNER] = spot_inner_cos
    l[L_OUTER] = spot_outer_cos
    return l


class _Builder:
    def __init__(self):
        self.verts: List[np.ndarray] = []
        self.tris: List[np.ndarray] = []
        self.instances: List[tuple] = []
        self.nv = 0
        self.nt = 0

    def add(self, verts: np.ndarray, tris: np.ndarray, material_index: int):
        verts = np.asarray(verts, dtype=np.float32).reshape(-1, 3)
        tris = np.asarray(tris, dtype=np.int64).reshape(-1, 3) + self.nv
        self.instances.append((self.nt, tris.shape[0], material_index))
        self.verts.append(verts)
        self.tris.append(tris.astype(np.uint32))
        self.nv += verts.shape[0]
        self.nt += tris.shape[0]

    def arrays(self):
        return (np.concatenate(self.verts).astype(np.float32),
                np.concatenate(self.tris).astype(np.uint32),
                np.array(self.instances, dtype=np.uint32).reshape(-1, 3))


def _quad(p0, p1, p2, p3):
    """Quad p0-p1-p2-p3 as two triangles (0,1,2), (0,2,3)."""
    return np.array([p0, p1, p2, p3], dtype=np.float32), np.array([[0, 1, 2], [0, 2, 3]])


def _box(center, half, yaw_deg):
    """Axis-aligned box rotated about +y; 8 vertices, 12 triangles."""
    cx, cy, cz = center
    hx, hy, hz = half
    a = math.radians(yaw_deg)
    c, s = math.cos(a), math.sin(a)
    corners = []
    for (sx, sy, sz) in [(-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1),
                         (-1, -1, 1), (1, -1, 1), (1, 1, 1), (-1, 1, 1)]:
        x, y, z = sx * hx, sy * hy, sz * hz
        corners.append((cx + c * x + s * z, cy + y, cz - s * x + c * z))
    tris = [[0, 5, 4], [0, 1, 5], [3, 7, 6], [3, 6, 2], [0, 2, 1], [0, 3, 2],
            [4, 5, 6], [4, 6, 7], [0, 4, 7], [0, 7, 3], [1, 2, 6], [1, 6, 5]]
    return np.array(corners, dtype=np.float32), np.array(tris)


def _room(b: _Builder, materials: list, st: Stream, albedo_lo=0.1, albedo_hi=0.8):
    """Unit box x,z in [-0.5,0.5], y in [0,1], open towards +z: 5 inward quads (10 tris)."""
    walls = [
        ((-0.5, 0, -0.5), (-0.5, 0, 0.5), (0.5, 0, 0.5), (0.5, 0, -0.5)),      # floor
        ((-0.5, 1, -0.5), (0.5, 1, -0.5), (0.5, 1, 0.5), (-0.5, 1, 0.5)),      # ceiling
        ((-0.5, 0, -0.5), (0.5, 0, -0.5), (0.5, 1, -0.5), (-0.5, 1, -0.5)),    # back
        ((-0.5, 0, -0.5), (-0.5, 1, -0.5), (-0.5, 1, 0.5), (-0.5, 0, 0.5)),    # left
        ((0.5, 0, -0.5), (0.5, 0, 0.5), (0.5, 1, 0.5), (0.5, 1, -0.5)),        # right
    ]
    for w in walls:
        alb = tuple(st.uniform(albedo_lo, albedo_hi) for _ in range(3))
        materials.append(material(albedo=alb, roughness=1.0))
        v, t = _quad(*w)
        b.add(v, t, len(materials) - 1)


def _ceiling_light(b: _Builder, materials: list, lights: list, size=0.25, radiance=(17.0, 12.0, 4.0),
                   height=0.999, center=(0.0, 0.0)):
    """Emissive quad plus the co-located point light that drives NEE.

    The reference's NEE samples only point/sphere lights, so an area light is
    represented as in its Cornell fixture (assets/scenes/cornell_native.json:
    emissive quad + point light at the same spot): intensity = quad area.
    """
    h = size * 0.5
    cx, cz = center
    materials.append(material(albedo=(0.78, 0.78, 0.78), emissive=radiance, roughness=1.0))
    v, t = _quad((cx - h, height, cz - h), (cx + h, height, cz - h), (cx + h, height, cz + h), (cx - h, height, cz + h))
    b.add(v, t, len(materials) - 1)
    lights.append(point_light((cx, height - 0.001, cz), radiance, size * size))


def cornell_box(seed: int = 1) -> Scene:
    """Closed box (10 tris) + 2 boxes rotated U[-30,30] deg (24 tris) + 0.25x0.25 light (2 tris)."""
    st = Stream(seed)
    b = _Builder()
    mats: list = []
    lights: list = []
    _room(b, mats, st)
    for center, half in [((-0.17, 0.3, -0.15), (0.14, 0.3, 0.14)), ((0.18, 0.15, 0.12), (0.14, 0.15, 0.14))]:
        alb = tuple(st.uniform(0.1, 0.8) for _ in range(3))
        mats.append(material(albedo=alb, roughness=1.0))
        yaw = st.uniform(-30.0, 30.0)
        v, t = _box(center, half, yaw)
        b.add(v, t, len(mats) - 1)
    _ceiling_light(b, mats, lights)
    v, t, inst = b.arrays()
    cam = Camera(position=(0.0, 0.5, 1.9), target=(0.0, 0.5, 0.0), up=(0.0, 1.0, 0.0), fov_deg=40.0)
    return Scene(v, t, inst, np.array(mats), np.array(lights), (0.0, 0.0, 0.0), cam, "cornell_box").contiguous()


def effect_gallery(seed: int = 11) -> Scene:
    """The closed box with every procedural material effect (1..19): 19 small
    boxes on the floor, one per effect, with varied roughness, clear coat and
    sheen (the wood species read both); parquet floor and checker back wall."""
    st = Stream(seed)
    b = _Builder()
    mats: list = []
    lights: list = []
    _room(b, mats, st)
    mats[0][M_EFFECT] = 17.0   # floor: parquet
    mats[2][M_EFFECT] = 9.0    # back wall: check pattern
    for k in range(19):
        gx, gz = k % 5, k // 5
        cx, cz = -0.36 + 0.18 * gx, -0.33 + 0.18 * gz
        hy = st.uniform(0.03, 0.09)
        alb = tuple(st.uniform(0.2, 0.9) for _ in range(3))
        rough = (0.2, 0.5, 0.8, 1.0)[k % 4]
        model = (0, 3, 6, 7)[k % 4]
        mats.append(material(albedo=alb, roughness=rough, model=model, clearcoat=0.5 if model == 7 else 0.0,
                             sheen=0.7 if model == 6 else 0.0, effect=k + 1))
        v, t = _box((cx, hy, cz), (0.06, hy, 0.06), st.uniform(-30.0, 30.0))
        b.add(v, t, len(mats) - 1)
    _ceiling_light(b, mats, lights)
    v, t, inst = b.arrays()
    cam = Camera(position=(0.0, 0.5, 1.9), target=(0.0, 0.3, 0.0), up=(0.0, 1.0, 0.0), fov_deg=40.0)
    return Scene(v, t, inst, np.array(mats), np.array(lights), (0.02, 0.02, 0.03), cam, "effect_gallery").contiguous()


def load_snapshot_dump(path: str, name: str = "") -> Scene:
    """A PathTracerSceneSnapshot written by the reference oracle's scene
    converter (vko_convert_scene_json: SceneDocument -> BuildSceneDataFromDocument),
    layout documented in oracle/ref_shim.cpp."""
    with open(path, "rb") as f:
        data = f.read()
    if data[:4] != b"VKSJ":
        raise ValueError("not a snapshot dump")
    head = np.frombuffer(data, np.uint32, 11, 4)
    version = int(head[0])
    if version not in (1, 2):
        raise ValueError("unknown snapshot dump version")
    nv, ni, ninst, nmat, nlight, nsdf, nlv, nli, ew, eh = (int(x) for x in head[1:])
    off = 48

    def take(dtype, n):
        nonlocal off
        a = np.frombuffer(data, dtype, n, off).copy()
        off += 4 * n
        return a

    vertices = take(np.float32, 3 * nv).reshape(-1, 3)
    indices = take(np.uint32, ni)
    instances = take(np.uint32, 3 * ninst).reshape(-1, 3)
    instance_local = take(np.uint32, 5 * ninst).reshape(-1, 5)
    instance_transforms = take(np.float32, 10 * ninst).reshape(-1, 10)
    materials = take(np.float32, 16 * nmat).reshape(-1, 16)
    lights = take(np.float32, 16 * nlight).reshape(-1, 16)
    sdf = take(np.float32, 16 * nsdf).reshape(-1, 16)
    local_vertices = take(np.float32, 3 * nlv).reshape(-1, 3)
    local_indices = take(np.uint32, nli)
    env = take(np.float32, 3)
    cam = take(np.float32, 12).astype(np.float64)
    env_scale = take(np.float32, 3)
    env_map = take(np.float32, 3 * ew * eh).reshape(eh, ew, 3) if ew * eh else None
    camera = Camera(tuple(cam[0:3]), tuple(cam[3:6]), tuple(cam[6:9]), float(cam[9]), float(cam[10]), float(cam[11]))
    if version >= 2:   # lens shape
        camera.iris_blade_count = int(take(np.uint32, 1)[0])
        lens = take(np.float32, 3).astype(np.float64)
        camera.iris_rotation_degrees, camera.iris_roundness, camera.anamorphic_squeeze = (float(x) for x in lens)
    # trailing partial triangles are ignored by the accelerator (index checks), so keep the flat array
    return Scene(vertices, indices.reshape(-1, 3) if ni % 3 == 0 else indices, instances, materials, lights,
                 tuple(float(x) for x in env), camera, name or "snapshot", env_map=env_map,
                 env_scale=tuple(float(x) for x in env_scale), sdf=sdf if nsdf else None,
                 instance_local=instance_local, instance_transforms=instance_transforms,
                 local_vertices=local_vertices, local_indices=local_indices).contiguous()


SDF_SHAPES = {"sphere": 0, "box": 1, "rounded_box": 2, "plane": 3, "torus": 4, "capsule": 5}


def sdf_primitive(shape: str, position, scale=(1.0, 1.0, 1.0), rotation=(0.0, 0.0, 0.0), material: int = 0,
                  radius: float = 0.5, param_a: float = 0.0, param_b: float = 0.0) -> np.ndarray:
    """One RTSdfPrimitive record (src/pathtracer/PathTracer.h:330-339) as 16
    floats: shape, position3, scale3, rotation3 (Euler radians), material,
    radius, param_a, param_b, 0, 0.  The reference measures a box's and a
    rounded box's half extents in primitive space (world / scale), so their
    world half extents are scale * scale."""
    r = np.zeros(16, np.float32)
    r[0] = SDF_SHAPES[shape]
    r[1:4], r[4:7], r[7:10] = position, scale, rotation
    r[10], r[11], r[12], r[13] = material, radius, param_a, param_b
    return r


def sdf_gallery(seed: int = 7, glass: bool = False) -> Scene:
    """One SDF primitive of every shape on a triangle ground with two triangle
    boxes: a scaled, rotated ellipsoid (analytic sphere test), a box, a rounded
    box, a torus (scaled) and a capsule (sphere-traced), and a vertical SDF
    plane as the back wall.  The marched shapes keep scale ~1: the reference
    marches by primitive-space distance (world / scale), which overshoots thin
    shapes at small scales.  Materials span Lambert, glossy, metal, mirror and
    sheen; glass=True makes the ellipsoid transmissive (the shadow test then
    steps through it).  One point light and a constant sky."""
    st = Stream(seed)
    b = _Builder()
    mats: list = [material(albedo=(0.55, 0.55, 0.5), roughness=1.0)]
    v, t = _quad((-8.0, 0.0, -8.0), (-8.0, 0.0, 8.0), (8.0, 0.0, 8.0), (8.0, 0.0, -8.0))
    b.add(v, t, 0)
    for k in range(2):
        mats.append(material(albedo=tuple(st.uniform(0.3, 0.8) for _ in range(3)), roughness=1.0))
        v, t = _box((-3.2 + 6.0 * k, 0.4, 2.6 - 5.0 * k), (0.4, 0.4, 0.4), st.uniform(-30.0, 30.0))
        b.add(v, t, len(mats) - 1)
    lights = [point_light((3.0, 8.0, 5.0), (1.0, 0.95, 0.9), 120.0)]
    base = len(mats)
    mats.append(material(albedo=(0.9, 0.9, 0.95), roughness=0.0, model=5, ior=1.5, transmission=0.9) if glass
                else material(albedo=(0.8, 0.3, 0.2), roughness=0.35, model=3))
    mats.append(material(albedo=(0.3, 0.6, 0.8), roughness=1.0))
    mats.append(material(albedo=(0.9, 0.75, 0.4), roughness=0.3, metallic=0.9, model=4))
    mats.append(material(albedo=(0.95, 0.95, 0.95), roughness=0.0, model=2))
    mats.append(material(albedo=(0.5, 0.8, 0.4), roughness=0.7, model=6, sheen=0.6))
    mats.append(material(albedo=(0.7, 0.62, 0.55), roughness=1.0))
    sdf = np.stack([
        sdf_primitive("sphere", (-3.0, 1.0, 0.0), (1.2, 1.0, 0.9), (0.3, 0.5, 0.0), base + 0, radius=1.0),
        sdf_primitive("box", (0.0, 1.0, -1.5), (1.0, 1.0, 1.0), (0.0, 0.6, 0.0), base + 1),
        sdf_primitive("rounded_box", (3.0, 1.0, -0.5), (1.0, 1.0, 1.0), (0.2, -0.4, 0.1), base + 2, param_a=0.3),
        sdf_primitive("torus", (-1.3, 0.9, 2.2), (0.8, 0.8, 0.8), (1.1, 0.3, 0.0), base + 3, radius=0.3,
                      param_a=1.0),
        sdf_primitive("capsule", (1.8, 1.4, 2.0), (1.0, 1.0, 1.0), (0.0, 0.0, 0.7), base + 4, radius=0.5,
                      param_a=0.8),
        sdf_primitive("plane", (0.0, 0.0, -6.0), (1.0, 1.0, 1.0), (1.5707964, 0.0, 0.0), base + 5),
    ])
    v, t, inst = b.arrays()
    cam = Camera(position=(0.0, 4.5, 10.0), target=(0.0, 0.8, 0.0), up=(0.0, 1.0, 0.0), fov_deg=45.0)
    return Scene(v, t, inst, np.array(mats), np.array(lights), (0.25, 0.3, 0.4), cam,
                 "sdf_glass" if glass else "sdf_gallery", sdf=sdf).contiguous()


def sdf_complexity() -> Scene:
    """SDF primitives only (no triangles), after the reference's SDF
    complexity scene (assets/scenes/sdf_complexity.json): a sphere of scale
    0.8 at (0, 1, 0) and a box of scale (0.4, 0.6, 0.4) at (1.2, 0.5, 0) in
    one matte material, on an SDF ground plane, lit by one point light and a
    constant sky."""
    mats = np.array([material(albedo=(0.72, 0.72, 0.88), roughness=1.0),
                     material(albedo=(0.5, 0.5, 0.45), roughness=1.0)])
    lights = np.array([point_light((2.0, 4.0, 3.0), (0.85, 0.9, 1.0), 14.0)])
    sdf = np.stack([
        sdf_primitive("sphere", (0.0, 1.0, 0.0), (0.8, 0.8, 0.8), material=0, radius=0.8),
        sdf_primitive("box", (1.2, 0.5, 0.0), (0.4, 0.6, 0.4), material=0, radius=1.0, param_a=0.4),
        sdf_primitive("plane", (0.0, 0.0, 0.0), material=1),
    ])
    cam = Camera(position=(0.6, 1.4, 4.2), target=(0.5, 0.6, 0.0), up=(0.0, 1.0, 0.0), fov_deg=58.0)
    empty_v = np.zeros((0, 3), np.float32)
    empty_t = np.zeros((0, 3), np.uint32)
    return Scene(empty_v, empty_t, np.zeros((0, 3), np.uint32), mats, lights, (0.35, 0.4, 0.5), cam,
                 "sdf_complexity", sdf=sdf).contiguous()


def cornell_settings(width=256, height=256, spp=16) -> RenderSettings:
    return RenderSettings(width=width, height=height, spp=spp, max_depth=8, seed=1234,
                          enable_nee=True, enable_mis=True)


# ---------------------------------------------------------------- value noise
def _lattice(ix, iy, iz, octave: int, seed: int) -> np.ndarray:
    key = (ix.astype(np.int64).astype(np.uint64) * np.uint64(0x9E3779B1)) ^ \
          (iy.astype(np.int64).astype(np.uint64) * np.uint64(0x85EBCA77) << np.uint64(20)) ^ \
          (iz.astype(np.int64).astype(np.uint64) * np.uint64(0xC2B2AE3D) << np.uint64(40))
    key = key ^ np.uint64(splitmix64((seed * 131 + octave) & MASK64))
    return (splitmix64_np(key) >> np.uint64(40)).astype(np.float64) * (1.0 / 16777216.0)


def value_noise(p: np.ndarray, octaves: int, seed: int) -> np.ndarray:
    """fBm of trilinear value noise with smoothstep weights, in [-1, 1] (float64)."""
    total = np.zeros(p.shape[0])
    norm = 0.0
    amp = 1.0
    freq = 2.0
    for o in range(octaves):
        q = p * freq
        i0 = np.floor(q)
        f = q - i0
        w = f * f * (3.0 - 2.0 * f)
        ix, iy, iz = i0[:, 0], i0[:, 1], i0[:, 2]
        acc = np.zeros(p.shape[0])
        for dx in (0, 1):
            wx = w[:, 0] if dx else 1.0 - w[:, 0]
            for dy in (0, 1):
                wy = w[:, 1] if dy else 1.0 - w[:, 1]
                for dz in (0, 1):
                    wz = w[:, 2] if dz else 1.0 - w[:, 2]
                    acc += wx * wy * wz * _lattice(ix + dx, iy + dy, iz + dz, o, seed)
        total += amp * (2.0 * acc - 1.0)
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return total / norm


def _uv_sphere(n_lat: int, n_lon: int):
    """Grid sphere: n_lat rows pole to pole x n_lon columns; 2*(n_lat-1)*n_lon triangles."""
    theta = np.linspace(0.0, math.pi, n_lat)
    phi = np.arange(n_lon) * (2.0 * math.pi / n_lon)
    st, ct = np.sin(theta)[:, None], np.cos(theta)[:, None]
    dirs = np.stack([st * np.cos(phi)[None, :], np.broadcast_to(ct, (n_lat, n_lon)), st * np.sin(phi)[None, :]], axis=-1)
    dirs = dirs.reshape(-1, 3)
    i = np.arange(n_lat - 1)[:, None]
    j = np.arange(n_lon)[None, :]
    a = i * n_lon + j
    b2 = i * n_lon + (j + 1) % n_lon
    c = (i + 1) * n_lon + j
    d = (i + 1) * n_lon + (j + 1) % n_lon
    t1 = np.stack([a, c, b2], axis=-1).reshape(-1, 3)
    t2 = np.stack([b2, c, d], axis=-1).reshape(-1, 3)
    tris = np.stack([t1, t2], axis=1).reshape(-1, 3)
    return dirs, tris


def displaced_sphere(resolution: int = 724, amplitude: float = 0.05, octaves: int = 8,
                     seed: int = 2, scale: float = 16.0, weld_poles: bool = False) -> Scene:
    """Grid sphere (resolution x resolution vertices), radius 1 displaced radially by
    value-noise fBm of the given amplitude, then scaled uniformly.

    At resolution 724 this is 2*723*724 = 1,046,904 triangles.  The scale factor
    16 keeps triangles clear of the reference's absolute |det| < 1e-4 cull,
    which rejects every triangle of the unit-radius mesh.

    sin(pi) is not 0 in floating point, so the last row is a ring of distinct
    vertices about 1e-15 apart around the south pole: a hole no triangle
    covers.  weld_poles=True moves each pole row onto one vertex, which makes
    the mesh closed (for watertightness checks).
    """
    dirs, tris = _uv_sphere(resolution, resolution)
    r = 1.0 + amplitude * value_noise(dirs, octaves, seed)
    verts = (dirs * (r * scale)[:, None]).astype(np.float32)
    if weld_poles:
        verts[:resolution] = verts[0]
        verts[-resolution:] = np.array([0.0, verts[-resolution:, 1].mean(), 0.0], np.float32)
    mats = np.array([material(albedo=(0.7, 0.7, 0.7), roughness=1.0)])
    inst = np.array([[0, tris.shape[0], 0]], dtype=np.uint32)
    cam = Camera(position=(0.0, 0.0, 3.0 * scale), target=(0.0, 0.0, 0.0), fov_deg=45.0)
    return Scene(verts, tris.astype(np.uint32), inst, mats, np.zeros((0, 16), np.float32),
                 (0.0, 0.0, 0.0), cam, "displaced_sphere").contiguous()


def edge_probe_rays(scene: Scene, origins, edge_fracs=(0.5, 1.0 / 3.0), max_rays: int = 0,
                    seed: int = 0) -> np.ndarray:
    """(N,6) float32 rays from each origin aimed at every vertex of the scene
    and at points along every edge (fractions edge_fracs): the rays that slip
    between the triangles of a closed mesh when the triangle test is not
    watertight.  max_rays > 0 keeps a seeded random subset of that size."""
    v = np.asarray(scene.vertices, np.float64)
    tri = np.asarray(scene.indices, np.int64).reshape(-1, 3)
    edges = np.concatenate([tri[:, [0, 1]], tri[:, [1, 2]], tri[:, [2, 0]]])
    edges = np.unique(np.sort(edges, axis=1), axis=0)
    targets = np.concatenate([v] + [v[edges[:, 0]] + f * (v[edges[:, 1]] - v[edges[:, 0]]) for f in edge_fracs])
    out = []
    for o in origins:
        o = np.asarray(o, np.float64)
        d = targets - o
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        out.append(np.concatenate([np.broadcast_to(o, d.shape), d], axis=1))
    rays = np.concatenate(out).astype(np.float32)
    if max_rays and rays.shape[0] > max_rays:
        keep = np.sort(np.random.RandomState(seed).choice(rays.shape[0], max_rays, replace=False))
        rays = rays[keep]
    return np.ascontiguousarray(rays)


def _normalize_f32(v: np.ndarray) -> np.ndarray:
    v = v.astype(np.float32)
    n = np.sqrt((v * v).sum(axis=1, dtype=np.float32)).astype(np.float32)
    return (v / n[:, None]).astype(np.float32)


def primary_rays(camera: Camera, width: int, height: int) -> np.ndarray:
    """Pinhole rays through pixel centres, (N,6) float32 rows o3,d3, row-major pixels."""
    pos = np.array(camera.position, np.float64)
    fwd = np.array(camera.target, np.float64) - pos
    fwd /= np.linalg.norm(fwd)
    right = np.cross(fwd, np.array(camera.up, np.float64))
    right /= np.linalg.norm(right)
    up = np.cross(right, fwd)
    th = math.tan(0.5 * math.radians(camera.fov_deg))
    aspect = width / height
    xs = (2.0 * (np.arange(width) + 0.5) / width - 1.0) * aspect * th
    ys = (1.0 - 2.0 * (np.arange(height) + 0.5) / height) * th
    nx, ny = np.meshgrid(xs, ys)
    d = fwd[None, :] + right[None, :] * nx.reshape(-1, 1) + up[None, :] * ny.reshape(-1, 1)
    d = _normalize_f32(d)
    o = np.broadcast_to(pos.astype(np.float32), d.shape)
    return np.ascontiguousarray(np.concatenate([o, d], axis=1), dtype=np.float32)


def random_rays(n: int, half_extent: float, seed: int) -> np.ndarray:
    """Origins uniform in [-h,h]^3, directions uniform on the unit sphere; (n,6) float32."""
    st = Stream(seed)
    ox, oy, oz = (st.uniform_np(n) * 2.0 - 1.0) * half_extent, (st.uniform_np(n) * 2.0 - 1.0) * half_extent, \
                 (st.uniform_np(n) * 2.0 - 1.0) * half_extent
    z = 1.0 - 2.0 * st.uniform_np(n)
    ph = 2.0 * math.pi * st.uniform_np(n)
    rr = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    d = _normalize_f32(np.stack([rr * np.cos(ph), rr * np.sin(ph), z], axis=1))
    o = np.stack([ox, oy, oz], axis=1).astype(np.float32)
    return np.ascontiguousarray(np.concatenate([o, d], axis=1), dtype=np.float32)


def ray_query_rays(scene: Scene, primary_side: int = 2048, random_count: int = 4194304,
                   scale: float = 16.0, seed: int = 3) -> np.ndarray:
    """The ray-query workload: primary_side^2 coherent camera rays followed by
    random_count incoherent rays (origins in [-1.5,1.5]^3 * scale)."""
    prim = primary_rays(scene.camera, primary_side, primary_side)
    rnd = random_rays(random_count, 1.5 * scale, seed)
    return np.ascontiguousarray(np.concatenate([prim, rnd], axis=0))


# ----------------------------------------------------------------- sphere grid
def _displaced_unit_sphere_mesh(n_lat: int, n_lon: int, amplitude: float, seed: int, octaves: int = 4):
    dirs, tris = _uv_sphere(n_lat, n_lon)
    r = 1.0 + amplitude * value_noise(dirs, octaves, seed)
    return dirs * r[:, None], tris


def sphere_field(grid: int, n_lat: int, n_lon: int, seed: int, spacing: float = 3.0, radius: float = 1.0,
                 n_lights: int = 16, environment: float = 0.1, light_size: float = 6.0,
                 light_height: float = 14.0) -> Scene:
    """grid x grid displaced spheres with the mixed material set:
    50% Lambert (albedo U[0.05,0.9]^3), 30% glossy (roughness U[0.05,0.5], F0 U[0.02,0.9]),
    20% mirror; n_lights quad area lights with radiance U[1,20]^3; constant environment.

    "GGX glossy (roughness, F0)" maps onto the reference's glossy lobe: a
    roughness-driven Phong lobe with ior = (1+sqrt(F0))/(1-sqrt(F0)), since the
    reference integrator has no GGX (src/pathtracer/ScalarCpuPathTracer.cpp:1240-1251).
    """
    st = Stream(seed)
    b = _Builder()
    mats: list = []
    lights: list = []
    # A handful of distinct sphere shapes, instanced by translation (vertices are baked).
    shapes = [_displaced_unit_sphere_mesh(n_lat, n_lon, 0.05, seed * 17 + k) for k in range(8)]
    half = 0.5 * (grid - 1) * spacing
    for gy in range(grid):
        for gx in range(grid):
            dirs, tris = shapes[st.randint(0, len(shapes) - 1)]
            center = np.array([gx * spacing - half, radius, gy * spacing - half])
            pick = st.uniform()
            if pick < 0.5:
                alb = tuple(st.uniform(0.05, 0.9) for _ in range(3))
                mats.append(material(albedo=alb, roughness=1.0, model=0))
            elif pick < 0.8:
                alb = tuple(st.uniform(0.05, 0.9) for _ in range(3))
                rough = st.uniform(0.05, 0.5)
                f0 = st.uniform(0.02, 0.9)
                sf = math.sqrt(f0)
                ior = (1.0 + sf) / max(1e-6, 1.0 - sf)
                mats.append(material(albedo=alb, roughness=rough, model=3, ior=ior))
            else:
                alb = tuple(st.uniform(0.7, 0.98) for _ in range(3))
                mats.append(material(albedo=alb, roughness=0.0, model=2))
            b.add(center[None, :] + dirs * radius, tris, len(mats) - 1)
    # Ground plane under the field.
    mats.append(material(albedo=(0.5, 0.5, 0.5), roughness=1.0))
    g = half + 2.0 * spacing
    v, t = _quad((-g, 0.0, -g), (-g, 0.0, g), (g, 0.0, g), (g, 0.0, -g))
    b.add(v, t, len(mats) - 1)
    # Quad area lights on a 4x4 lattice above the field.
    side = int(math.ceil(math.sqrt(n_lights)))
    for k in range(n_lights):
        lx = ((k % side) + 0.5) / side * 2.0 * half - half
        lz = ((k // side) + 0.5) / side * 2.0 * half - half
        le = tuple(st.uniform(1.0, 20.0) for _ in range(3))
        hs = 0.5 * light_size
        mats.append(material(albedo=(0.78, 0.78, 0.78), emissive=le, roughness=1.0))
        v, t = _quad((lx - hs, light_height, lz - hs), (lx + hs, light_height, lz - hs),
                     (lx + hs, light_height, lz + hs), (lx - hs, light_height, lz + hs))
        b.add(v, t, len(mats) - 1)
        lights.append(point_light((lx, light_height - 0.001, lz), le, light_size * light_size))
    v, t, inst = b.arrays()
    cam = Camera(position=(0.0, 0.55 * half + 6.0, half + 0.45 * half), target=(0.0, 0.0, 0.1 * half),
                 fov_deg=50.0)
    return Scene(v, t, inst, np.array(mats), np.array(lights),
                 (environment, environment, environment), cam, f"sphere_field_{grid}").contiguous()


def dynamic_sphere_field(grid: int = 64, n_lat: int = 15, n_lon: int = 18, seed: int = 4) -> Scene:
    """The sphere field as dynamic-transform instances: every sphere is an
    instance of one local mesh (a displaced unit sphere) with its own
    translation, rotation and scale, as the reference's scene conversion emits
    physics-driven entities; a static ground plane.  grid 64: 4096 instances,
    2,064,384 sphere triangles."""
    st = Stream(seed)
    dirs, tris = _displaced_unit_sphere_mesh(n_lat, n_lon, 0.05, seed * 17)
    nt = tris.shape[0]
    spacing, half = 3.0, 0.5 * (grid - 1) * 3.0
    mats, inst, inst_local, inst_tr = [], [], [], []
    for gy in range(grid):
        for gx in range(grid):
            r = st.uniform(0.7, 1.0)
            a = st.uniform(0.0, 2.0 * math.pi)
            t = (gx * spacing - half, r, gy * spacing - half)
            mats.append(material(albedo=tuple(st.uniform(0.05, 0.9) for _ in range(3)),
                                 roughness=(1.0, 0.3, 0.0)[st.randint(0, 2)], model=(0, 3, 2)[st.randint(0, 2)]))
            inst.append((len(inst) * nt, nt, len(mats) - 1))
            inst_local.append((1, 0, dirs.shape[0], 0, 3 * nt))
            inst_tr.append(t + (0.0, math.sin(a / 2), 0.0, math.cos(a / 2)) + (r, r, r))
    # global arrays: the world-space copies (used only where a local index is out of range)
    glob_v = np.concatenate([dirs * tr[7] + np.array(tr[0:3]) for tr in inst_tr]).astype(np.float32)
    glob_t = np.concatenate([tris + k * dirs.shape[0] for k in range(len(inst_tr))]).astype(np.uint32)
    mats.append(material(albedo=(0.5, 0.5, 0.5), roughness=1.0))
    g = half + 6.0
    gv, gt = _quad((-g, 0.0, -g), (-g, 0.0, g), (g, 0.0, g), (g, 0.0, -g))
    inst.append((glob_t.shape[0], gt.shape[0], len(mats) - 1))
    inst_local.append((0, 0, 0, 0, 0))
    inst_tr.append((0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 1.0, 1.0, 1.0))
    v = np.concatenate([glob_v, np.asarray(gv, np.float32)])
    t = np.concatenate([glob_t, np.asarray(gt, np.uint32) + glob_v.shape[0]])
    lights = [point_light((0.0, 14.0, 0.0), (1.0, 0.95, 0.9), 400.0)]
    cam = Camera(position=(0.0, 0.55 * half + 6.0, 1.45 * half), target=(0.0, 0.0, 0.1 * half), fov_deg=50.0)
    return Scene(v, t, np.array(inst, np.uint32), np.array(mats), np.array(lights), (0.1, 0.1, 0.1), cam,
                 f"dynamic_sphere_field_{grid}", instance_local=np.array(inst_local, np.uint32),
                 instance_transforms=np.array(inst_tr, np.float32), local_vertices=dirs.astype(np.float32),
                 local_indices=tris.astype(np.uint32).reshape(-1)).contiguous()


def sky_map(width: int = 128, height: int = 64, seed: int = 2, sun_dir=(0.4, 0.55, -0.73),
            sun_radiance: float = 40.0) -> np.ndarray:
    """Equirectangular sky, (height, width, 3) float32, row 0 toward +y, in the
    reference's mapping (u = 0.5 + atan2(z, x) / 2pi, v = acos(y) / pi): a blue
    gradient, a warm horizon, a darker ground, seeded value-noise clouds and a
    small bright sun."""
    v = (np.arange(height, dtype=np.float64) + 0.5) / height
    u = (np.arange(width, dtype=np.float64) + 0.5) / width
    theta = v[:, None] * math.pi
    phi = (u[None, :] - 0.5) * 2.0 * math.pi
    y = np.cos(theta) * np.ones_like(phi)
    x = np.sin(theta) * np.cos(phi)
    z = np.sin(theta) * np.sin(phi)
    up = np.clip(y, 0.0, 1.0)[..., None]
    sky = (1.0 - up) * np.array([1.0, 0.75, 0.5]) + up * np.array([0.25, 0.45, 0.95])
    ground = np.array([0.18, 0.15, 0.12]) * np.ones_like(sky)
    img = np.where((y >= 0.0)[..., None], sky, ground)
    pts = np.stack([x, y, z], axis=-1).reshape(-1, 3) * 3.0
    cloud = value_noise(pts, 4, seed).reshape(height, width)
    cloud = np.clip((cloud - 0.55) * 3.0, 0.0, 1.0) * (y > 0.05)
    img = img * (1.0 - 0.6 * cloud[..., None]) + 0.9 * cloud[..., None]
    sd = np.asarray(sun_dir, np.float64)
    sd = sd / np.linalg.norm(sd)
    cosang = x * sd[0] + y * sd[1] + z * sd[2]
    img = img + (cosang > 0.995)[..., None] * sun_radiance * np.array([1.0, 0.9, 0.7])
    return np.ascontiguousarray(img, np.float32)


def sky_scene(seed: int = 3, grid: int = 4) -> Scene:
    """Displaced spheres (Lambert, glossy, mirror) on a ground plane under the
    sky map, one sun-like point light for next-event estimation."""
    sc = sphere_field(grid, 14, 18, seed=seed, n_lights=1, light_size=0.5, light_height=12.0)
    sc.env_map = sky_map(seed=seed)
    sc.env_scale = (1.0, 1.0, 1.0)
    sc.name = "sky_scene"
    return sc


def sphere_grid(seed: int = 4, grid: int = 64) -> Scene:
    """64x64 displaced spheres of 2*14*18 = 504 triangles: 2,064,386 triangles with lights and ground."""
    return sphere_field(grid, 15, 18, seed)


def sphere_grid_settings(width=1920, height=1080, spp=64) -> RenderSettings:
    return RenderSettings(width=width, height=height, spp=spp, max_depth=16, seed=1234,
                          enable_nee=True, enable_mis=True, firefly_clamp=10.0)


# ---------------------------------------------------------------- batched jobs
@dataclasses.dataclass
class Job:
    scene: Scene
    settings: RenderSettings
    target_triangles: int


def _log_uniform(st: Stream, lo: float, hi: float) -> float:
    return math.exp(st.uniform(math.log(lo), math.log(hi)))


def batch_jobs(count: int = 64, seed: int = 5, max_triangles: int = 500_000, max_side: int = 1024,
               min_triangles: int = 1_000, min_side: int = 128) -> List[Job]:
    """Uneven render jobs: triangle count log-uniform in [min,max], square side
    log-uniform in [min_side,max_side], spp in {4,8,16,32,64}, depth in {4,8,16},
    the sphere-field material mix; each job's seeds derive from the master seed.
    No firefly clamp (the batched workload takes only the full frame's
    material mix, and the reference has no clamp), so every job renders what
    the reference's CPU tracer renders for the same scene and settings."""
    st = Stream(seed)
    jobs = []
    for k in range(count):
        tris = _log_uniform(st, min_triangles, max_triangles)
        side = int(round(_log_uniform(st, min_side, max_side)))
        spp = [4, 8, 16, 32, 64][st.randint(0, 4)]
        depth = [4, 8, 16][st.randint(0, 2)]
        job_seed = st.next_u64() & 0xFFFFFFFF
        # Choose sphere resolution and grid so grid^2 * 2*(n_lat-1)*n_lon ~ tris.
        n_lat, n_lon = 15, 18
        per = 2 * (n_lat - 1) * n_lon
        grid = max(1, int(round(math.sqrt(tris / per))))
        if grid * grid * per > max_triangles * 1.2:
            grid = max(1, grid - 1)
        grid = max(grid, int(math.ceil(math.sqrt(min_triangles / per))))
        scene = sphere_field(grid, n_lat, n_lon, job_seed % 100000 + 7, n_lights=min(16, max(1, grid)),
                             light_size=max(1.0, 0.1 * grid * 3.0), light_height=max(4.0, 0.25 * grid * 3.0))
        settings = RenderSettings(width=side, height=side, spp=spp, max_depth=depth, seed=job_seed,
                                  enable_nee=True, enable_mis=True)
        jobs.append(Job(scene, settings, int(tris)))
    return jobs


# -------------------------------------------------------- inverse rendering
def inverse_box_scene(params: Optional[np.ndarray] = None, seed: int = 6, n_objects: int = 16) -> Scene:
    """Box room + n_objects seeded boxes (12 tris each).  params is the (n_objects,4)
    vector of per-object RGB albedo and roughness; None draws the held-out
    target parameters U[0.1,0.8]."""
    st = Stream(seed)
    b = _Builder()
    mats: list = []
    lights: list = []
    _room(b, mats, Stream(seed + 1000))
    if params is None:
        pst = Stream(seed + 2000)
        params = np.array([[pst.uniform(0.1, 0.8) for _ in range(4)] for _ in range(n_objects)], np.float32)
    params = np.asarray(params, np.float32).reshape(n_objects, 4)
    for k in range(n_objects):
        cx = st.uniform(-0.38, 0.38)
        cz = st.uniform(-0.38, 0.38)
        hy = st.uniform(0.03, 0.12)
        hx = st.uniform(0.03, 0.07)
        hz = st.uniform(0.03, 0.07)
        cy = st.uniform(hy, 0.7)
        yaw = st.uniform(-30.0, 30.0)
        mats.append(material(albedo=tuple(params[k, :3]), roughness=float(params[k, 3]), model=3, ior=1.5))
        v, t = _box((cx, cy, cz), (hx, hy, hz), yaw)
        b.add(v, t, len(mats) - 1)
    _ceiling_light(b, mats, lights)
    v, t, inst = b.arrays()
    cam = Camera(position=(0.0, 0.5, 1.9), target=(0.0, 0.5, 0.0), up=(0.0, 1.0, 0.0), fov_deg=40.0)
    return Scene(v, t, inst, np.array(mats), np.array(lights), (0.0, 0.0, 0.0), cam, "inverse_box").contiguous()


def inverse_settings(width=128, height=128, spp=32) -> RenderSettings:
    return RenderSettings(width=width, height=height, spp=spp, max_depth=6, seed=4321,
                          enable_nee=True, enable_mis=True)
