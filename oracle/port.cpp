// port.cpp -- TEST INFRASTRUCTURE: CPU restatement of the reference's render hot path.
//
// A line-by-line restatement (own code, same floating-point operation order)
// of the reference's scalar CPU tracer, used as the checker wherever the
// reference sources are not available (the GPU box).  It is pinned
// bit-for-bit against the reference itself (oracle/_ref/libvkptref.so) by
// tests/test_oracle_pin.py: identical films, counters, BVH nodes and hit ids.
// The product library never links this file.
//
// Followed, function by function (paths within the reference project):
//   splitmix64, Rng                 src/pathtracer/ScalarCpuPathTracer.cpp:36-41, 383-393
//   compute_camera_basis            src/pathtracer/ScalarCpuPathTracer.cpp:139-152
//   camera_rays                     src/pathtracer/ScalarCpuPathTracer.Render.cpp:55-119
//   shade_pixel                     src/pathtracer/ScalarCpuPathTracer.Render.cpp:228-284
//   trace                           src/pathtracer/ScalarCpuPathTracer.cpp:1148-1289
//   sample_direct_light             src/pathtracer/ScalarCpuPathTracer.cpp:1022-1118
//   light_pdf_for_direction, Mis    src/pathtracer/ScalarCpuPathTracer.cpp:1120-1146
//   sample_hemisphere / phong lobe  src/pathtracer/ScalarCpuPathTracer.cpp:978-1020
//   apply_material_effect           src/pathtracer/ScalarCpuPathTracer.cpp:186-355
//   schlick_fresnel, refract_dir    src/pathtracer/ScalarCpuPathTracer.cpp:357-377
//   accelerator build / intersect   src/pathtracer/CpuBvhAccelerator.cpp:84-154, 161-263, 360-477
//   midpoint BVH builder            src/cpu/ParallelBvhBuilder.cpp:13-257
//   leaf triangle batch             src/cpu/BvhTriangleIntersector.cpp:25-74, 186-209
//   FilmBuffer::add_sample          src/pathtracer/FilmBuffer.cpp:80-91
//   SDF primitives: rotate_x/y/z, rotate_euler(_inv), divide_by_scale
//                                   src/pathtracer/ScalarCpuPathTracer.cpp:113-159
//     sdf_distance, sdf_normal      src/pathtracer/ScalarCpuPathTracer.cpp:808-853
//     intersect_sphere, the march   src/pathtracer/ScalarCpuPathTracer.cpp:855-930
//     nearest-hit reduction         src/pathtracer/ScalarCpuPathTracer.Intersect.cpp:91-129
//   dynamic-instance flattening     src/pathtracer/CpuBvhAccelerator.cpp:47-74, 173-247
//   instance transform refit        src/pathtracer/CpuBvhAccelerator.cpp:265-358, 527-606
//   ApplyFilmResolve, WhiteBalanceScale, ColorTemperatureToRgb
//                                   src/pathtracer/FilmBuffer.cpp:30-49, 216-224, 253-325

#include "vkpt_oracle.h"
#include "worker_pool.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

namespace {

thread_local std::string g_error;
thread_local std::vector<vko_instance_update> g_updates;
int fail(const std::string& m) { g_error = m; return 1; }

constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.31830988618f;
constexpr float kEps = 1e-4f;

struct V3 { float x, y, z; };
inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 neg(V3 a) { return {-a.x, -a.y, -a.z}; }
inline V3 mul(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 mulv(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline V3 divs(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline float fmax_std(float a, float b) { return (a < b) ? b : a; }   // std::max
inline float fmin_std(float a, float b) { return (b < a) ? b : a; }   // std::min
inline float clampf(float v, float lo, float hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }
// normalize(): division by the length, (0,1,0) below 1e-4.
inline V3 unit(V3 v) {
  const float l = std::sqrt(dot(v, v));
  if (l <= kEps) return {0.0f, 1.0f, 0.0f};
  return divs(v, l);
}
inline float clamp01(float v) {
  if (!std::isfinite(v)) return 0.0f;
  return fmin_std(1.0f, fmax_std(0.0f, v));
}
inline float pow5(float v) { const float v2 = v * v; return v2 * v2 * v; }

// ---- procedural material effects (ScalarCpuPathTracer.cpp:186-355) ----------
// hash01: fract(sin(dot(p, k) + seed * k4) * 43758.5453).
inline float fx_hash(float x, float y, float z, float seed) {
  const float v = std::sin(x * 12.9898f + y * 78.233f + z * 37.719f + seed * 19.19f) * 43758.5453f;
  return v - std::floor(v);
}
inline float fx_smooth(float e0, float e1, float x) {
  const float t = clamp01((x - e0) / fmax_std(1.0e-6f, e1 - e0));
  return t * t * (3.0f - 2.0f * t);
}
inline V3 fx_lin(V3 a, float sa, V3 b, float sb) { return add(mul(a, sa), mul(b, sb)); }

// Wood species 16..19 (16 plain, 17 parquet, 18 walnut, 19 sandalwood).
inline V3 fx_wood(V3 base, V3 p, float roughness, float clearcoat, uint32_t style) {
  const float rough = clamp01(roughness), coat = clamp01(clearcoat);
  const float polish = clamp01(coat * (1.25f - rough * 0.75f));
  const float par = style == 17u ? 1.0f : 0.0f, wal = style == 18u ? 1.0f : 0.0f, san = style == 19u ? 1.0f : 0.0f;
  const float pw = 0.40f + 0.16f * par + 0.08f * polish - 0.18f * wal;
  const float pl = 1.15f + 0.85f * par + 0.55f * polish - 0.55f * wal;
  const float u = (p.x + san * p.y * 0.35f) / fmax_std(0.12f, pw);
  const float v = (p.z + wal * p.y * 0.70f + san * p.x * 0.22f) / fmax_std(0.30f, pl);
  const float cu = std::floor(u), cv = std::floor(v);
  const float lu = u - cu, lv = v - cv;
  const float seed = fx_hash(cu, cv, 0.0f, 16.0f);
  const float macro = fx_hash(std::floor(p.x * 3.7f), std::floor(p.y * 3.7f), std::floor(p.z * 3.7f),
                              31.0f + static_cast<float>(style));
  const float micro = fx_hash(std::floor(p.x * 34.0f), std::floor(p.y * 34.0f), std::floor(p.z * 34.0f),
                              47.0f + static_cast<float>(style));
  const bool rot = par > 0.5f && std::fmod(cu + cv, 2.0f) >= 1.0f;
  const float along = rot ? lv : lu, across = rot ? lu : lv;
  const float wobble = (macro - 0.5f) * (0.06f + rough * 0.12f + wal * 0.08f + san * 0.04f);
  const float wa = along + wobble + std::sin(across * 6.0f + seed * 5.0f) * 0.018f;
  const float freq = 12.0f + rough * 8.0f + wal * 22.0f + san * 36.0f;
  const float wave = std::sin((wa * freq + seed * 6.2831853f) +
                              std::sin(across * (6.0f + rough * 8.0f) + seed * 4.0f) *
                                  (0.25f + rough * 0.45f + wal * 0.45f));
  const float fine = std::sin(wa * (55.0f + rough * 55.0f + san * 110.0f) + across * (9.0f + wal * 25.0f) +
                              seed * 12.0f);
  const float fw = 0.10f + rough * 0.18f + wal * 0.18f + san * 0.22f;
  const float ring = fx_smooth(-0.35f + polish * 0.18f, 0.82f, wave) * (1.0f - fw) + (0.5f + 0.5f * fine) * fw;
  const float su = fmin_std(lu, 1.0f - lu), sv = fmin_std(lv, 1.0f - lv);
  const float seam = (1.0f - san) * (1.0f - fx_smooth(0.0f, 0.028f + polish * 0.018f, fmin_std(su, sv)));
  const V3 dark = mul(base, 0.46f - rough * 0.10f - wal * 0.18f);
  const V3 amber = add(mul(base, 1.14f + coat * 0.22f + san * 0.18f),
                       V3{0.08f + san * 0.18f, 0.055f + san * 0.06f, 0.025f});
  V3 wood = fx_lin(dark, 1.0f - ring, amber, ring);
  const float tint = 0.92f + (0.08f + wal * 0.12f + san * 0.06f) * seed + (macro - 0.5f) * (0.08f + rough * 0.06f);
  const float pores = fx_smooth(0.74f - wal * 0.08f, 1.0f, micro) *
                      (0.025f + rough * 0.055f + wal * 0.055f + san * 0.018f);
  wood = mul(wood, tint);
  wood = mul(wood, 1.0f - pores);
  wood = mul(wood, 1.0f - seam * (0.10f + rough * 0.35f + par * 0.18f) * (1.0f - coat * 0.45f));
  const float mix = 0.30f + rough * 0.34f - polish * 0.14f + wal * 0.26f + san * 0.18f;
  return fx_lin(base, 1.0f - mix, wood, mix);
}
inline V3 ld3(const float* p) { return {p[0], p[1], p[2]}; }

uint64_t mix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ULL;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}

struct Stream {
  uint64_t s;
  // key order: seed, frame, sample, path_id, dimension, depth, pixel
  Stream(uint64_t seed, uint64_t frame, uint64_t sample, uint64_t path_id, uint64_t dim, uint64_t depth,
         uint64_t pixel) {
    const uint64_t m = mix64(seed ^ mix64(frame) ^ mix64(sample) ^ mix64(path_id) ^ mix64(dim) ^ mix64(depth));
    s = mix64(m + mix64(pixel));
  }
  float u() {
    s = mix64(s);
    return static_cast<float>((s >> 8) & 0x00ffffffu) * (1.0f / 16777215.0f);
  }
};

struct Material {
  V3 albedo, emissive;
  float roughness, metallic, ior, transmission, clearcoat, sheen, alpha;
  uint32_t model, effect;
  bool emissive_any() const { return emissive.x > 0.0f || emissive.y > 0.0f || emissive.z > 0.0f; }
};

struct Light {
  V3 pos, color, dir;
  float intensity, radius, inner, outer;
};

struct Prim {
  uint32_t material, index;
  V3 v0, e1, e2, n;
  V3 v1, v2;   // the other two vertices as given (the watertight test reads vertices, not edges)
};

// Triangle test of every traversal: 0 = the reference's Moller-Trumbore
// (BvhTriangleIntersector.cpp:35-74), 1 = watertight (an extension the
// reference does not have; see wt_test).
int g_triangle_test = 0;

// The watertight ray/triangle test of Woop, Benthin and Wald ("Watertight
// Ray/Triangle Intersection", JCGT 2(1), 2013), without back-face culling:
// shear the ray onto +z along its dominant axis (the first largest |d| on
// ties, the other two axes swapped when d[kz] < 0), take the three 2D edge
// functions of the sheared vertices (redone in double when one rounds to
// exactly 0), reject mixed signs and a zero determinant, and return
// t = T / det (-1 on a miss).
struct WtRay {
  int kx, ky, kz;
  float sx, sy, sz;
};

inline float axis_of(V3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

WtRay prep_wt(V3 d) {
  const float ax = std::fabs(d.x), ay = std::fabs(d.y), az = std::fabs(d.z);
  int kz = 0;
  float m = ax;
  if (ay > m) {
    kz = 1;
    m = ay;
  }
  if (az > m) kz = 2;
  int kx = kz == 2 ? 0 : kz + 1;
  int ky = kx == 2 ? 0 : kx + 1;
  const float dz = axis_of(d, kz);
  if (dz < 0.0f) std::swap(kx, ky);
  return WtRay{kx, ky, kz, axis_of(d, kx) / dz, axis_of(d, ky) / dz, 1.0f / dz};
}

float wt_test(const Prim& p, V3 o, const WtRay& w) {
  const V3 a{p.v0.x - o.x, p.v0.y - o.y, p.v0.z - o.z};
  const V3 b{p.v1.x - o.x, p.v1.y - o.y, p.v1.z - o.z};
  const V3 c{p.v2.x - o.x, p.v2.y - o.y, p.v2.z - o.z};
  const float akz = axis_of(a, w.kz), bkz = axis_of(b, w.kz), ckz = axis_of(c, w.kz);
  const float Ax = axis_of(a, w.kx) - w.sx * akz, Ay = axis_of(a, w.ky) - w.sy * akz;
  const float Bx = axis_of(b, w.kx) - w.sx * bkz, By = axis_of(b, w.ky) - w.sy * bkz;
  const float Cx = axis_of(c, w.kx) - w.sx * ckz, Cy = axis_of(c, w.ky) - w.sy * ckz;
  float U = Cx * By - Cy * Bx;
  float V = Ax * Cy - Ay * Cx;
  float W = Bx * Ay - By * Ax;
  if (U == 0.0f || V == 0.0f || W == 0.0f) {
    U = static_cast<float>(static_cast<double>(Cx) * By - static_cast<double>(Cy) * Bx);
    V = static_cast<float>(static_cast<double>(Ax) * Cy - static_cast<double>(Ay) * Cx);
    W = static_cast<float>(static_cast<double>(Bx) * Ay - static_cast<double>(By) * Ax);
  }
  if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return -1.0f;
  const float det = U + V + W;
  if (det == 0.0f) return -1.0f;
  const float Az = w.sz * akz, Bz = w.sz * bkz, Cz = w.sz * ckz;
  const float T = U * Az + V * Bz + W * Cz;
  return T / det;
}

struct Box { float lo[3], hi[3]; };
struct Node { Box box; int32_t left, right, first, count; };

struct Stats {
  uint64_t tri_tests = 0, tri_hits = 0, nodes = 0, leaves = 0, shadow = 0;
  uint64_t sdf_tests = 0, sdf_steps = 0, sdf_hits = 0, sdf_misses = 0;
};

// ------------------------------------------------------------ SDF primitives
struct Sdf {
  uint32_t shape, material;   // shape 0..5 (sphere, box, rounded box, plane, torus, capsule)
  V3 pos, scale, rot;
  float radius, pa, pb;
};

// Rotation about one axis by `a` radians, the sine and cosine taken per call.
inline V3 turn_x(V3 v, float a) { const float s = std::sin(a), c = std::cos(a); return {v.x, c * v.y - s * v.z, s * v.y + c * v.z}; }
inline V3 turn_y(V3 v, float a) { const float s = std::sin(a), c = std::cos(a); return {c * v.x + s * v.z, v.y, -s * v.x + c * v.z}; }
inline V3 turn_z(V3 v, float a) { const float s = std::sin(a), c = std::cos(a); return {c * v.x - s * v.y, s * v.x + c * v.y, v.z}; }
inline V3 unscale(V3 v, V3 s) {
  return {v.x / (s.x != 0.0f ? s.x : 1.0f), v.y / (s.y != 0.0f ? s.y : 1.0f), v.z / (s.z != 0.0f ? s.z : 1.0f)};
}
// World vector -> primitive space: inverse Euler rotation (x, y, z order), then 1/scale.
inline V3 sdf_local(const Sdf& p, V3 v) {
  return unscale(turn_z(turn_y(turn_x(v, -p.rot.x), -p.rot.y), -p.rot.z), p.scale);
}
inline float vlen(V3 v) { return std::sqrt(dot(v, v)); }

float sdf_value(const Sdf& p, V3 w) {
  const V3 l = sdf_local(p, sub(w, p.pos));
  switch (p.shape) {
    case 0: return vlen(l) - p.radius;
    case 1: {
      const V3 q{std::fabs(l.x) - p.scale.x, std::fabs(l.y) - p.scale.y, std::fabs(l.z) - p.scale.z};
      const V3 m{fmax_std(0.0f, q.x), fmax_std(0.0f, q.y), fmax_std(0.0f, q.z)};
      return vlen(m) + fmin_std(fmax_std(q.x, fmax_std(q.y, q.z)), 0.0f);
    }
    case 2: {
      const V3 q{std::fabs(l.x) - p.scale.x + p.pa, std::fabs(l.y) - p.scale.y + p.pa, std::fabs(l.z) - p.scale.z + p.pa};
      const V3 m{fmax_std(0.0f, q.x), fmax_std(0.0f, q.y), fmax_std(0.0f, q.z)};
      return vlen(m) + fmin_std(fmax_std(q.x, fmax_std(q.y, q.z)), 0.0f) - p.pa;
    }
    case 3: return l.y + p.pb;
    case 4: {
      const float ring = fmax_std(0.05f, p.pa), tube = fmax_std(0.02f, p.radius);
      const float qx = vlen(V3{l.x, 0.0f, l.z}) - ring;
      return vlen(V3{qx, l.y, 0.0f}) - tube;
    }
    default: {
      const V3 a{0.0f, -p.pa, 0.0f}, b{0.0f, p.pa, 0.0f};
      const V3 ab = sub(b, a);
      const float s = dot(sub(l, a), ab) / fmax_std(kEps, dot(ab, ab));
      const float c = fmax_std(0.0f, fmin_std(1.0f, s));
      return vlen(sub(l, add(a, mul(ab, c)))) - p.radius;
    }
  }
}

// Closest intersection of one primitive; t is the caller's (0 on entry).
bool sdf_hit(const Sdf& p, V3 o, V3 d, float& t, V3& n, Stats& st) {
  ++st.sdf_tests;
  if (p.shape == 0u) {   // analytic sphere
    ++st.sdf_steps;
    const float r = fmax_std(0.01f, p.radius);
    const V3 lo = sdf_local(p, sub(o, p.pos)), ld = sdf_local(p, d);
    const float a = dot(ld, ld);
    if (a <= kEps * kEps) { ++st.sdf_misses; return false; }
    const float hb = dot(lo, ld);
    const float c = dot(lo, lo) - r * r;
    const float disc = hb * hb - a * c;
    if (disc < 0.0f) { ++st.sdf_misses; return false; }
    const float root = std::sqrt(disc);
    float cand = (-hb - root) / a;
    if (cand <= kEps) cand = (-hb + root) / a;
    if (cand <= kEps || !std::isfinite(cand)) { ++st.sdf_misses; return false; }
    t = cand;
    const V3 ln = unscale(unit(add(lo, mul(ld, t))), p.scale);
    n = unit(turn_x(turn_y(turn_z(ln, p.rot.z), p.rot.y), p.rot.x));
    ++st.sdf_hits;
    return true;
  }
  for (uint32_t i = 0; i < 192u; ++i) {   // sphere tracing
    ++st.sdf_steps;
    const V3 x = add(o, mul(d, t));
    const float dist = sdf_value(p, x);
    if (dist <= kEps) {
      const float e = 0.0005f;
      const float gx = sdf_value(p, add(x, V3{e, 0.0f, 0.0f})) - sdf_value(p, sub(x, V3{e, 0.0f, 0.0f}));
      const float gy = sdf_value(p, add(x, V3{0.0f, e, 0.0f})) - sdf_value(p, sub(x, V3{0.0f, e, 0.0f}));
      const float gz = sdf_value(p, add(x, V3{0.0f, 0.0f, e})) - sdf_value(p, sub(x, V3{0.0f, 0.0f, e}));
      n = unit(mul(V3{gx, gy, gz}, 0.5f));
      ++st.sdf_hits;
      return true;
    }
    t += fmax_std(1.0e-3f, dist);
    if (t > 10000.0f) break;
  }
  ++st.sdf_misses;
  return false;
}

// ----------------------------------------------------------------- BVH build
struct Builder {
  const std::vector<Box>* boxes;
  std::vector<Node>* nodes;
  std::vector<uint32_t>* order;
  int32_t next = 1;
  bool stable = true;
  size_t leaf = 4;

  static float centroid(const Box& b, int ax) { return 0.5f * (b.lo[ax] + b.hi[ax]); }

  void build(int32_t id, uint32_t* idx, size_t n) {
    Box bb;
    Box cb;
    for (int a = 0; a < 3; ++a) {
      bb.lo[a] = cb.lo[a] = std::numeric_limits<float>::max();
      bb.hi[a] = cb.hi[a] = -std::numeric_limits<float>::max();
    }
    for (size_t i = 0; i < n; ++i) {
      const Box& p = (*boxes)[idx[i]];
      for (int a = 0; a < 3; ++a) {
        bb.lo[a] = fmin_std(bb.lo[a], p.lo[a]);
        bb.hi[a] = fmax_std(bb.hi[a], p.hi[a]);
      }
    }
    (*nodes)[id].box = bb;
    if (n <= leaf) {
      Node& nd = (*nodes)[id];
      nd.left = nd.right = -1;
      nd.first = static_cast<int32_t>(idx - order->data());
      nd.count = static_cast<int32_t>(n);
      return;
    }
    for (size_t i = 0; i < n; ++i) {
      const Box& p = (*boxes)[idx[i]];
      for (int a = 0; a < 3; ++a) {
        const float c = centroid(p, a);
        cb.lo[a] = fmin_std(cb.lo[a], c);
        cb.hi[a] = fmax_std(cb.hi[a], c);
      }
    }
    int axis = 0;
    float ext = cb.hi[0] - cb.lo[0];
    for (int a = 1; a < 3; ++a) {
      const float e = cb.hi[a] - cb.lo[a];
      if (e > ext) { ext = e; axis = a; }
    }
    const float split = 0.5f * (cb.lo[axis] + cb.hi[axis]);
    auto pred = [&](uint32_t k) { return centroid((*boxes)[k], axis) < split; };
    uint32_t* mid = stable ? std::stable_partition(idx, idx + n, pred) : std::partition(idx, idx + n, pred);
    size_t nl = static_cast<size_t>(mid - idx);
    if (nl == 0 || nl == n) nl = n / 2;
    const int32_t l = next++;
    const int32_t r = next++;
    Node& nd = (*nodes)[id];
    nd.left = l;
    nd.right = r;
    nd.first = -1;
    nd.count = 0;
    build(l, idx, nl);
    build(r, idx + nl, n - nl);
  }
};

// --------------------------------------------------------------- the scene
struct World {
  std::vector<Prim> prims;
  std::vector<Box> boxes;
  std::vector<Node> nodes;
  std::vector<uint32_t> order;
  std::vector<Material> mats;
  std::vector<Light> lights;
  V3 env{};
  std::vector<V3> env_map;   // equirectangular texels, row-major (empty: constant environment)
  uint32_t env_w = 0, env_h = 0;
  V3 env_scale{1.0f, 1.0f, 1.0f};
  std::vector<Sdf> sdfs;
  V3 cam_pos{}, cam_fwd{}, cam_right{}, cam_up{};

  // SampleSceneEnvironment (src/pathtracer/PathTracer.cpp:213-272).
  V3 environment(V3 d) const {
    if (env_map.empty()) return env;
    const float len_sq = d.x * d.x + d.y * d.y + d.z * d.z;
    if (len_sq <= 1.0e-12f) return env;
    const float inv_len = 1.0f / std::sqrt(len_sq);
    const V3 dir{d.x * inv_len, d.y * inv_len, d.z * inv_len};
    float u = 0.5f + std::atan2(dir.z, dir.x) * 0.15915494309189533577f;
    u -= std::floor(u);
    const float v = std::acos(clampf(dir.y, -1.0f, 1.0f)) * 0.31830988618379067154f;
    const float x = u * static_cast<float>(env_w);
    const float y = clampf(v, 0.0f, 1.0f) * static_cast<float>(env_h - 1u);
    const uint32_t x0 = static_cast<uint32_t>(std::floor(x)) % env_w, x1 = (x0 + 1u) % env_w;
    const uint32_t y0 = static_cast<uint32_t>(std::floor(y)), y1 = std::min(y0 + 1u, env_h - 1u);
    const float tx = x - std::floor(x), ty = y - std::floor(y);
    auto at = [&](uint32_t px, uint32_t py) { return env_map[static_cast<size_t>(py) * env_w + px]; };
    const V3 c00 = at(x0, y0), c10 = at(x1, y0), c01 = at(x0, y1), c11 = at(x1, y1);
    const V3 top{c00.x + (c10.x - c00.x) * tx, c00.y + (c10.y - c00.y) * tx, c00.z + (c10.z - c00.z) * tx};
    const V3 bot{c01.x + (c11.x - c01.x) * tx, c01.y + (c11.y - c01.y) * tx, c01.z + (c11.z - c01.z) * tx};
    V3 c{top.x + (bot.x - top.x) * ty, top.y + (bot.y - top.y) * ty, top.z + (bot.z - top.z) * ty};
    c.x *= env_scale.x;
    c.y *= env_scale.y;
    c.z *= env_scale.z;
    return c;
  }
  float fov = 60.0f;
  float aperture = 0.0f, focus = 0.0f;
  uint32_t iris_blades = 0u;
  float iris_rotation = 0.0f, iris_roundness = 1.0f, squeeze = 1.0f;

  // transform_instance_vertex: scale, rotate by the normalized quaternion, translate.
  static V3 instance_vertex(V3 l, const float* t) {
    const V3 sc{l.x * t[7], l.y * t[8], l.z * t[9]};
    const float len_sq = t[3] * t[3] + t[4] * t[4] + t[5] * t[5] + t[6] * t[6];
    V3 r = sc;
    if (!(len_sq <= kEps * kEps)) {
      const float inv = 1.0f / std::sqrt(len_sq);
      const V3 q{t[3] * inv, t[4] * inv, t[5] * inv};
      const float qw = t[6] * inv;
      const V3 tt = mul(cross(q, sc), 2.0f);
      r = add(add(sc, mul(tt, qw)), cross(q, tt));
    }
    return add(r, V3{t[0], t[1], t[2]});
  }

  const vko_scene* src = nullptr;
  std::vector<uint32_t> inst_first, inst_count;   // flattened primitive range per instance

  void load(const vko_scene& s, bool stable = true, size_t leaf = 4) {
    src = &s;
    const bool dyn = s.instance_local && s.instance_transforms;
    for (uint32_t i = 0; i < s.instance_count; ++i) {
      inst_first.push_back(static_cast<uint32_t>(prims.size()));
      const uint32_t first = s.instances[3 * i], count = s.instances[3 * i + 1], mat = s.instances[3 * i + 2];
      const uint32_t* loc = dyn ? s.instance_local + 5 * i : nullptr;
      const bool use_local = loc && (loc[0] & 1u) && loc[2] > 0u && loc[4] > 0u;
      for (uint32_t k = 0; k < count; ++k) {
        V3 v0{}, v1{}, v2{};
        bool loaded = false;
        if (use_local) {
          const uint32_t lb = loc[3] + k * 3u, le = loc[1] + loc[2];
          if (lb < 0xFFFFFFFEu && lb + 2u < s.local_index_count) {
            const uint32_t a = loc[1] + s.local_indices[lb], b = loc[1] + s.local_indices[lb + 1],
                           c = loc[1] + s.local_indices[lb + 2];
            if (a < le && b < le && c < le && a < s.local_vertex_count && b < s.local_vertex_count &&
                c < s.local_vertex_count) {
              const float* t = s.instance_transforms + 10 * i;
              v0 = instance_vertex(ld3(s.local_vertices + 3 * a), t);
              v1 = instance_vertex(ld3(s.local_vertices + 3 * b), t);
              v2 = instance_vertex(ld3(s.local_vertices + 3 * c), t);
              loaded = true;
            }
          }
        }
        if (!loaded) {
          const uint32_t base = (first + k) * 3u;
          if (base >= 0xFFFFFFFEu || base + 2u >= s.index_count) continue;
          const uint32_t a = s.indices[base], b = s.indices[base + 1], c = s.indices[base + 2];
          if (a >= s.vertex_count || b >= s.vertex_count || c >= s.vertex_count) continue;
          v0 = ld3(s.vertices + 3 * a);
          v1 = ld3(s.vertices + 3 * b);
          v2 = ld3(s.vertices + 3 * c);
        }
        Box bx;
        bx.lo[0] = std::min({v0.x, v1.x, v2.x}) - kEps;
        bx.lo[1] = std::min({v0.y, v1.y, v2.y}) - kEps;
        bx.lo[2] = std::min({v0.z, v1.z, v2.z}) - kEps;
        bx.hi[0] = std::max({v0.x, v1.x, v2.x}) + kEps;
        bx.hi[1] = std::max({v0.y, v1.y, v2.y}) + kEps;
        bx.hi[2] = std::max({v0.z, v1.z, v2.z}) + kEps;
        Prim p;
        p.material = mat;
        p.index = static_cast<uint32_t>(prims.size());
        p.v0 = v0;
        p.v1 = v1;
        p.v2 = v2;
        p.e1 = sub(v1, v0);
        p.e2 = sub(v2, v0);
        // normalize_vec3 of the accelerator: multiply by 1/sqrt(len^2).
        const V3 cr = cross(p.e1, p.e2);
        const float l2 = dot(cr, cr);
        p.n = (l2 <= kEps * kEps) ? V3{0.0f, 1.0f, 0.0f} : mul(cr, 1.0f / std::sqrt(l2));
        prims.push_back(p);
        boxes.push_back(bx);
      }
      inst_count.push_back(static_cast<uint32_t>(prims.size()) - inst_first.back());
    }
    if (!prims.empty()) {
      nodes.assign(2 * prims.size() - 1, Node{});
      order.resize(prims.size());
      std::iota(order.begin(), order.end(), 0u);
      Builder b{&boxes, &nodes, &order, 1, stable, leaf};
      b.build(0, order.data(), order.size());
      nodes.resize(static_cast<size_t>(b.next));
    }
    for (uint32_t i = 0; i < s.material_count; ++i) {
      const float* m = s.materials + 16 * i;
      Material q;
      q.albedo = ld3(m);
      q.emissive = ld3(m + 3);
      q.roughness = m[6];
      q.model = static_cast<uint32_t>(m[7] + 0.5f);
      q.metallic = m[8];
      q.ior = m[9];
      q.transmission = m[10];
      q.clearcoat = m[11];
      q.sheen = m[12];
      q.alpha = m[14];
      q.effect = static_cast<uint32_t>(m[15] + 0.5f) & 1023u;
      mats.push_back(q);
    }
    if (mats.empty()) {
      Material q{};
      q.albedo = {1.0f, 1.0f, 1.0f};
      q.emissive = {0.0f, 0.0f, 0.0f};
      q.roughness = 1.0f;
      q.ior = 1.5f;
      q.alpha = 1.0f;
      mats.push_back(q);
    }
    for (uint32_t i = 0; i < s.light_count; ++i) {
      const float* l = s.lights + 16 * i;
      lights.push_back(Light{ld3(l), ld3(l + 3), ld3(l + 8), l[6], l[7], l[11], l[12]});
    }
    env = ld3(s.environment);
    if (s.environment_map && s.environment_map_width && s.environment_map_height) {
      env_w = s.environment_map_width;
      env_h = s.environment_map_height;
      env_map.resize(static_cast<size_t>(env_w) * env_h);
      for (size_t i = 0; i < env_map.size(); ++i) env_map[i] = ld3(s.environment_map + 3 * i);
      env_scale = ld3(s.environment_map_scale);
      if (fmax_std(fmax_std(env_scale.x, env_scale.y), env_scale.z) <= 1.0e-6f) env_scale = {1.0f, 1.0f, 1.0f};
    }
    for (uint32_t i = 0; i < s.sdf_count; ++i) {
      const float* q = s.sdf_primitives + 16 * static_cast<size_t>(i);
      if (!(q[0] >= 0.0f && q[0] < 5.5f)) continue;   // unknown shape: never hits, counts nothing
      Sdf p;
      p.shape = static_cast<uint32_t>(q[0] + 0.5f);
      p.pos = ld3(q + 1);
      p.scale = ld3(q + 4);
      p.rot = ld3(q + 7);
      p.material = q[10] >= 0.0f ? static_cast<uint32_t>(q[10] + 0.5f) : 0u;
      p.radius = q[11];
      p.pa = q[12];
      p.pb = q[13];
      sdfs.push_back(p);
    }
    cam_pos = ld3(s.camera_position);
    fov = s.camera_fov_deg;
    aperture = s.camera_aperture_radius;
    focus = s.camera_focus_distance;
    if (s.camera_lens_set) {
      iris_blades = s.camera_iris_blade_count;
      iris_rotation = s.camera_iris_rotation_degrees;
      iris_roundness = s.camera_iris_roundness;
      squeeze = s.camera_anamorphic_squeeze;
    }
    // camera basis
    cam_fwd = unit(sub(ld3(s.camera_target), cam_pos));
    cam_right = unit(cross(cam_fwd, ld3(s.camera_up)));
    if (dot(cam_right, cam_right) <= kEps * kEps) cam_right = {1.0f, 0.0f, 0.0f};
    cam_up = unit(cross(cam_right, cam_fwd));
    if (dot(cam_up, cam_up) <= kEps * kEps) cam_up = {0.0f, 1.0f, 0.0f};
  }

  // Slab test with per-axis early exit; axes with |d| <= 1e-4 use an inside test.
  struct RayBox { float o[3], inv[3]; bool par[3]; };
  // The reference's slab setup: an axis with |d| <= 1e-4 counts as parallel
  // (origin-inside-slab test).  With the watertight test the boxes are tested
  // geometrically instead (only |d| < 1e-20 is parallel): the rule can cull a
  // box that a ray drifting up to 1e-4 t along that axis enters.
  static RayBox prep(V3 o, V3 d) {
    RayBox r;
    const float oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
    for (int a = 0; a < 3; ++a) {
      r.o[a] = oo[a];
      r.par[a] = g_triangle_test ? std::fabs(dd[a]) < 1e-20f : std::fabs(dd[a]) <= kEps;
      r.inv[a] = r.par[a] ? 0.0f : 1.0f / dd[a];
    }
    return r;
  }
  static bool slab(const Box& b, const RayBox& r, float tmax_in, float& tnear) {
    float lo = kEps, hi = tmax_in;
    for (int a = 0; a < 3; ++a) {
      if (r.par[a]) {
        if (r.o[a] < b.lo[a] || r.o[a] > b.hi[a]) return false;
        continue;
      }
      float t0 = (b.lo[a] - r.o[a]) * r.inv[a];
      float t1 = (b.hi[a] - r.o[a]) * r.inv[a];
      if (t0 > t1) std::swap(t0, t1);
      lo = fmax_std(lo, t0);
      hi = fmin_std(hi, t1);
      if (lo > hi) return false;
    }
    tnear = lo;
    return hi > kEps;
  }

  // Closest hit: returns prim slot or -1, with t.
  int64_t closest(V3 o, V3 d, float& t_out, Stats& st) const {
    if (nodes.empty() || prims.empty()) return -1;
    float best = std::numeric_limits<float>::infinity();
    int64_t hit = -1;
    const RayBox rb = prep(o, d);
    const WtRay wr = g_triangle_test ? prep_wt(d) : WtRay{};
    std::vector<int32_t> stack;
    stack.reserve(128);
    stack.push_back(0);
    while (!stack.empty()) {
      const int32_t id = stack.back();
      stack.pop_back();
      if (id < 0 || static_cast<size_t>(id) >= nodes.size()) continue;
      const Node& nd = nodes[static_cast<size_t>(id)];
      ++st.nodes;
      float tn = 0.0f;
      if (!slab(nd.box, rb, best, tn)) continue;
      if (nd.count > 0) {
        ++st.leaves;
        // Leaf batches of up to 8 lanes; a lane commits only when 1e-4 < t < best.
        st.tri_tests += static_cast<uint64_t>(nd.count);
        if (!(best > kEps)) continue;
        for (int32_t i = 0; i < nd.count; ++i) {
          const uint32_t pi = order[static_cast<size_t>(nd.first + i)];
          const Prim& p = prims[pi];
          if (g_triangle_test) {
            const float t = wt_test(p, o, wr);
            if (!(t > kEps) || !(t < best)) continue;   // a NaN t never commits
            ++st.tri_hits;
            best = t;
            hit = pi;
            continue;
          }
          const float hx = d.y * p.e2.z - d.z * p.e2.y;
          const float hy = d.z * p.e2.x - d.x * p.e2.z;
          const float hz = d.x * p.e2.y - d.y * p.e2.x;
          const float det = p.e1.x * hx + p.e1.y * hy + p.e1.z * hz;
          if (std::fabs(det) < kEps) continue;
          const float inv = 1.0f / det;
          const float sx = o.x - p.v0.x, sy = o.y - p.v0.y, sz = o.z - p.v0.z;
          const float u = (sx * hx + sy * hy + sz * hz) * inv;
          if (u < 0.0f || u > 1.0f) continue;
          const float qx = sy * p.e1.z - sz * p.e1.y;
          const float qy = sz * p.e1.x - sx * p.e1.z;
          const float qz = sx * p.e1.y - sy * p.e1.x;
          const float v = (d.x * qx + d.y * qy + d.z * qz) * inv;
          if (v < 0.0f || u + v > 1.0f) continue;
          const float t = (p.e2.x * qx + p.e2.y * qy + p.e2.z * qz) * inv;
          if (t <= kEps || t >= best) continue;
          ++st.tri_hits;
          best = t;
          hit = pi;
        }
        continue;
      }
      float tl = 0.0f, tr = 0.0f;
      const bool hl = nd.left >= 0 && slab(nodes[static_cast<size_t>(nd.left)].box, rb, best, tl);
      const bool hr = nd.right >= 0 && slab(nodes[static_cast<size_t>(nd.right)].box, rb, best, tr);
      if (hl && hr) {
        if (tl <= tr) { stack.push_back(nd.right); stack.push_back(nd.left); }
        else { stack.push_back(nd.left); stack.push_back(nd.right); }
      } else if (hl) {
        stack.push_back(nd.left);
      } else if (hr) {
        stack.push_back(nd.right);
      }
    }
    t_out = best;
    return hit;
  }

  struct Hit { bool hit; float t; V3 p, n; uint32_t mat; };

  bool intersect(V3 o, V3 d, Hit& h, Stats& st) const {
    h = Hit{false, 0.0f, {}, {}, 0};
    float t = 0.0f;
    float best = std::numeric_limits<float>::infinity();
    const int64_t k = closest(o, d, t, st);
    if (k >= 0) {
      const Prim& p = prims[static_cast<size_t>(k)];
      h.hit = true;
      h.t = t;
      h.p = add(o, mul(d, t));
      h.n = p.n;
      h.mat = p.material;
      best = t;
    }
    for (const Sdf& p : sdfs) {
      float ts = 0.0f;
      V3 n{};
      if (!sdf_hit(p, o, d, ts, n, st) || ts >= best) continue;
      best = ts;
      h.hit = true;
      h.t = ts;
      h.p = add(o, mul(d, ts));
      h.n = unit(n);
      h.mat = p.material;
    }
    return h.hit;
  }

  // apply_instance_transform_update of the CPU accelerator: every update checked
  // (dynamic instance with local geometry, complete primitive range, local
  // indices in range), the primitives recomputed with the new transform, then
  // refit_node(0) over the unchanged topology.
  bool apply_updates(const std::vector<vko_instance_update>& ups, std::string& why) {
    const vko_scene& s = *src;
    for (const auto& u : ups) {
      const uint32_t i = u.instance_index;
      if (i >= s.instance_count) { why = "unknown instance"; return false; }
      const uint32_t* loc = (s.instance_local && s.instance_transforms) ? s.instance_local + 5 * i : nullptr;
      if (!loc || !(loc[0] & 1u) || loc[2] == 0u || loc[4] == 0u) { why = "needs dynamic local geometry"; return false; }
    }
    for (const auto& u : ups) {
      const uint32_t i = u.instance_index;
      const uint32_t* loc = s.instance_local + 5 * i;
      const uint32_t count = s.instances[3 * i + 1], mat = s.instances[3 * i + 2];
      if (inst_count[i] != count) { why = "primitive range"; return false; }
      const float t[10] = {u.translation[0], u.translation[1], u.translation[2], u.rotation[0], u.rotation[1],
                           u.rotation[2], u.rotation[3], u.scale[0], u.scale[1], u.scale[2]};
      for (uint32_t k = 0; k < count; ++k) {
        const uint32_t lb = loc[3] + k * 3u, le = loc[1] + loc[2];
        if (lb >= 0xFFFFFFFEu || lb + 2u >= s.local_index_count) { why = "local indices"; return false; }
        V3 v[3];
        for (int j = 0; j < 3; ++j) {
          const uint32_t a = loc[1] + s.local_indices[lb + j];
          if (a >= le || a >= s.local_vertex_count) { why = "local vertices"; return false; }
          v[j] = instance_vertex(ld3(s.local_vertices + 3 * a), t);
        }
        Prim& p = prims[inst_first[i] + k];
        p.material = mat;
        p.v0 = v[0];
        p.v1 = v[1];
        p.v2 = v[2];
        p.e1 = sub(v[1], v[0]);
        p.e2 = sub(v[2], v[0]);
        const V3 cr = cross(p.e1, p.e2);
        const float l2 = dot(cr, cr);
        p.n = (l2 <= kEps * kEps) ? V3{0.0f, 1.0f, 0.0f} : mul(cr, 1.0f / std::sqrt(l2));
        Box& bx = boxes[inst_first[i] + k];
        bx.lo[0] = std::min({v[0].x, v[1].x, v[2].x}) - kEps;
        bx.lo[1] = std::min({v[0].y, v[1].y, v[2].y}) - kEps;
        bx.lo[2] = std::min({v[0].z, v[1].z, v[2].z}) - kEps;
        bx.hi[0] = std::max({v[0].x, v[1].x, v[2].x}) + kEps;
        bx.hi[1] = std::max({v[0].y, v[1].y, v[2].y}) + kEps;
        bx.hi[2] = std::max({v[0].z, v[1].z, v[2].z}) + kEps;
      }
    }
    if (!nodes.empty()) refit(0);
    return true;
  }

  Box refit(int32_t id) {
    Node& nd = nodes[static_cast<size_t>(id)];
    if (nd.count > 0) {
      Box b = boxes[order[static_cast<size_t>(nd.first)]];
      for (int32_t k = 1; k < nd.count; ++k) {
        const Box& o = boxes[order[static_cast<size_t>(nd.first + k)]];
        for (int a = 0; a < 3; ++a) {
          b.lo[a] = fmin_std(b.lo[a], o.lo[a]);
          b.hi[a] = fmax_std(b.hi[a], o.hi[a]);
        }
      }
      nd.box = b;
      return b;
    }
    const Box l = refit(nd.left), r = refit(nd.right);
    Box b;
    for (int a = 0; a < 3; ++a) {
      b.lo[a] = fmin_std(l.lo[a], r.lo[a]);
      b.hi[a] = fmax_std(l.hi[a], r.hi[a]);
    }
    nodes[static_cast<size_t>(id)].box = b;
    return b;
  }

  const Material& mat(uint32_t i) const { return mats[std::min<size_t>(i, mats.size() - 1)]; }
};

// ---------------------------------------------------------------- integrator
struct Integrator {
  const World& w;
  const vko_settings& cfg;

  // The material's albedo after its procedural effect at point p (normal n,
  // ray direction `in`), clamped to [0, 1.5].
  V3 albedo_of(const Material& m, V3 p, V3 n, V3 in) const {
    V3 c = m.albedo;
    const uint32_t fx = m.effect;
    if (fx != 0u) {
      const float h = fx_hash(p.x, p.y, p.z, static_cast<float>(fx));
      const float facing = dot(n, neg(in));
      switch (fx) {
        case 1u: {
          const float g = fmax_std(0.0f, 1.0f - std::fabs(facing));
          c = fx_lin(c, 0.65f + 0.25f * h, V3{0.25f, 0.22f, 0.28f}, g * g * (0.4f + m.sheen));
          break;
        }
        case 2u:
          c = mul(c, 0.45f + 0.55f * (0.5f + 0.5f * std::sin(p.x * 7.0f + p.z * 5.0f + h * 6.0f)));
          break;
        case 3u:
          c = mul(c, h > 0.72f ? 0.18f : 1.0f);
          break;
        case 4u: {
          const float vein = 0.5f + 0.5f * std::sin((p.x + p.y * 0.4f + p.z * 0.7f) * 9.0f + h * 3.0f);
          c = fx_lin(c, 0.55f + 0.45f * vein, V3{0.18f, 0.20f, 0.23f}, 1.0f - vein);
          break;
        }
        case 5u:
          c = fx_lin(c, 0.55f + 0.35f * h, V3{0.45f, 0.16f, 0.04f}, 0.25f + 0.25f * h);
          break;
        case 6u:
          c = mul(c, 0.65f + 0.35f * h);
          break;
        case 7u:
          c = fx_lin(c, 0.78f, V3{1.0f, 0.62f, 0.42f}, 0.16f);
          break;
        case 8u:
          c = fx_lin(c, 0.55f, V3{0.35f + 0.45f * h, 0.25f + 0.35f * (1.0f - h), 0.85f}, 0.45f);
          break;
        case 9u:
          c = mul(c, std::fmod(std::floor(p.x * 4.0f) + std::floor(p.z * 4.0f), 2.0f) < 0.5f ? 1.0f : 0.28f);
          break;
        case 10u:
          c = fx_lin(c, 0.45f, V3{1.0f, 0.35f + 0.3f * h, 0.08f}, 0.55f);
          break;
        case 11u:
          c = mul(c, 0.55f + 0.45f * (0.5f + 0.5f * std::sin(p.y * 18.0f + h * 5.0f)));
          break;
        case 12u: {
          const float f2 = fmax_std(0.0f, facing) * fmax_std(0.0f, facing);
          c = add(c, mul(V3{0.55f, 0.65f, 0.95f}, f2 * f2 * f2));
          break;
        }
        case 13u:
          c = mul(c, 0.65f + 0.35f * std::fabs(std::sin(p.x * 10.0f) * std::cos(p.z * 10.0f)));
          break;
        case 14u:
          c = mul(V3{0.15f, 0.75f, 1.0f}, 0.2f + 0.8f * std::pow(fmax_std(0.0f, 1.0f - std::fabs(facing)), 0.8f));
          break;
        case 15u: {
          const float bands = 0.5f + 0.5f * std::sin(p.y * 11.0f + p.x * 3.0f + h * 7.0f);
          const float rim = std::pow(fmax_std(0.0f, 1.0f - std::fabs(facing)), 1.5f);
          c = fx_lin(c, 0.25f + 0.45f * bands, V3{0.48f, 0.56f, 0.68f}, 0.18f + 0.32f * rim);
          break;
        }
        case 16u: case 17u: case 18u: case 19u:
          c = fx_wood(c, p, m.roughness, m.clearcoat, fx);
          break;
        default:
          break;
      }
    }
    return {fmin_std(1.5f, fmax_std(0.0f, c.x)), fmin_std(1.5f, fmax_std(0.0f, c.y)),
            fmin_std(1.5f, fmax_std(0.0f, c.z))};
  }

  V3 hemisphere(Stream& rng, V3 n) const {
    const float u1 = rng.u();
    const float u2 = rng.u();
    const float r = std::sqrt(fmax_std(0.0f, 1.0f - u1));
    const float phi = 2.0f * kPi * u2;
    const V3 loc{r * std::cos(phi), r * std::sin(phi), std::sqrt(fmax_std(0.0f, u1))};
    V3 t = cross((std::fabs(n.z) < 0.999f) ? V3{0.0f, 0.0f, 1.0f} : V3{0.0f, 1.0f, 0.0f}, n);
    t = unit(t);
    const V3 b = cross(n, t);
    return unit(add(add(mul(t, loc.x), mul(b, loc.y)), mul(n, loc.z)));
  }

  V3 phong(Stream& rng, V3 refl, float expo, V3 n) const {
    const float u1 = rng.u();
    const float u2 = rng.u();
    const float ct = std::pow(fmax_std(0.0f, u1), 1.0f / (expo + 1.0f));
    const float sn = std::sqrt(fmax_std(0.0f, 1.0f - ct * ct));
    const float phi = 2.0f * kPi * u2;
    const V3 ref = (std::fabs(refl.z) < 0.999f) ? V3{0.0f, 0.0f, 1.0f} : V3{0.0f, 1.0f, 0.0f};
    const V3 t = unit(cross(ref, refl));
    const V3 b = cross(refl, t);
    V3 out = unit(add(add(mul(t, sn * std::cos(phi)), mul(b, sn * std::sin(phi))), mul(refl, ct)));
    if (dot(out, n) <= 0.0f) {
      out = sub(out, mul(n, 2.0f * dot(out, n)));
      if (dot(out, n) <= 0.0f) return hemisphere(rng, n);
    }
    return out;
  }

  static float spot(const Light& l, V3 from_light) {
    if (l.inner <= -0.999f) return 1.0f;
    const float cone = dot(unit(from_light), unit(l.dir));
    if (cone <= l.outer) return 0.0f;
    if (cone >= l.inner || l.inner <= l.outer) return 1.0f;
    const float t = clampf((cone - l.outer) / (l.inner - l.outer), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
  }

  // NEE toward one uniformly picked light; returns false when no contribution.
  bool direct(const World::Hit& h, V3 view, Stream& rng, V3& out, Stats& st) const {
    if (w.lights.empty()) return false;
    const size_t nl = w.lights.size();
    const size_t pick = std::min(static_cast<size_t>(rng.u() * static_cast<float>(nl)), nl - 1u);
    const Light& L = w.lights[pick];
    V3 lp = L.pos;
    if (L.radius > 1.0e-5f) {
      const float uz = 1.0f - 2.0f * rng.u();
      const float r = std::sqrt(fmax_std(0.0f, 1.0f - uz * uz));
      const float phi = 6.28318530718f * rng.u();
      lp = add(lp, mul(V3{r * std::cos(phi), uz, r * std::sin(phi)}, L.radius));
    }
    const V3 tl = sub(lp, h.p);
    const float d2 = dot(tl, tl);
    const float dist = std::sqrt(d2);
    if (dist < kEps) return false;
    const V3 ldir = divs(tl, dist);
    const float cth = dot(h.n, ldir);
    if (cth <= 0.0f) return false;
    const float sf = spot(L, neg(ldir));
    if (sf <= 0.0f) return false;
    const Material& m = w.mat(h.mat);
    const float rough = clamp01(m.roughness);
    const bool mirror = m.model == 2u || rough <= 0.001f;
    const bool metal = m.model == 4u || m.metallic > 0.65f;
    const bool trans = m.model == 5u || m.transmission > 0.05f;
    const bool coat = m.model == 7u || m.clearcoat > 0.05f;
    ++st.shadow;
    V3 so = add(h.p, mul(h.n, 0.002f));
    float remain = dist - 0.004f;
    for (uint32_t skips = 0; skips < 8u && remain > 0.004f; ++skips) {
      World::Hit sh;
      if (!w.intersect(so, ldir, sh, st) || sh.t >= remain) break;
      const Material& sm = w.mat(sh.mat);
      if (!(sm.model == 5u || sm.transmission > 0.05f)) return false;
      const float adv = sh.t + 0.004f;
      so = add(so, mul(ldir, adv));
      remain -= adv;
    }
    const V3 alb = albedo_of(m, h.p, h.n, neg(ldir));
    const V3 irr = mul(L.color, (L.intensity * sf) / (d2 + kEps));
    V3 acc{0.0f, 0.0f, 0.0f};
    if (!mirror && !trans) {
      acc = add(acc, mul(mul(mulv(mul(alb, kInvPi), irr), cth), static_cast<float>(nl)));
    }
    if (mirror || metal || coat || trans || rough < 0.65f) {
      const V3 hv = unit(add(ldir, unit(view)));
      const float er = fmax_std(0.025f, rough * (metal ? 0.65f : 1.0f));
      const float a2 = er * er;
      const float pw = clampf(2.0f / fmax_std(0.0005f, a2 * a2) - 2.0f, 4.0f, 96.0f);
      const float spec = std::pow(fmax_std(0.0f, dot(h.n, hv)), pw);
      const float cv = fmax_std(0.0f, dot(h.n, unit(view)));
      float f0 = (1.0f - m.ior) / (1.0f + m.ior);
      f0 *= f0;
      const float fr = f0 + (1.0f - f0) * pow5(1.0f - cv);
      const float ss = clamp01((1.0f - rough) * 0.8f + m.metallic * 0.45f + m.clearcoat * 0.35f +
                               (mirror ? 0.75f : 0.0f) + (trans ? fr : 0.0f));
      const V3 tint = add(mul(V3{1.0f, 1.0f, 1.0f}, metal ? 0.15f : 0.88f), mul(alb, metal ? 0.85f : 0.12f));
      acc = add(acc, mul(mulv(tint, irr), spec * cth * static_cast<float>(nl) * fmax_std(0.15f, ss)));
    }
    out = acc;
    return true;
  }

  float light_pdf(V3 p, V3 dir) const {
    if (w.lights.empty()) return 0.0f;
    const float inv_n = 1.0f / static_cast<float>(w.lights.size());
    float total = 0.0f;
    for (const Light& L : w.lights) {
      const V3 tl = sub(L.pos, p);
      const float dist = std::sqrt(dot(tl, tl));
      if (dist < kEps) continue;
      if (dot(divs(tl, dist), dir) > 0.9999f) total += inv_n / (dist * dist + kEps);
    }
    return total;
  }

  static float mis(float a, float b) {
    const float a2 = a * a, b2 = b * b, den = a2 + b2;
    if (den <= 0.0f) return 1.0f;
    return a2 / den;
  }

  static float schlick(float c, float ior) {
    const float si = fmax_std(1.01f, ior);
    float r0 = (1.0f - si) / (1.0f + si);
    r0 *= r0;
    const float m = 1.0f - fmin_std(1.0f, fmax_std(0.0f, c));
    return r0 + (1.0f - r0) * m * m * m * m * m;
  }

  static V3 refract(V3 i, V3 n, float eta, bool& tir) {
    const float ci = fmin_std(1.0f, fmax_std(0.0f, dot(neg(i), n)));
    const float k = 1.0f - eta * eta * (1.0f - ci * ci);
    if (k < 0.0f) { tir = true; return {0.0f, 0.0f, 0.0f}; }
    tir = false;
    return unit(add(mul(i, eta), mul(n, eta * ci - std::sqrt(k))));
  }

  V3 trace(V3 o, V3 d, Stream& rng, uint64_t& segs, Stats& st) const {
    V3 rad{0.0f, 0.0f, 0.0f};
    V3 thr{1.0f, 1.0f, 1.0f};
    for (uint32_t depth = 0; depth < cfg.max_depth; ++depth) {
      ++segs;
      World::Hit h;
      if (!w.intersect(o, d, h, st)) {
        rad = add(rad, mulv(thr, w.environment(d)));
        break;
      }
      const bool entering = dot(d, h.n) < 0.0f;
      const V3 n = entering ? h.n : neg(h.n);
      const Material& m = w.mat(h.mat);
      const V3 alb = albedo_of(m, h.p, n, d);
      const float rough = clamp01(m.roughness);
      const bool emissive_model = m.model == 1u || m.emissive_any();
      const bool mirror = m.model == 2u || rough <= 0.001f;
      const bool metal = m.model == 4u || m.metallic > 0.65f;
      const bool trans = m.model == 5u || m.transmission > 0.05f;
      const bool diffuse = rough >= 0.999f && !mirror && !metal && !trans;
      const bool sheen = m.model == 6u;
      const bool coat = m.model == 7u || m.clearcoat > 0.05f;
      const bool toon = m.model == 8u;

      if (!cfg.enable_nee || depth == 0) {
        rad = add(rad, mulv(thr, m.emissive));
      } else if (cfg.enable_mis && emissive_model) {
        const float bp = fmax_std(0.0f, dot(n, neg(d))) * kInvPi;
        const float lp = light_pdf(o, d);
        rad = add(rad, mul(mulv(thr, m.emissive), mis(bp, lp)));
      }

      if (cfg.enable_nee && depth < cfg.max_depth - 1u) {
        World::Hit lh = h;
        lh.n = n;
        V3 nee{};
        if (direct(lh, neg(d), rng, nee, st)) {
          if (cfg.enable_mis) {
            const V3 tl = w.lights.empty() ? V3{0.0f, 0.0f, 0.0f} : sub(w.lights[0].pos, h.p);
            const V3 ld = unit(tl);
            const float bp = fmax_std(0.0f, dot(n, ld)) * kInvPi;
            const float lp = w.lights.empty() ? 1.0f : (1.0f / static_cast<float>(w.lights.size()));
            rad = add(rad, mul(mulv(thr, nee), mis(lp, bp)));
          } else {
            rad = add(rad, mulv(thr, nee));
          }
        }
      }

      V3 out;
      bool refracted = false;
      const V3 refl = sub(d, mul(n, 2.0f * dot(n, d)));
      if (mirror) {
        out = refl;
      } else if (trans) {
        const float ct = fmax_std(0.0f, dot(n, neg(d)));
        const float fr = schlick(ct, m.ior);
        if (rng.u() < fmin_std(0.98f, fr + m.clearcoat * 0.015f)) {
          out = refl;
        } else {
          bool tir = false;
          const float si = fmax_std(1.01f, m.ior);
          out = refract(d, n, entering ? (1.0f / si) : si, tir);
          if (tir || dot(out, out) <= 1.0e-8f) out = refl;
          else refracted = true;
        }
      } else if (diffuse || toon) {
        out = hemisphere(rng, n);
      } else {
        const float er = fmax_std(0.025f, rough * (metal ? 0.75f : 1.0f) * (coat ? 0.65f : 1.0f));
        const float a2 = er * er;
        const float ex = fmax_std(0.0f, 2.0f / (a2 * a2) - 2.0f);
        out = phong(rng, refl, ex, n);
        if (sheen && rng.u() < m.sheen * 0.35f) out = hemisphere(rng, n);
      }
      if (!trans && dot(out, n) <= 0.0f) break;
      V3 wgt = alb;
      if (metal || mirror) {
        wgt = mul(alb, 0.65f + 0.35f * m.metallic);
      } else if (trans) {
        const float ts = clamp01(m.alpha) * m.transmission;
        wgt = add(mul(V3{1.0f, 1.0f, 1.0f}, 1.0f - ts), mul(alb, ts));
        if (refracted) wgt = mul(wgt, fmax_std(0.55f, m.transmission));
      }
      if (toon) wgt = mul(wgt, dot(out, n) > 0.55f ? 1.0f : 0.45f);
      thr = mulv(thr, wgt);
      const float tmax = fmax_std(thr.x, fmax_std(thr.y, thr.z));
      if (tmax < 0.001f) break;
      const float rr = fmin_std(cfg.rr_max, fmax_std(cfg.rr_min, tmax));
      if (depth >= cfg.rr_start && rng.u() > rr) break;
      thr = divs(thr, rr);
      o = add(h.p, mul(out, 0.002f));
      d = out;
    }
    return rad;
  }

  // One camera path of pixel (x, y); returns false when the sample is not finite.
  bool shade(uint32_t x, uint32_t y, uint32_t sample, V3& out, uint64_t& segs, Stats& st) const {
    const uint32_t W = cfg.width, H = cfg.height;
    const uint64_t sample_seed = (static_cast<uint64_t>(y) << 32) | x;
    const uint64_t path_id = sample_seed + sample + 0u;
    uint64_t cam_seed = 0;
    // Camera stream: pixel = y*W + x, path id truncated to 32 bits.
    Stream crng(cfg.seed, 0u, sample, static_cast<uint32_t>(path_id), 0u, 0u,
                static_cast<uint64_t>(y) * W + x);
    const float fx = (static_cast<float>(x) + crng.u()) / static_cast<float>(std::max(1u, W));
    const float fy = (static_cast<float>(y) + crng.u()) / static_cast<float>(std::max(1u, H));
    cam_seed ^= static_cast<uint64_t>(crng.u() * static_cast<float>(0xffffu));
    const float aspect = static_cast<float>(W) / fmax_std(1.0f, static_cast<float>(H));
    const float thf = std::tan(0.5f * (w.fov * (kPi / 180.0f)));
    const float nx = (2.0f * fx - 1.0f) * aspect * thf;
    const float ny = (1.0f - 2.0f * fy) * thf;
    const V3 dir = unit(add(add(w.cam_fwd, mul(w.cam_right, nx)), mul(w.cam_up, ny)));
    V3 o = w.cam_pos;
    V3 d = dir;
    if (w.aperture > 0.0f && w.focus > kEps) {
      const float lr = std::sqrt(crng.u());
      const float lphi = 2.0f * kPi * crng.u();
      // polygonal aperture and anamorphic squeeze
      // (src/pathtracer/ScalarCpuPathTracer.Render.cpp:94-113)
      float boundary = 1.0f;
      const uint32_t blades = std::min(w.iris_blades, 64u);
      const float roundness = clamp01(w.iris_roundness);
      if (blades >= 3u && roundness < 0.999f) {
        const float sector = 2.0f * kPi / static_cast<float>(blades);
        const float local_phi = lphi - w.iris_rotation * (kPi / 180.0f);
        const float wrapped = local_phi - sector * std::floor(local_phi / sector);
        const float centered = wrapped > sector * 0.5f ? wrapped - sector : wrapped;
        const float polygon = std::cos(sector * 0.5f) / fmax_std(0.1f, std::cos(centered));
        boundary = polygon * (1.0f - roundness) + roundness;
      }
      const float r = w.aperture * lr * boundary;
      const float sq = std::isfinite(w.squeeze) ? fmax_std(0.01f, w.squeeze) : 1.0f;
      const V3 off = add(mul(w.cam_right, r * std::cos(lphi) * sq), mul(w.cam_up, r * std::sin(lphi)));
      const V3 fp = add(w.cam_pos, mul(dir, w.focus));
      o = add(w.cam_pos, off);
      d = unit(sub(fp, o));
    }
    Stream prng(cfg.seed + sample_seed + cam_seed, 0u, sample, path_id, 0u, 0u, sample_seed);
    uint64_t path_segs = 0;
    V3 c = trace(o, d, prng, path_segs, st);
    // A non-finite sample is dropped together with its segment count.
    if (!(std::isfinite(c.x) && std::isfinite(c.y) && std::isfinite(c.z))) return false;
    segs += path_segs;
    if (cfg.firefly_clamp > 0.0f) {
      c.x = fmin_std(c.x, cfg.firefly_clamp);
      c.y = fmin_std(c.y, cfg.firefly_clamp);
      c.z = fmin_std(c.z, cfg.firefly_clamp);
    }
    out = c;
    return true;
  }
};

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

extern "C" {

const char* vko_last_error(void) { return g_error.c_str(); }
const char* vko_impl_name(void) { return "port"; }

int vko_set_triangle_test(uint32_t mode) {
  if (mode > 1u) return fail("unknown triangle test");
  g_triangle_test = static_cast<int>(mode);
  return 0;
}

int vko_set_instance_updates(const vko_instance_update* updates, uint32_t count) {
  g_updates.assign(updates, updates + count);
  return 0;
}

int vko_render(const vko_scene* scene, const vko_settings* settings, uint32_t first_sample,
               uint32_t n_samples, uint32_t threads, const uint32_t* pixels, uint32_t pixel_count,
               float* film_sum, uint32_t* film_count, float* film_invalid, float* per_sample,
               vko_counters* counters) {
  if (!scene || !settings) return fail("null scene or settings");
  World w;
  w.load(*scene);
  if (!g_updates.empty()) {
    std::string why;
    if (!w.apply_updates(g_updates, why)) return fail("transform update rejected: " + why);
  }
  Integrator it{w, *settings};
  const uint32_t W = settings->width, H = settings->height;
  const size_t npx = static_cast<size_t>(W) * H;
  std::vector<uint32_t> list;
  if (pixels) {
    list.assign(pixels, pixels + pixel_count);
  } else {
    list.resize(npx);
    std::iota(list.begin(), list.end(), 0u);
  }
  std::vector<float> sum(3 * npx, 0.0f);
  std::vector<uint32_t> cnt(npx, 0u);
  std::vector<float> inv(npx, 0.0f);
  const uint32_t nt = std::max(1u, threads);
  std::vector<Stats> stats(nt);
  std::vector<uint64_t> segs(nt, 0u), samples(nt, 0u);
  double ms = 0.0;
  for (uint32_t k = 0; k < n_samples; ++k) {
    const uint32_t s = first_sample + k;
    float* ps = per_sample ? per_sample + static_cast<size_t>(k) * 3 * npx : nullptr;
    if (ps) std::fill(ps, ps + 3 * npx, 0.0f);
    const auto t0 = std::chrono::steady_clock::now();
    auto work = [&](uint32_t t) {
      const size_t b = list.size() * t / nt, e = list.size() * (t + 1) / nt;
      for (size_t i = b; i < e; ++i) {
        const uint32_t p = list[i];
        if (p >= npx) continue;
        V3 c{};
        const bool ok = it.shade(p % W, p / W, s, c, segs[t], stats[t]);
        if (!ok) { inv[p] += 1.0f; continue; }   // non-finite: dropped
        ++samples[t];
        sum[3 * p + 0] = sum[3 * p + 0] + c.x;
        sum[3 * p + 1] = sum[3 * p + 1] + c.y;
        sum[3 * p + 2] = sum[3 * p + 2] + c.z;
        cnt[p] += 1u;
        if (ps) { ps[3 * p] = c.x; ps[3 * p + 1] = c.y; ps[3 * p + 2] = c.z; }
      }
    };
    if (nt == 1) {
      work(0);
    } else {
      std::vector<std::thread> pool;
      for (uint32_t t = 0; t < nt; ++t) pool.emplace_back(work, t);
      for (auto& th : pool) th.join();
    }
    ms += ms_since(t0);
  }
  // The reference drops a non-finite sample before the film sees it
  // (ScalarCpuPathTracer.Render.cpp:268-275), so invalid_samples stays 0.
  std::fill(inv.begin(), inv.end(), 0.0f);
  if (film_sum) std::memcpy(film_sum, sum.data(), sum.size() * sizeof(float));
  if (film_count) std::memcpy(film_count, cnt.data(), cnt.size() * sizeof(uint32_t));
  if (film_invalid) std::memcpy(film_invalid, inv.data(), inv.size() * sizeof(float));
  if (counters) {
    std::memset(counters, 0, sizeof(*counters));
    for (uint32_t t = 0; t < nt; ++t) {
      counters->samples += samples[t];
      counters->rays += segs[t];
      counters->triangle_tests += stats[t].tri_tests;
      counters->triangle_hits += stats[t].tri_hits;
      counters->bvh_node_visits += stats[t].nodes;
      counters->bvh_leaf_visits += stats[t].leaves;
      counters->shadow_tests += stats[t].shadow;
      counters->sdf_tests += stats[t].sdf_tests;
      counters->sdf_steps += stats[t].sdf_steps;
      counters->sdf_hits += stats[t].sdf_hits;
      counters->sdf_misses += stats[t].sdf_misses;
    }
    counters->render_ms = ms;
  }
  return 0;
}

int vko_render_jobs(vko_job* jobs, uint32_t job_count, uint32_t threads, double* render_ms) {
  if (!jobs && job_count) return fail("null job list");
  const uint32_t nt = std::max(1u, threads);
  vko::WorkerPool pool(nt);
  double total_ms = 0.0;
  for (uint32_t j = 0; j < job_count; ++j) {
    vko_job& J = jobs[j];
    std::memset(&J.counters, 0, sizeof(J.counters));
    if (!J.scene || !J.settings) return fail("null scene or settings");
    if (J.pixel_count == 0 || J.n_samples == 0) continue;
    if (!J.pixels || !J.film_sum || !J.film_count) return fail("null pixel list or film");
    const uint32_t W = J.settings->width, H = J.settings->height;
    const size_t npx = static_cast<size_t>(W) * H;
    for (uint32_t i = 0; i < J.pixel_count; ++i)
      if (J.pixels[i] >= npx) return fail("pixel index outside the film");
    World w;
    w.load(*J.scene);
    Integrator it{w, *J.settings};
    const uint32_t chunk = vko::chunk_pixels(J.pixel_count, nt);
    const uint32_t chunks = (J.pixel_count + chunk - 1) / chunk;
    std::vector<float> sum(3u * J.pixel_count, 0.0f), m2(sum.size(), 0.0f);
    std::vector<uint32_t> cnt(J.pixel_count, 0u);
    std::vector<Stats> stats(nt);
    std::vector<uint64_t> segs(nt, 0u), samples(nt, 0u);
    std::atomic<uint32_t> next{0u};
    const double ms = pool.run([&](uint32_t t) {
      for (;;) {
        const uint32_t c = next.fetch_add(1u);
        if (c >= chunks) return;
        const uint32_t b = c * chunk, e = std::min(J.pixel_count, b + chunk);
        for (uint32_t k = 0; k < J.n_samples; ++k) {
          const uint32_t s = J.first_sample + k;
          for (uint32_t i = b; i < e; ++i) {
            const uint32_t p = J.pixels[i];
            V3 c3{};
            if (!it.shade(p % W, p / W, s, c3, segs[t], stats[t])) continue;   // non-finite: dropped
            ++samples[t];
            sum[3 * i + 0] = sum[3 * i + 0] + c3.x;
            sum[3 * i + 1] = sum[3 * i + 1] + c3.y;
            sum[3 * i + 2] = sum[3 * i + 2] + c3.z;
            m2[3 * i + 0] += c3.x * c3.x;
            m2[3 * i + 1] += c3.y * c3.y;
            m2[3 * i + 2] += c3.z * c3.z;
            cnt[i] += 1u;
          }
        }
      }
    });
    std::memcpy(J.film_sum, sum.data(), sum.size() * sizeof(float));
    std::memcpy(J.film_count, cnt.data(), cnt.size() * sizeof(uint32_t));
    if (J.film_m2) std::memcpy(J.film_m2, m2.data(), m2.size() * sizeof(float));
    for (uint32_t t = 0; t < nt; ++t) {
      J.counters.samples += samples[t];
      J.counters.rays += segs[t];
      J.counters.triangle_tests += stats[t].tri_tests;
      J.counters.triangle_hits += stats[t].tri_hits;
      J.counters.bvh_node_visits += stats[t].nodes;
      J.counters.bvh_leaf_visits += stats[t].leaves;
      J.counters.shadow_tests += stats[t].shadow;
      J.counters.sdf_tests += stats[t].sdf_tests;
      J.counters.sdf_steps += stats[t].sdf_steps;
      J.counters.sdf_hits += stats[t].sdf_hits;
      J.counters.sdf_misses += stats[t].sdf_misses;
    }
    J.counters.render_ms = ms;
    total_ms += ms;
  }
  if (render_ms) *render_ms = total_ms;
  return 0;
}

static void temperature_rgb(float kelvin, float rgb[3]) {
  const float t = std::clamp(kelvin, 1000.0f, 40000.0f) / 100.0f;
  if (t <= 66.0f) {
    rgb[0] = 1.0f;
    rgb[1] = std::clamp(0.39008158f * std::log(std::max(1.0f, t)) - 0.63184144f, 0.0f, 1.0f);
    rgb[2] = t <= 19.0f ? 0.0f
                        : std::clamp(0.5432068f * std::log(std::max(1.0f, t - 10.0f)) - 1.1962541f, 0.0f, 1.0f);
  } else {
    rgb[0] = std::clamp(1.2929362f * std::pow(t - 60.0f, -0.13320476f), 0.0f, 1.0f);
    rgb[1] = std::clamp(1.1298909f * std::pow(t - 60.0f, -0.075514846f), 0.0f, 1.0f);
    rgb[2] = 1.0f;
  }
}

int vko_apply_film_resolve(const float* hdr, uint32_t width, uint32_t height, const vko_resolve* s, uint8_t* rgba) {
  if (!hdr || !s || !rgba) return fail("null argument");
  float d65[3], target[3], wb[3];
  temperature_rgb(6500.0f, d65);
  temperature_rgb(s->white_balance_kelvin, target);
  for (int k = 0; k < 3; ++k) wb[k] = d65[k] / std::max(1.0e-3f, target[k]);
  const float inv_gamma = 1.0f / std::max(0.01f, s->gamma);
  auto tonemap = [&](float x) -> float {
    switch (s->tone_map) {
      case 1u: return x / (1.0f + x);
      case 2u: {
        auto F = [](float v) {
          const float A = 0.15f, B = 0.50f, C = 0.10f, D = 0.20f, E = 0.02f, Fc = 0.30f;
          return ((v * (A * v + C * B) + D * E) / (v * (A * v + B) + D * Fc)) - E / Fc;
        };
        return F(x) / F(11.2f);
      }
      case 3u: return (x * (2.51f * x + 0.03f)) / (x * (2.43f * x + 0.59f) + 0.14f);
      default: return x;
    }
  };
  const size_t n = static_cast<size_t>(width) * height;
  for (size_t i = 0; i < n; ++i) {
    for (int k = 0; k < 3; ++k) {
      float x = hdr[3 * i + k] * s->exposure * wb[k];
      if (!std::isfinite(x)) x = 0.0f;
      x = tonemap(x);
      if (s->output_transform == 0u) x = std::pow(std::max(0.0f, x), inv_gamma);
      if (s->clamp_output) x = std::min(1.0f, std::max(0.0f, x));
      rgba[4 * i + k] = static_cast<uint8_t>(x * 255.0f + 0.5f);
    }
    rgba[4 * i + 3] = 255u;
  }
  return 0;
}

int vko_build_bvh(const vko_scene* scene, uint32_t leaf_threshold, int deterministic, uint32_t* nodes_out,
                  uint32_t* node_count, uint32_t* prim_indices_out) {
  if (!scene || !nodes_out || !node_count || !prim_indices_out) return fail("null argument");
  World w;
  w.load(*scene, deterministic != 0, leaf_threshold == 0 ? 4u : leaf_threshold);
  *node_count = static_cast<uint32_t>(w.nodes.size());
  for (size_t i = 0; i < w.nodes.size(); ++i) {
    const Node& n = w.nodes[i];
    uint32_t* o = nodes_out + 10 * i;
    std::memcpy(o, n.box.lo, 12);
    std::memcpy(o + 3, n.box.hi, 12);
    std::memcpy(o + 6, &n.left, 4);
    std::memcpy(o + 7, &n.right, 4);
    std::memcpy(o + 8, &n.first, 4);
    std::memcpy(o + 9, &n.count, 4);
  }
  std::copy(w.order.begin(), w.order.end(), prim_indices_out);
  return 0;
}

int vko_intersect(const vko_scene* scene, const float* rays, uint64_t ray_count, uint32_t threads,
                  uint32_t* prim_out, float* t_out, uint64_t* stats, double* elapsed_ms) {
  if (!scene || !rays || !prim_out || !t_out) return fail("null argument");
  World w;
  w.load(*scene);
  const uint32_t nt = std::max(1u, threads);
  std::vector<Stats> st(nt);
  const auto t0 = std::chrono::steady_clock::now();
  auto work = [&](uint32_t t) {
    const uint64_t b = ray_count * t / nt, e = ray_count * (t + 1) / nt;
    for (uint64_t i = b; i < e; ++i) {
      float tt = 0.0f;
      const int64_t k = w.closest(ld3(rays + 6 * i), ld3(rays + 6 * i + 3), tt, st[t]);
      prim_out[i] = k < 0 ? 0xFFFFFFFFu : w.prims[static_cast<size_t>(k)].index;
      t_out[i] = k < 0 ? std::numeric_limits<float>::infinity() : tt;
    }
  };
  std::vector<std::thread> pool;
  for (uint32_t t = 0; t < nt; ++t) pool.emplace_back(work, t);
  for (auto& th : pool) th.join();
  if (elapsed_ms) *elapsed_ms = ms_since(t0);
  if (stats) {
    std::memset(stats, 0, 4 * sizeof(uint64_t));
    for (const Stats& s : st) {
      stats[0] += s.tri_tests;
      stats[1] += s.tri_hits;
      stats[2] += s.nodes;
      stats[3] += s.leaves;
    }
  }
  return 0;
}

}  // extern "C"
