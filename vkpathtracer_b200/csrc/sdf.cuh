// sdf.cuh -- analytic / sphere-traced SDF primitives next to the triangle BVH.
//
// The reference tests every SDF primitive for every ray after the triangle
// accelerator and keeps the nearest surface
// (ScalarCpuPathTracer::intersect_scene, src/pathtracer/ScalarCpuPathTracer.Intersect.cpp:91-129).
// Spheres are solved analytically (intersect_sphere,
// src/pathtracer/ScalarCpuPathTracer.cpp:855-901); boxes, rounded boxes,
// planes, tori and capsules are sphere-traced from t = 0 with at most 192
// steps (intersect_box, :903-930, which the other shapes call) over the
// distance functions of sdf_distance (:808-845), and the normal of a marched
// hit is the central difference of sdf_normal (:847-853).  Every expression
// keeps the reference's operation order, so hit distances and normals are
// bit-identical to it under -fmad=false.
//
// Record (8 float4 per primitive, built on the host by context.cu):
//   [0] position xyz, shape bits      [1] scale xyz (as given), material bits
//   [2] divisor xyz (scale, 0 -> 1), radius
//   [3] param_a, param_b, flags (bit 0: all divisors 1, bit 1: all angles 0), -
//   [4] sin/cos(-rx), sin/cos(-ry)    [5] sin/cos(-rz), sin/cos(rz)
//   [6] sin/cos(ry), sin/cos(rx)
//   [7] cull radius, cull margin factor, -, -
// The sines and cosines are the host's sinf/cosf of the same angles the
// reference passes to std::sin/std::cos (rotate_x/y/z, :113-137), computed
// once per primitive instead of per distance evaluation.
//
// Work the reference does and this code skips, without changing any hit:
// * a closest-hit march stops once t reaches the nearest hit so far (a later
//   hit would be rejected by the t < best test);
// * a marched shape with a bounded surface set {distance <= 1e-4} has a
//   world-space bounding sphere (radius from the shape's parameters, times
//   the largest scale divisor); a ray whose line passes farther than that
//   radius plus a rounding margin from the centre cannot produce a sample
//   point with distance <= 1e-4, so its march is not run (a miss).  The margin
//   (1e-4 relative to the magnitudes involved, times the divisor ratio, plus
//   1e-3) is about a hundred times the rounding error of the march's point
//   arithmetic.  Planes and non-finite parameters are never culled.
// * the world -> primitive map of a distance evaluation skips the division
//   when every divisor is 1 (x / 1 is x exactly) and the rotation when every
//   angle is 0 (sin 0 = 0, cos 0 = 1: the rotated vector equals the input up
//   to the sign of zero components, which no distance value depends on:
//   boxes take fabs, spheres, tori and capsules square, a plane's value is
//   only compared and clamped).  The hit normal keeps the full map.
#pragma once

#include "common.cuh"

namespace vkptc {

constexpr uint32_t kSdfTag = 0x80000000u;   // primitive id of SDF k: kSdfTag | k
constexpr uint32_t kSdfWords = 8;            // float4 per record
constexpr uint32_t kSdfMaxSteps = 192u;
constexpr float kSdfMinStep = 1.0e-3f;
constexpr float kSdfMaxDistance = 10000.0f;
__device__ __forceinline__ float sdf_inf() { return __int_as_float(0x7f800000); }

enum SdfShape : uint32_t { kSdfSphere = 0, kSdfBox, kSdfRoundedBox, kSdfPlane, kSdfTorus, kSdfCapsule };

struct SdfPrim {
  V3 pos, scale, div;
  uint32_t shape, material, flags;
  float radius, pa, pb;
  float sx_i, cx_i, sy_i, cy_i, sz_i, cz_i;   // inverse rotation (angles negated)
  float sz, cz, sy, cy, sx, cx;               // forward rotation
  float cull_r, cull_k;                       // bounding radius (0: never culled), margin factor
};

__device__ __forceinline__ SdfPrim load_sdf(const float4* rec) {
  const float4 a = __ldg(rec), b = __ldg(rec + 1), c = __ldg(rec + 2), d = __ldg(rec + 3);
  const float4 e = __ldg(rec + 4), f = __ldg(rec + 5), g = __ldg(rec + 6), h = __ldg(rec + 7);
  SdfPrim p;
  p.pos = mk(a.x, a.y, a.z);
  p.shape = __float_as_uint(a.w);
  p.scale = mk(b.x, b.y, b.z);
  p.material = __float_as_uint(b.w);
  p.div = mk(c.x, c.y, c.z);
  p.radius = c.w;
  p.pa = d.x;
  p.pb = d.y;
  p.flags = __float_as_uint(d.z);
  p.sx_i = e.x; p.cx_i = e.y; p.sy_i = e.z; p.cy_i = e.w;
  p.sz_i = f.x; p.cz_i = f.y; p.sz = f.z; p.cz = f.w;
  p.sy = g.x; p.cy = g.y; p.sx = g.z; p.cx = g.w;
  p.cull_r = h.x;
  p.cull_k = h.y;
  return p;
}

__device__ __forceinline__ float sdf_len(V3 v) { return sqrtf(dot(v, v)); }

// rotate_x / rotate_y / rotate_z with precomputed sine and cosine.
__device__ __forceinline__ V3 rot_x(V3 v, float s, float c) { return mk(v.x, c * v.y - s * v.z, s * v.y + c * v.z); }
__device__ __forceinline__ V3 rot_y(V3 v, float s, float c) { return mk(c * v.x + s * v.z, v.y, -s * v.x + c * v.z); }
__device__ __forceinline__ V3 rot_z(V3 v, float s, float c) { return mk(c * v.x - s * v.y, s * v.x + c * v.y, v.z); }

constexpr uint32_t kSdfUnitScale = 1u, kSdfNoRotation = 2u;

// divide_by_scale(rotate_euler_inv(v)), the world -> primitive-space map.
__device__ __forceinline__ V3 sdf_to_local(const SdfPrim& p, V3 v) {
  const V3 r = rot_z(rot_y(rot_x(v, p.sx_i, p.cx_i), p.sy_i, p.cy_i), p.sz_i, p.cz_i);
  return mk(r.x / p.div.x, r.y / p.div.y, r.z / p.div.z);
}

// The same map for distance evaluations, with identity steps skipped.
__device__ __forceinline__ V3 sdf_to_local_dist(const SdfPrim& p, V3 v) {
  const V3 r = (p.flags & kSdfNoRotation) ? v : rot_z(rot_y(rot_x(v, p.sx_i, p.cx_i), p.sy_i, p.cy_i), p.sz_i, p.cz_i);
  if (p.flags & kSdfUnitScale) return r;
  return mk(r.x / p.div.x, r.y / p.div.y, r.z / p.div.z);
}

__device__ __forceinline__ float sdf_distance(const SdfPrim& p, V3 world) {
  const V3 l = sdf_to_local_dist(p, sub(world, p.pos));
  switch (p.shape) {
    case kSdfSphere:
      return sdf_len(l) - p.radius;
    case kSdfBox: {
      const V3 q = mk(fabsf(l.x) - p.scale.x, fabsf(l.y) - p.scale.y, fabsf(l.z) - p.scale.z);
      const V3 mq = mk(smax(0.0f, q.x), smax(0.0f, q.y), smax(0.0f, q.z));
      return sdf_len(mq) + smin(smax(q.x, smax(q.y, q.z)), 0.0f);
    }
    case kSdfRoundedBox: {
      const float r = p.pa;
      const V3 q = mk(fabsf(l.x) - p.scale.x + r, fabsf(l.y) - p.scale.y + r, fabsf(l.z) - p.scale.z + r);
      const V3 mq = mk(smax(0.0f, q.x), smax(0.0f, q.y), smax(0.0f, q.z));
      return sdf_len(mq) + smin(smax(q.x, smax(q.y, q.z)), 0.0f) - p.pa;
    }
    case kSdfPlane:
      return l.y + p.pb;
    case kSdfTorus: {
      const float a = smax(0.05f, p.pa);
      const float b = smax(0.02f, p.radius);
      const float qx = sdf_len(mk(l.x, 0.0f, l.z)) - a;
      return sdf_len(mk(qx, l.y, 0.0f)) - b;
    }
    default: {   // capsule
      const V3 a = mk(0.0f, -p.pa, 0.0f);
      const V3 b = mk(0.0f, p.pa, 0.0f);
      const V3 ab = sub(b, a);
      const float t = dot(sub(l, a), ab) / smax(kEps, dot(ab, ab));
      const float c = smax(0.0f, smin(1.0f, t));
      const V3 closest = add(a, mul(ab, c));
      return sdf_len(sub(l, closest)) - p.radius;
    }
  }
}

// sdf_normal: central differences with e = 5e-4, normalised.
static __device__ __noinline__ V3 sdf_march_normal(const SdfPrim& p, V3 w) {
  const float e = 0.0005f;
  const float dx = sdf_distance(p, add(w, mk(e, 0.0f, 0.0f))) - sdf_distance(p, sub(w, mk(e, 0.0f, 0.0f)));
  const float dy = sdf_distance(p, add(w, mk(0.0f, e, 0.0f))) - sdf_distance(p, sub(w, mk(0.0f, e, 0.0f)));
  const float dz = sdf_distance(p, add(w, mk(0.0f, 0.0f, e))) - sdf_distance(p, sub(w, mk(0.0f, 0.0f, e)));
  return unit(mul(mk(dx, dy, dz), 0.5f));
}

struct SdfCount {
  uint32_t tests = 0u, steps = 0u, hits = 0u;
};

// Analytic sphere; returns the hit distance or a negative value on a miss.
__device__ __forceinline__ float sdf_sphere_t(const SdfPrim& p, V3 o, V3 d, V3& lo, V3& ld) {
  const float radius = smax(0.01f, p.radius);
  lo = sdf_to_local(p, sub(o, p.pos));
  ld = sdf_to_local(p, d);
  const float a = dot(ld, ld);
  if (a <= kEps * kEps) return -1.0f;
  const float half_b = dot(lo, ld);
  const float c = dot(lo, lo) - radius * radius;
  const float disc = half_b * half_b - a * c;
  if (disc < 0.0f) return -1.0f;
  const float root = sqrtf(disc);
  float cand = (-half_b - root) / a;
  if (cand <= kEps) cand = (-half_b + root) / a;
  if (cand <= kEps || !isfinite(cand)) return -1.0f;
  return cand;
}

// Sphere tracing from t = 0.  Returns the distance of the first point whose
// distance value is <= 1e-4, or a negative value on a miss.  A march that
// reaches t >= t_stop (any-hit queries) gives up early: every later hit is at
// t >= t_stop.
__device__ __forceinline__ float sdf_march_t(const SdfPrim& p, V3 o, V3 d, float t_stop, uint32_t& steps) {
  float t = 0.0f;
  for (uint32_t i = 0; i < kSdfMaxSteps; ++i) {
    if (!(t < t_stop)) return -1.0f;
    ++steps;
    const float dist = sdf_distance(p, add(o, mul(d, t)));
    if (dist <= kEps) return t;
    t += smax(kSdfMinStep, dist);
    if (t > kSdfMaxDistance) return -1.0f;
  }
  return -1.0f;
}

// True when the line o + d t (t >= 0) passes within the primitive's bounding
// sphere plus the rounding margin (or the primitive is never culled).
__device__ __forceinline__ bool sdf_near(const SdfPrim& p, V3 o, V3 d) {
  if (!(p.cull_r > 0.0f)) return true;
  const V3 c = sub(p.pos, o);
  const float dd = dot(d, d);
  const float tc = dd > 0.0f ? fmaxf(0.0f, dot(c, d) / dd) : 0.0f;
  const V3 w = sub(c, mul(d, tc));
  const float mag = fabsf(o.x) + fabsf(o.y) + fabsf(o.z) + fabsf(p.pos.x) + fabsf(p.pos.y) + fabsf(p.pos.z) +
                    tc * sqrtf(dd) + p.cull_r;
  const float r = p.cull_r + p.cull_k * 1.0e-4f * mag + 1.0e-3f;
  return dot(w, w) <= r * r;
}

// Distance of primitive p along (o, d) (negative: miss), counting its work.
__device__ __forceinline__ float sdf_test(const SdfPrim& p, V3 o, V3 d, float t_stop, SdfCount& n) {
  ++n.tests;
  float t;
  if (p.shape != kSdfSphere && !sdf_near(p, o, d)) return -1.0f;
  if (p.shape == kSdfSphere) {
    V3 lo, ld;
    t = sdf_sphere_t(p, o, d, lo, ld);
    ++n.steps;
  } else {
    t = sdf_march_t(p, o, d, t_stop, n.steps);
  }
  if (t >= 0.0f) ++n.hits;
  return t;
}

// The nearest-hit reduction of intersect_scene over the SDF table: replaces
// (best_t, prim) when a primitive is strictly nearer than the triangle hit and
// than every earlier primitive.
__device__ __forceinline__ void sdf_closest(const float4* sdf, uint32_t count, V3 o, V3 d, float& best_t,
                                            uint32_t& prim, SdfCount& n) {
  for (uint32_t k = 0; k < count; ++k) {
    const SdfPrim p = load_sdf(sdf + kSdfWords * k);
    const float t = sdf_test(p, o, d, best_t, n);
    if (t >= 0.0f && t < best_t) {
      best_t = t;
      prim = kSdfTag | k;
    }
  }
}

// Any SDF hit nearer than tmax (the shadow test of an opaque scene).
__device__ __forceinline__ bool sdf_any(const float4* sdf, uint32_t count, V3 o, V3 d, float tmax, SdfCount& n) {
  for (uint32_t k = 0; k < count; ++k) {
    const SdfPrim p = load_sdf(sdf + kSdfWords * k);
    const float t = sdf_test(p, o, d, tmax, n);
    if (t >= 0.0f && t < tmax) return true;
  }
  return false;
}

// ------------------------------------------------ load-balanced SDF stages
// The same tests as sdf_closest / sdf_any, one query per lane, advanced one
// unit of work per call: the start of a primitive (the analytic sphere, or the
// cull test) or one sphere-tracing step.  A lane whose query is done claims
// another (warp-aggregated, as the traversal does), so a warp is not held by
// its longest march.  Results are identical to the per-query loops.
struct SdfLane {
  V3 o, d;
  float best;        // closest: nearest hit so far; any: the query's upper bound
  uint32_t prim;     // closest: its primitive id; any: 1 when occluded
  const float4* sdf;
  uint32_t count, k, i;   // primitive count, current primitive, march steps taken on it
  float t;                // march distance on primitive k
  SdfPrim p;              // primitive k
};

__device__ __forceinline__ void sdf_lane_next(SdfLane& L) {
  ++L.k;
  L.i = 0u;
  L.t = 0.0f;
}

// Returns true when the lane's query is finished.
template <bool kAny>
__device__ __forceinline__ bool sdf_lane_step(SdfLane& L, SdfCount& n) {
  if (L.k >= L.count) return true;
  if (L.i == 0u) {   // start of primitive k (its first march step follows below)
    L.p = load_sdf(L.sdf + kSdfWords * L.k);
    ++n.tests;
    if (L.p.shape == kSdfSphere) {
      V3 lo, ld;
      const float t = sdf_sphere_t(L.p, L.o, L.d, lo, ld);
      ++n.steps;
      if (t >= 0.0f) {
        ++n.hits;
        if (t < L.best) {
          if (kAny) {
            L.prim = 1u;
            return true;
          }
          L.best = t;
          L.prim = kSdfTag | L.k;
        }
      }
      sdf_lane_next(L);
      return L.k >= L.count;
    }
    if (!sdf_near(L.p, L.o, L.d)) {
      sdf_lane_next(L);
      return L.k >= L.count;
    }
  }
  // one step of intersect_box's march (t starts at 0, at most 192 steps)
  if (!(L.t < L.best)) {
    sdf_lane_next(L);
    return L.k >= L.count;
  }
  ++n.steps;
  const float dist = sdf_distance(L.p, add(L.o, mul(L.d, L.t)));
  if (dist <= kEps) {
    ++n.hits;
    if (kAny) {
      L.prim = 1u;
      return true;
    }
    L.best = L.t;
    L.prim = kSdfTag | L.k;
    sdf_lane_next(L);
    return L.k >= L.count;
  }
  L.t += smax(kSdfMinStep, dist);
  ++L.i;
  if (L.t > kSdfMaxDistance || L.i >= kSdfMaxSteps) {
    sdf_lane_next(L);
    return L.k >= L.count;
  }
  return false;
}

// Persistent lanes over n queries: Src::load(j, L) fills o, d, best, prim, sdf,
// count (count 0: nothing to test); Src::finish(j, L) stores the result.
template <class Src, bool kAny>
__device__ __forceinline__ void sdf_persistent(const Src& src, uint32_t n, uint32_t* fetch, int steps, SdfCount& cnt) {
  const unsigned lane_id = threadIdx.x & 31u;
  SdfLane L;
  bool active = false, exhausted = false;
  uint32_t tag = 0u;
  while (true) {
    const unsigned idle = __ballot_sync(0xffffffffu, !active);
    if (idle != 0u && !exhausted) {
      uint32_t base = 0u;
      if (lane_id == 0u) base = atomicAdd(fetch, static_cast<uint32_t>(__popc(idle)));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (base >= n) exhausted = true;
      if (!active) {
        const uint32_t j = base + static_cast<uint32_t>(__popc(idle & ((1u << lane_id) - 1u)));
        if (j < n && j >= base) {
          src.load(j, L);
          L.k = 0u;
          L.i = 0u;
          L.t = 0.0f;
          if (L.count == 0u) {
            src.finish(j, L);
          } else {
            tag = j;
            active = true;
          }
        }
      }
    }
    if (!__any_sync(0xffffffffu, active)) break;
    if (active) {
      for (int s = 0; s < steps; ++s) {
        if (sdf_lane_step<kAny>(L, cnt)) {
          src.finish(tag, L);
          active = false;
          break;
        }
      }
    }
  }
}

// Surface normal of the hit of primitive k at distance t along (o, d), as the
// reference reports it (out.normal = normalize(normal)).
static __device__ __noinline__ V3 sdf_hit_normal(const float4* sdf, uint32_t k, V3 o, V3 d, float t) {
  const SdfPrim p = load_sdf(sdf + kSdfWords * k);
  V3 n;
  if (p.shape == kSdfSphere) {
    V3 lo, ld;
    sdf_sphere_t(p, o, d, lo, ld);
    const V3 local_hit = add(lo, mul(ld, t));
    const V3 ln = unit(local_hit);
    const V3 ls = mk(ln.x / p.div.x, ln.y / p.div.y, ln.z / p.div.z);
    n = unit(rot_x(rot_y(rot_z(ls, p.sz, p.cz), p.sy, p.cy), p.sx, p.cx));
  } else {
    n = sdf_march_normal(p, add(o, mul(d, t)));
  }
  return unit(n);
}

__device__ __forceinline__ uint32_t sdf_material(const float4* sdf, uint32_t k) {
  return __float_as_uint(__ldg(sdf + kSdfWords * k + 1).w);
}

}  // namespace vkptc
