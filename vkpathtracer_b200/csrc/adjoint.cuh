// adjoint.cuh -- differentiable path tracing: the per-vertex integrator math
// written once over a scalar type, instantiated with float for the primal
// replay and with a 7-tangent dual number for the local Jacobians of the
// reverse sweep.
//
// There is no counterpart in the reference (its tracer has no derivative
// path).  The float instantiation follows the reference's trace loop
// (src/pathtracer/ScalarCpuPathTracer.cpp:1148-1289), sample_direct_light
// (:1022-1118) and sample_phong_lobe (:996-1020) in the same operation order
// as shade_bounce / nee_setup / sample_phong, for the materials the adjoint
// supports: Lambertian and Phong-lobe glossy (models 0, 1, 3; no metal,
// mirror, clear coat or transmission), optionally emissive.
//
// Estimator differentiated (it is the one the FP64 CPU adjoint restates):
//   * directions are reparameterized: a Phong-lobe direction is a function of
//     its two uniforms, the reflected direction and the exponent, so it moves
//     with the roughness and with the incoming direction; a hemisphere
//     direction depends on nothing differentiable;
//   * the Russian-roulette survival probability is held constant (detached):
//     throughput divides by it, but no derivative flows through it;
//   * every discrete decision (hit primitive, visibility, lobe fallback,
//     frame choice, termination) is taken from the primal replay, so
//     visibility-boundary terms are excluded.
#pragma once

#include "integrator.cuh"

namespace vkptc {

constexpr int kAdjN = 7;                  // tangents: origin xyz, direction xyz, roughness
constexpr uint32_t kAdjMaxDepth = 8u;     // vertices recorded per path
constexpr uint32_t kAdjParams = 7u;       // per material: albedo rgb, roughness, emission rgb
constexpr uint32_t kAdjMaxMaterials = 64u;

// Vertex flags recorded by the primal replay.
enum : uint32_t {
  kVfEntering = 1u << 0,    // the ray arrived from the geometric normal's side
  kVfNeeValid = 1u << 1,    // sample_direct_light produced a candidate
  kVfNeeVis = 1u << 2,      // ... and its contribution was added
  kVfFrameAlt = 1u << 3,    // Phong frame built around (0,1,0)
  kVfReflected = 1u << 4,   // Phong direction mirrored about the normal
  kVfHemi = 1u << 5,        // ... and replaced by a hemisphere direction
  kVfCont = 1u << 6,        // the path continues to the next vertex
  kVfMiss = 1u << 7,        // the ray left the scene (environment term)
};

// ------------------------------------------------------------- dual numbers
struct Dual {
  float v;
  float g[kAdjN];
};
__device__ __forceinline__ Dual dconst(float v) {
  Dual r;
  r.v = v;
#pragma unroll
  for (int i = 0; i < kAdjN; ++i) r.g[i] = 0.0f;
  return r;
}
__device__ __forceinline__ float val(float a) { return a; }
__device__ __forceinline__ float val(const Dual& a) { return a.v; }

__device__ __forceinline__ Dual operator+(const Dual& a, const Dual& b) {
  Dual r;
  r.v = a.v + b.v;
#pragma unroll
  for (int i = 0; i < kAdjN; ++i) r.g[i] = a.g[i] + b.g[i];
  return r;
}
__device__ __forceinline__ Dual operator+(const Dual& a, float b) {
  Dual r = a;
  r.v = a.v + b;
  return r;
}
__device__ __forceinline__ Dual operator+(float a, const Dual& b) { return b + a; }
__device__ __forceinline__ Dual operator-(const Dual& a, const Dual& b) {
  Dual r;
  r.v = a.v - b.v;
#pragma unroll
  for (int i = 0; i < kAdjN; ++i) r.g[i] = a.g[i] - b.g[i];
  return r;
}
__device__ __forceinline__ Dual operator-(const Dual& a, float b) {
  Dual r = a;
  r.v = a.v - b;
  return r;
}
__device__ __forceinline__ Dual operator-(float a, const Dual& b) {
  Dual r;
  r.v = a - b.v;
#pragma unroll
  for (int i = 0; i < kAdjN; ++i) r.g[i] = -b.g[i];
  return r;
}
__device__ __forceinline__ Dual operator-(const Dual& a) {
  Dual r;
  r.v = -a.v;
#pragma unroll
  for (int i = 0; i < kAdjN; ++i) r.g[i] = -a.g[i];
  return r;
}
__device__ __forceinline__ Dual operator*(const Dual& a, const Dual& b) {
  Dual r;
  r.v = a.v * b.v;
#pragma unroll
  for (int i = 0; i < kAdjN; ++i) r.g[i] = a.g[i] * b.v + a.v * b.g[i];
  return r;
}
__device__ __forceinline__ Dual operator*(const Dual& a, float b) {
  Dual r;
  r.v = a.v * b;
#pragma unroll
  for (int i = 0; i < kAdjN; ++i) r.g[i] = a.g[i] * b;
  return r;
}
__device__ __forceinline__ Dual operator*(float a, const Dual& b) {
  Dual r;
  r.v = a * b.v;
#pragma unroll
  for (int i = 0; i < kAdjN; ++i) r.g[i] = a * b.g[i];
  return r;
}
__device__ __forceinline__ Dual operator/(const Dual& a, const Dual& b) {
  Dual r;
  r.v = a.v / b.v;
  const float inv = 1.0f / b.v;
#pragma unroll
  for (int i = 0; i < kAdjN; ++i) r.g[i] = (a.g[i] - r.v * b.g[i]) * inv;
  return r;
}
__device__ __forceinline__ Dual operator/(const Dual& a, float b) {
  Dual r;
  r.v = a.v / b;
  const float inv = 1.0f / b;
#pragma unroll
  for (int i = 0; i < kAdjN; ++i) r.g[i] = a.g[i] * inv;
  return r;
}
__device__ __forceinline__ Dual operator/(float a, const Dual& b) {
  Dual r;
  r.v = a / b.v;
  const float s = -r.v / b.v;
#pragma unroll
  for (int i = 0; i < kAdjN; ++i) r.g[i] = s * b.g[i];
  return r;
}
// std::max / std::min / std::clamp with the float versions' comparison order.
__device__ __forceinline__ Dual smax(const Dual& a, float b) { return (a.v < b) ? dconst(b) : a; }
__device__ __forceinline__ Dual smax(float a, const Dual& b) { return (a < b.v) ? b : dconst(a); }
__device__ __forceinline__ Dual smin(const Dual& a, float b) { return (b < a.v) ? dconst(b) : a; }
__device__ __forceinline__ Dual smin(float a, const Dual& b) { return (b.v < a) ? b : dconst(a); }
__device__ __forceinline__ Dual sclamp(const Dual& v, float lo, float hi) {
  return (v.v < lo) ? dconst(lo) : ((hi < v.v) ? dconst(hi) : v);
}
__device__ __forceinline__ Dual clamp01(const Dual& v) {
  if (!isfinite(v.v)) return dconst(0.0f);
  return smin(1.0f, smax(0.0f, v));
}
__device__ __forceinline__ float gsqrt(float a) { return sqrtf(a); }
__device__ __forceinline__ Dual gsqrt(const Dual& a) {
  Dual r;
  r.v = sqrtf(a.v);
  const float s = r.v > 0.0f ? 0.5f / r.v : 0.0f;
#pragma unroll
  for (int i = 0; i < kAdjN; ++i) r.g[i] = a.g[i] * s;
  return r;
}
// x^y for the primal (float) and both-dual forms.
template <bool kParity>
__device__ __forceinline__ float gpow(float x, float y) { return t_pow<kParity>(x, y); }
template <bool kParity>
__device__ __forceinline__ Dual gpow(const Dual& x, const Dual& y) {
  Dual r;
  r.v = t_pow<kParity>(x.v, y.v);
  if (!(x.v > 0.0f)) {
#pragma unroll
    for (int i = 0; i < kAdjN; ++i) r.g[i] = 0.0f;
    return r;
  }
  const float a = r.v * y.v / x.v, b = r.v * logf(x.v);
#pragma unroll
  for (int i = 0; i < kAdjN; ++i) r.g[i] = a * x.g[i] + b * y.g[i];
  return r;
}
template <bool kParity>
__device__ __forceinline__ Dual gpow(float x, const Dual& y) { return gpow<kParity>(dconst(x), y); }
__device__ __forceinline__ float lift_s(float v, float) { return v; }
__device__ __forceinline__ Dual lift_s(float v, const Dual&) { return dconst(v); }

// ------------------------------------------------------------- dual vectors
struct DV3 {
  Dual x, y, z;
};
__device__ __forceinline__ V3 vval(V3 a) { return a; }
__device__ __forceinline__ V3 vval(const DV3& a) { return mk(a.x.v, a.y.v, a.z.v); }
template <class VT> __device__ __forceinline__ VT lift(V3 a);
template <> __device__ __forceinline__ V3 lift<V3>(V3 a) { return a; }
template <> __device__ __forceinline__ DV3 lift<DV3>(V3 a) { return DV3{dconst(a.x), dconst(a.y), dconst(a.z)}; }

__device__ __forceinline__ DV3 add(const DV3& a, const DV3& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ DV3 sub(const DV3& a, const DV3& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ DV3 neg(const DV3& a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ DV3 mul(const DV3& a, const Dual& s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ DV3 mul(const DV3& a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ DV3 mul(V3 a, const Dual& s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ DV3 mulv(const DV3& a, const DV3& b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ DV3 mulv(V3 a, const DV3& b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ DV3 divs(const DV3& a, const Dual& s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ Dual dot(const DV3& a, const DV3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ DV3 cross(const DV3& a, const DV3& b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// Mixed constant/dual forms: a constant operand contributes no tangent, so
// these skip the zero-tangent arithmetic the all-dual forms would execute
// (IEEE rules keep the compiler from folding x * 0 away).
__device__ __forceinline__ DV3 sub(V3 a, const DV3& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ Dual dot(V3 a, const DV3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ Dual dot(const DV3& a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ DV3 cross(V3 a, const DV3& b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ DV3 unit(const DV3& v) {
  const Dual l = gsqrt(dot(v, v));
  if (l.v <= kEps) return lift<DV3>(mk(0.0f, 1.0f, 0.0f));
  return divs(v, l);
}

// ------------------------------------------------------------- vertex math
// Emission MIS weight's light pdf (light_pdf_for_direction,
// ScalarCpuPathTracer.cpp:1120-1138) over a generic origin/direction.
template <class S, class VT>
__device__ __forceinline__ S adj_light_pdf(const DevScene& s, const float* lights, const VT& p, const VT& dir) {
  S total = lift_s(0.0f, S{});
  if (s.light_count == 0u) return total;
  const float inv_n = 1.0f / static_cast<float>(s.light_count);
  for (uint32_t k = 0; k < s.light_count; ++k) {
    const VT tl = sub(ld3(lights + 16u * k), p);
    const S dist = gsqrt(dot(tl, tl));
    if (val(dist) < kEps) continue;
    if (val(dot(divs(tl, dist), dir)) > 0.9999f) total = total + inv_n / (dist * dist + kEps);
  }
  return total;
}

template <class S>
__device__ __forceinline__ S adj_mis(const S& a, const S& b) {
  const S a2 = a * a, b2 = b * b, den = a2 + b2;
  if (val(den) <= 0.0f) return lift_s(1.0f, a);
  return a2 / den;
}

template <class S, class VT>
__device__ __forceinline__ S adj_spot(const float* L, const VT& from_light) {
  const float inner = L[11], outer = L[12];
  if (inner <= -0.999f) return lift_s(1.0f, S{});
  const S cone = dot(unit(from_light), unit(ld3(L + 8)));
  if (val(cone) <= outer) return lift_s(0.0f, S{});
  if (val(cone) >= inner || inner <= outer) return lift_s(1.0f, S{});
  const S t = sclamp((cone - outer) / (inner - outer), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}

// Next-event estimate at `p` (normal n, material m, viewing direction view):
// radiance R (before the MIS weight and the throughput), the shadow segment,
// and P = dR/d(albedo) per channel (R is affine in the albedo).
template <class S, class VT>
struct AdjNee {
  VT radiance;
  V3 origin, dir, p_alb;
  float remain;
};

template <class S, class VT, bool kParity, bool kReplay>
__device__ __forceinline__ bool adj_nee(const DevScene& s, const float* lights, const VT& p, V3 n,
                                        const MaterialRec& m, const S& rough, const VT& view, uint64_t& rng,
                                        uint32_t& flags, AdjNee<S, VT>& q) {
  const uint32_t nl = s.light_count;
  if (nl == 0u) return false;
  uint32_t pick = static_cast<uint32_t>(next01(rng) * static_cast<float>(nl));
  if (pick > nl - 1u) pick = nl - 1u;
  const float* L = lights + 16u * pick;
  V3 lp = ld3(L);
  const float radius = L[7];
  if (radius > 1.0e-5f) {
    const float uz = 1.0f - 2.0f * next01(rng);
    const float r = sqrtf(smax(0.0f, 1.0f - uz * uz));
    const float phi = 6.28318530718f * next01(rng);
    lp = add(lp, mul(mk(r * t_cos<kParity>(phi), uz, r * t_sin<kParity>(phi)), radius));
  }
  const VT tl = sub(lp, p);
  const S d2 = dot(tl, tl);
  const S dist = gsqrt(d2);
  if (kReplay) {
    if (!(flags & kVfNeeValid)) return false;
  } else if (val(dist) < kEps) {
    return false;
  }
  const VT ldir = divs(tl, dist);
  const S cth = dot(n, ldir);
  if (!kReplay && val(cth) <= 0.0f) return false;
  const S sf = adj_spot<S, VT>(L, neg(ldir));
  if (!kReplay && val(sf) <= 0.0f) return false;
  const V3 alb = albedo_effect0(m);
  const VT irr = mul(ld3(L + 3), (L[6] * sf) / (d2 + kEps));
  const float fnl = static_cast<float>(nl);
  // Diffuse term (no mirror or transmissive material reaches here).
  VT acc = mul(mul(mulv(mul(alb, kInvPi), irr), cth), fnl);
  S spec_w = lift_s(0.0f, rough);
  if (val(rough) < 0.65f) {
    const VT hv = unit(add(ldir, unit(view)));
    const S er = smax(0.025f, rough * 1.0f);
    const S a2 = er * er;
    const S pw = sclamp(2.0f / smax(0.0005f, a2 * a2) - 2.0f, 4.0f, 96.0f);
    const S spec = gpow<kParity>(smax(0.0f, dot(n, hv)), pw);
    const S ss = clamp01((1.0f - rough) * 0.8f + m.metallic * 0.45f + m.clearcoat * 0.35f + 0.0f + 0.0f);
    const V3 tint = add(mul(mk(1.0f, 1.0f, 1.0f), 0.88f), mul(alb, 0.12f));
    spec_w = spec * cth * fnl * smax(0.15f, ss);
    acc = add(acc, mul(mulv(tint, irr), spec_w));
  }
  flags |= kVfNeeValid;
  q.radiance = acc;
  const V3 pv = vval(p), nv = vval(n);
  q.origin = add(pv, mul(nv, 0.002f));
  q.dir = vval(ldir);
  q.remain = val(dist) - 0.004f;
  const V3 iv = vval(irr);
  const float kd = val(cth) * fnl * kInvPi, ks = 0.12f * val(spec_w);
  q.p_alb = mk(iv.x * kd + iv.x * ks, iv.y * kd + iv.y * ks, iv.z * kd + iv.z * ks);
  return true;
}

// Phong-lobe direction around refl (sample_phong_lobe, :996-1020).
template <class S, class VT, bool kParity, bool kReplay>
__device__ __forceinline__ VT adj_phong(uint64_t& rng, const VT& refl, const S& ex, V3 n, uint32_t& flags) {
  const float u1 = next01(rng);
  const float u2 = next01(rng);
  const S ct = gpow<kParity>(smax(0.0f, u1), 1.0f / (ex + 1.0f));
  const S sn = gsqrt(smax(0.0f, 1.0f - ct * ct));
  const float phi = 2.0f * kPi * u2;
  bool alt;
  if (kReplay) alt = (flags & kVfFrameAlt) != 0u;
  else alt = !(fabsf(val(refl.z)) < 0.999f);
  if (alt) flags |= kVfFrameAlt;
  const V3 ref = alt ? mk(0.0f, 1.0f, 0.0f) : mk(0.0f, 0.0f, 1.0f);
  const VT t = unit(cross(ref, refl));
  const VT b = cross(refl, t);
  VT out = unit(add(add(mul(t, sn * t_cos<kParity>(phi)), mul(b, sn * t_sin<kParity>(phi))), mul(refl, ct)));
  bool reflected;
  if (kReplay) reflected = (flags & kVfReflected) != 0u;
  else reflected = val(dot(out, n)) <= 0.0f;
  if (reflected) {
    flags |= kVfReflected;
    out = sub(out, mul(n, 2.0f * dot(out, n)));
    bool hemi;
    if (kReplay) hemi = (flags & kVfHemi) != 0u;
    else hemi = val(dot(out, n)) <= 0.0f;
    if (hemi) {
      flags |= kVfHemi;
      return lift<VT>(sample_hemisphere<kParity>(rng, n));
    }
  }
  return out;
}

// What one vertex contributes, generic over float / dual.
template <class S, class VT>
struct AdjVertex {
  VT hp;
  S w_e;              // emission weight: (T * Le) * w_e is added
  bool nee;           // NEE candidate present (kVfNeeValid)
  AdjNee<S, VT> q;
  S w_n;              // NEE MIS weight: (T * R) * w_n is added when visible
  VT out;             // next direction (valid when the material scattered)
  bool scattered;     // a direction was sampled above the surface
};

// Hit shading of one vertex (without the visibility test and the
// throughput update, which the caller does).  rough is the material's
// roughness as a (possibly dual) scalar.
template <class S, class VT, bool kParity, bool kReplay>
__device__ __forceinline__ void adj_vertex(const DevScene& s, const DevSettings& st, const float* lights,
                                           uint32_t depth, const VT& o, const VT& d, const S& ht, V3 gn,
                                           const MaterialRec& m, const S& rough, uint64_t& rng, uint32_t& flags,
                                           AdjVertex<S, VT>& R) {
  R.hp = add(o, mul(d, ht));
  bool entering;
  if (kReplay) entering = (flags & kVfEntering) != 0u;
  else entering = val(dot(d, gn)) < 0.0f;
  if (entering) flags |= kVfEntering;
  const V3 nv = entering ? gn : neg(gn);
  const bool emissive_any = m.emissive.x > 0.0f || m.emissive.y > 0.0f || m.emissive.z > 0.0f;
  const bool emissive_model = m.model == 1u || emissive_any;
  const bool diffuse = val(rough) >= 0.999f;

  if (!st.enable_nee || depth == 0u) {
    R.w_e = lift_s(1.0f, rough);
  } else if (st.enable_mis && emissive_model) {
    const S bp = smax(0.0f, dot(nv, neg(d))) * kInvPi;
    const S lpdf = adj_light_pdf<S, VT>(s, lights, o, d);
    R.w_e = adj_mis(bp, lpdf);
  } else {
    R.w_e = lift_s(0.0f, rough);
  }

  R.nee = false;
  if (st.enable_nee && depth < st.max_depth - 1u) {
    R.nee = adj_nee<S, VT, kParity, kReplay>(s, lights, R.hp, nv, m, rough, neg(d), rng, flags, R.q);
    if (R.nee) {
      if (st.enable_mis) {
        const VT tl = sub(ld3(lights), R.hp);
        const VT ld = unit(tl);
        const S bp = smax(0.0f, dot(nv, ld)) * kInvPi;
        const float lpdf = 1.0f / static_cast<float>(s.light_count);
        R.w_n = adj_mis(lift_s(lpdf, rough), bp);
      } else {
        R.w_n = lift_s(1.0f, rough);
      }
    }
  }

  const VT refl = sub(d, mul(nv, 2.0f * dot(nv, d)));
  if (diffuse) {
    R.out = lift<VT>(sample_hemisphere<kParity>(rng, nv));
  } else {
    const S er = smax(0.025f, rough * 1.0f * 1.0f);
    const S a2 = er * er;
    const S ex = smax(0.0f, 2.0f / (a2 * a2) - 2.0f);
    R.out = adj_phong<S, VT, kParity, kReplay>(rng, refl, ex, nv, flags);
  }
  R.scattered = !(val(dot(R.out, nv)) <= 0.0f);
}

}  // namespace vkptc
