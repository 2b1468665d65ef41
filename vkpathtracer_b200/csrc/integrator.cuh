// integrator.cuh -- per-path integrator steps shared by the wavefront stages
// (kernels.cu) and the persistent batched renderer (batch.cu).
//
// Restates the reference's scalar CPU tracer:
//   camera_rays / shade_pixel   src/pathtracer/ScalarCpuPathTracer.Render.cpp:55-119, 228-284
//   trace (one bounce)          src/pathtracer/ScalarCpuPathTracer.cpp:1148-1289
//   sample_direct_light         src/pathtracer/ScalarCpuPathTracer.cpp:1022-1118
//   light_pdf / MisWeight       src/pathtracer/ScalarCpuPathTracer.cpp:1120-1146
//   hemisphere / Phong lobe     src/pathtracer/ScalarCpuPathTracer.cpp:978-1020
// Every expression keeps the reference's operation order (the TUs are built
// with -fmad=false), and the RNG stream of a path is keyed as the reference
// keys it, so a path draws the same numbers in any execution order.
#pragma once

#include "common.cuh"

namespace vkptc {

struct NeeQuery {
  bool valid;      // the reference's NeeResult::valid before the visibility test
  V3 radiance;     // contribution when visible (before the MIS / throughput factors)
  V3 origin, dir;
  float remain;
};

__device__ __forceinline__ float spot_factor(const float* L, V3 from_light) {
  const float inner = L[11], outer = L[12];
  if (inner <= -0.999f) return 1.0f;
  const float cone = dot(unit(from_light), unit(ld3(L + 8)));
  if (cone <= outer) return 0.0f;
  if (cone >= inner || inner <= outer) return 1.0f;
  const float t = sclamp((cone - outer) / (inner - outer), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}

__device__ __forceinline__ V3 albedo_effect0(const MaterialRec& m) {
  return {smin(1.5f, smax(0.0f, m.albedo.x)), smin(1.5f, smax(0.0f, m.albedo.y)),
          smin(1.5f, smax(0.0f, m.albedo.z))};
}

// sample_direct_light without the visibility loop (which the shadow stage runs).
template <bool kParity>
__device__ __forceinline__ NeeQuery nee_setup(const DevScene& s, const float* lights, V3 p, V3 n, uint32_t mat_index,
                                              V3 view, uint64_t& rng) {
  NeeQuery q;
  q.valid = false;
  const uint32_t nl = s.light_count;
  if (nl == 0u) return q;
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
  const V3 tl = sub(lp, p);
  const float d2 = dot(tl, tl);
  const float dist = sqrtf(d2);
  if (dist < kEps) return q;
  const V3 ldir = divs(tl, dist);
  const float cth = dot(n, ldir);
  if (cth <= 0.0f) return q;
  const float sf = spot_factor(L, neg(ldir));
  if (sf <= 0.0f) return q;
  const uint32_t mi = mat_index < s.material_count - 1u ? mat_index : s.material_count - 1u;
  const MaterialRec m = load_material(s.materials + 16u * mi);
  const float rough = clamp01(m.roughness);
  const bool mirror = m.model == 2u || rough <= 0.001f;
  const bool metal = m.model == 4u || m.metallic > 0.65f;
  const bool trans = m.model == 5u || m.transmission > 0.05f;
  const bool coat = m.model == 7u || m.clearcoat > 0.05f;
  const V3 alb = albedo_effect0(m);
  const V3 irr = mul(ld3(L + 3), (L[6] * sf) / (d2 + kEps));
  V3 acc = mk(0.0f, 0.0f, 0.0f);
  const float fnl = static_cast<float>(nl);
  if (!mirror && !trans) acc = add(acc, mul(mul(mulv(mul(alb, kInvPi), irr), cth), fnl));
  if (mirror || metal || coat || trans || rough < 0.65f) {
    const V3 hv = unit(add(ldir, unit(view)));
    const float er = smax(0.025f, rough * (metal ? 0.65f : 1.0f));
    const float a2 = er * er;
    const float pw = sclamp(2.0f / smax(0.0005f, a2 * a2) - 2.0f, 4.0f, 96.0f);
    const float spec = t_pow<kParity>(smax(0.0f, dot(n, hv)), pw);
    const float cv = smax(0.0f, dot(n, unit(view)));
    float f0 = (1.0f - m.ior) / (1.0f + m.ior);
    f0 *= f0;
    const float fr = f0 + (1.0f - f0) * pow5(1.0f - cv);
    const float ss = clamp01((1.0f - rough) * 0.8f + m.metallic * 0.45f + m.clearcoat * 0.35f +
                             (mirror ? 0.75f : 0.0f) + (trans ? fr : 0.0f));
    const V3 tint = add(mul(mk(1.0f, 1.0f, 1.0f), metal ? 0.15f : 0.88f), mul(alb, metal ? 0.85f : 0.12f));
    acc = add(acc, mul(mulv(tint, irr), spec * cth * fnl * smax(0.15f, ss)));
  }
  q.valid = true;
  q.radiance = acc;
  q.origin = add(p, mul(n, 0.002f));
  q.dir = ldir;
  q.remain = dist - 0.004f;
  return q;
}

template <bool kParity>
__device__ __forceinline__ V3 sample_hemisphere(uint64_t& rng, V3 n) {
  const float u1 = next01(rng);
  const float u2 = next01(rng);
  const float r = sqrtf(smax(0.0f, 1.0f - u1));
  const float phi = 2.0f * kPi * u2;
  const V3 loc = mk(r * t_cos<kParity>(phi), r * t_sin<kParity>(phi), sqrtf(smax(0.0f, u1)));
  V3 t = cross((fabsf(n.z) < 0.999f) ? mk(0.0f, 0.0f, 1.0f) : mk(0.0f, 1.0f, 0.0f), n);
  t = unit(t);
  const V3 b = cross(n, t);
  return unit(add(add(mul(t, loc.x), mul(b, loc.y)), mul(n, loc.z)));
}

template <bool kParity>
__device__ __forceinline__ V3 sample_phong(uint64_t& rng, V3 refl, float expo, V3 n) {
  const float u1 = next01(rng);
  const float u2 = next01(rng);
  const float ct = t_pow<kParity>(smax(0.0f, u1), 1.0f / (expo + 1.0f));
  const float sn = sqrtf(smax(0.0f, 1.0f - ct * ct));
  const float phi = 2.0f * kPi * u2;
  const V3 ref = (fabsf(refl.z) < 0.999f) ? mk(0.0f, 0.0f, 1.0f) : mk(0.0f, 1.0f, 0.0f);
  const V3 t = unit(cross(ref, refl));
  const V3 b = cross(refl, t);
  V3 out = unit(add(add(mul(t, sn * t_cos<kParity>(phi)), mul(b, sn * t_sin<kParity>(phi))), mul(refl, ct)));
  if (dot(out, n) <= 0.0f) {
    out = sub(out, mul(n, 2.0f * dot(out, n)));
    if (dot(out, n) <= 0.0f) return sample_hemisphere<kParity>(rng, n);
  }
  return out;
}

__device__ __forceinline__ float mis_weight(float a, float b) {
  const float a2 = a * a, b2 = b * b, den = a2 + b2;
  if (den <= 0.0f) return 1.0f;
  return a2 / den;
}

__device__ __forceinline__ float light_pdf_dir(const DevScene& s, const float* lights, V3 p, V3 dir) {
  if (s.light_count == 0u) return 0.0f;
  const float inv_n = 1.0f / static_cast<float>(s.light_count);
  float total = 0.0f;
  for (uint32_t k = 0; k < s.light_count; ++k) {
    const V3 tl = sub(ld3(lights + 16u * k), p);
    const float dist = sqrtf(dot(tl, tl));
    if (dist < kEps) continue;
    if (dot(divs(tl, dist), dir) > 0.9999f) total += inv_n / (dist * dist + kEps);
  }
  return total;
}


// Camera ray and the path's RNG state for pixel (x, y), sample `sample`.
template <bool kParity>
__device__ __forceinline__ void camera_path(const DevScene& s, const DevSettings& st, uint32_t x, uint32_t y,
                                            uint32_t sample, V3& o, V3& d, uint64_t& path_rng) {
  const uint32_t W = st.width, H = st.height;
  const uint64_t sample_seed = (static_cast<uint64_t>(y) << 32) | x;
  const uint64_t path_id = sample_seed + sample + st.frame;
  // Camera stream: pixel y*W+x, the path id truncated to 32 bits, dimension 0.
  uint64_t crng = stream_key(st.seed, st.frame, sample, static_cast<uint32_t>(path_id), 0u, 0u,
                               static_cast<uint64_t>(y) * W + x);
  const float fx = (static_cast<float>(x) + next01(crng)) / static_cast<float>(W > 1u ? W : 1u);
  const float fy = (static_cast<float>(y) + next01(crng)) / static_cast<float>(H > 1u ? H : 1u);
  const uint64_t cam_seed = static_cast<uint64_t>(next01(crng) * static_cast<float>(0xffffu));
  const float aspect = static_cast<float>(W) / smax(1.0f, static_cast<float>(H));
  const float nx = (2.0f * fx - 1.0f) * aspect * s.tan_half_fov;
  const float ny = (1.0f - 2.0f * fy) * s.tan_half_fov;
  const V3 dir = unit(add(add(s.cam_fwd, mul(s.cam_right, nx)), mul(s.cam_up, ny)));
  o = s.cam_pos;
  d = dir;
  if (s.aperture > 0.0f && s.focus > kEps) {
    const float lr = sqrtf(next01(crng));
    const float lphi = 2.0f * kPi * next01(crng);
    const float rr = s.aperture * lr * 1.0f;
    const V3 off = add(mul(s.cam_right, rr * t_cos<kParity>(lphi) * 1.0f), mul(s.cam_up, rr * t_sin<kParity>(lphi)));
    const V3 fp = add(s.cam_pos, mul(dir, s.focus));
    o = add(s.cam_pos, off);
    d = unit(sub(fp, o));
  }
  path_rng = stream_key(st.seed + sample_seed + cam_seed, st.frame, sample, path_id, 0u, 0u, sample_seed);
}

// Path registers between bounces.
struct PathRegs {
  V3 o, d, thr, rad;
  float segs;
  uint64_t rng;
};

// Result of shading one hit (or miss) at `depth`.
struct ShadeOut {
  bool next;          // the path continues with a new extension ray (o, d updated)
  bool shadow;        // a shadow query is pending (its term is added when visible)
  uint32_t shadow_tests;
  V3 sh_o, sh_d, sh_c;
  float sh_t;
};

// One bounce of the reference's trace loop for a path whose extension ray
// (P.o, P.d) hit primitive `prim` at distance `ht` (prim == kMiss: no hit).
template <bool kParity>
__device__ __forceinline__ ShadeOut shade_bounce(const DevScene& s, const DevSettings& st, const float* lights,
                                               uint32_t depth, PathRegs& P, float ht, uint32_t prim) {
  ShadeOut R;
  R.next = false;
  R.shadow = false;
  R.shadow_tests = 0u;
  R.sh_o = R.sh_d = R.sh_c = mk(0.0f, 0.0f, 0.0f);
  R.sh_t = 0.0f;
  const V3 o = P.o, d = P.d;
  V3 thr = P.thr, rad = P.rad;
  uint64_t rng = P.rng;
  P.segs = P.segs + 1.0f;
  if (prim == kMiss) {
    rad = add(rad, mulv(thr, s.env));
  } else {
    const V3 hp = add(o, mul(d, ht));
    const float4 sh = __ldg(s.shade + prim);
    const V3 gn = mk(sh.x, sh.y, sh.z);
    const uint32_t mat_index = __float_as_uint(sh.w);
    const bool entering = dot(d, gn) < 0.0f;
    const V3 nrm = entering ? gn : neg(gn);
    const uint32_t mi = mat_index < s.material_count - 1u ? mat_index : s.material_count - 1u;
    const MaterialRec m = load_material(s.materials + 16u * mi);
    const V3 alb = albedo_effect0(m);
    const float rough = clamp01(m.roughness);
    const bool emissive_any = m.emissive.x > 0.0f || m.emissive.y > 0.0f || m.emissive.z > 0.0f;
    const bool emissive_model = m.model == 1u || emissive_any;
    const bool mirror = m.model == 2u || rough <= 0.001f;
    const bool metal = m.model == 4u || m.metallic > 0.65f;
    const bool trans = m.model == 5u || m.transmission > 0.05f;
    const bool diffuse = rough >= 0.999f && !mirror && !metal && !trans;
    const bool sheen = m.model == 6u;
    const bool coat = m.model == 7u || m.clearcoat > 0.05f;
    const bool toon = m.model == 8u;

    if (!st.enable_nee || depth == 0u) {
      rad = add(rad, mulv(thr, m.emissive));
    } else if (st.enable_mis && emissive_model) {
      const float bp = smax(0.0f, dot(nrm, neg(d))) * kInvPi;
      const float lpdf = light_pdf_dir(s, lights, o, d);
      rad = add(rad, mul(mulv(thr, m.emissive), mis_weight(bp, lpdf)));
    }

    if (st.enable_nee && depth < st.max_depth - 1u) {
      const NeeQuery nq = nee_setup<kParity>(s, lights, hp, nrm, mat_index, neg(d), rng);
      if (nq.valid) {
        R.shadow_tests = 1u;
        V3 c;
        if (st.enable_mis) {
          const V3 tl = sub(ld3(lights), hp);
          const V3 ld = unit(tl);
          const float bp = smax(0.0f, dot(nrm, ld)) * kInvPi;
          const float lpdf = 1.0f / static_cast<float>(s.light_count);
          c = mul(mulv(thr, nq.radiance), mis_weight(lpdf, bp));
        } else {
          c = mulv(thr, nq.radiance);
        }
        if (nq.remain > 0.004f) {
          R.shadow = true;
          R.sh_o = nq.origin;
          R.sh_d = nq.dir;
          R.sh_t = nq.remain;
          R.sh_c = c;
        } else {
          rad = add(rad, c);   // no visibility test runs for so short a segment
        }
      }
    }

    V3 out;
    bool refracted = false;
    const V3 refl = sub(d, mul(nrm, 2.0f * dot(nrm, d)));
    if (mirror) {
      out = refl;
    } else if (trans) {
      const float ct = smax(0.0f, dot(nrm, neg(d)));
      const float si0 = smax(1.01f, m.ior);
      float r0 = (1.0f - si0) / (1.0f + si0);
      r0 *= r0;
      const float mm = 1.0f - smin(1.0f, smax(0.0f, ct));
      const float fres = r0 + (1.0f - r0) * mm * mm * mm * mm * mm;
      if (next01(rng) < smin(0.98f, fres + m.clearcoat * 0.015f)) {
        out = refl;
      } else {
        const float si = smax(1.01f, m.ior);
        const float eta = entering ? (1.0f / si) : si;
        const float ci = smin(1.0f, smax(0.0f, dot(neg(d), nrm)));
        const float k = 1.0f - eta * eta * (1.0f - ci * ci);
        if (k < 0.0f) {
          out = refl;
        } else {
          out = unit(add(mul(d, eta), mul(nrm, eta * ci - sqrtf(k))));
          if (dot(out, out) <= 1.0e-8f) out = refl;
          else refracted = true;
        }
      }
    } else if (diffuse || toon) {
      out = sample_hemisphere<kParity>(rng, nrm);
    } else {
      const float er = smax(0.025f, rough * (metal ? 0.75f : 1.0f) * (coat ? 0.65f : 1.0f));
      const float a2 = er * er;
      const float ex = smax(0.0f, 2.0f / (a2 * a2) - 2.0f);
      out = sample_phong<kParity>(rng, refl, ex, nrm);
      if (sheen && next01(rng) < m.sheen * 0.35f) out = sample_hemisphere<kParity>(rng, nrm);
    }
    bool alive = trans || !(dot(out, nrm) <= 0.0f);
    if (alive) {
      V3 wgt = alb;
      if (metal || mirror) {
        wgt = mul(alb, 0.65f + 0.35f * m.metallic);
      } else if (trans) {
        const float ts = clamp01(m.alpha) * m.transmission;
        wgt = add(mul(mk(1.0f, 1.0f, 1.0f), 1.0f - ts), mul(alb, ts));
        if (refracted) wgt = mul(wgt, smax(0.55f, m.transmission));
      }
      if (toon) wgt = mul(wgt, dot(out, nrm) > 0.55f ? 1.0f : 0.45f);
      thr = mulv(thr, wgt);
      const float tmx = smax(thr.x, smax(thr.y, thr.z));
      if (tmx < 0.001f) {
        alive = false;
      } else {
        const float rr = smin(st.rr_max, smax(st.rr_min, tmx));
        if (depth >= st.rr_start && next01(rng) > rr) {
          alive = false;
        } else {
          thr = divs(thr, rr);
          P.o = add(hp, mul(out, 0.002f));
          P.d = out;
          R.next = depth + 1u < st.max_depth;
        }
      }
    }
  }
  P.thr = thr;
  P.rad = rad;
  P.rng = rng;
  return R;
}

}  // namespace vkptc
