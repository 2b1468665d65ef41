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
#include "sdf.cuh"

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

// ---------------------------------------------------- procedural effects
// apply_material_effect (src/pathtracer/ScalarCpuPathTracer.cpp:186-355):
// the albedo a surface shows at point p (shading normal n, ray direction
// `in`), then clamped to [0, 1.5].  Effect 0 is the plain clamped albedo;
// 1..19 are the reference's procedural looks (fibres, cells, cracks, veins,
// oxidation, grain, subsurface tint, thin film, check mask, hot surface,
// streaks, retro sparkle, wave normal hint, x-ray rim, smoke bands and four
// wood species), evaluated in the reference's operation order.
template <bool kParity>
__device__ __forceinline__ float fx_hash(float x, float y, float z, float seed) {
  const float v = t_sin<kParity>(x * 12.9898f + y * 78.233f + z * 37.719f + seed * 19.19f) * 43758.5453f;
  return v - floorf(v);
}
__device__ __forceinline__ float fx_smooth(float e0, float e1, float x) {
  const float t = clamp01((x - e0) / smax(1.0e-6f, e1 - e0));
  return t * t * (3.0f - 2.0f * t);
}
__device__ __forceinline__ V3 fx_lin(V3 a, float sa, V3 b, float sb) { return add(mul(a, sa), mul(b, sb)); }

template <bool kParity>
__device__ __noinline__ V3 fx_wood(V3 base, V3 p, float roughness, float clearcoat, uint32_t style) {
  const float rough = clamp01(roughness), coat = clamp01(clearcoat);
  const float polish = clamp01(coat * (1.25f - rough * 0.75f));
  const float par = style == 17u ? 1.0f : 0.0f, wal = style == 18u ? 1.0f : 0.0f, san = style == 19u ? 1.0f : 0.0f;
  const float pw = 0.40f + 0.16f * par + 0.08f * polish - 0.18f * wal;
  const float pl = 1.15f + 0.85f * par + 0.55f * polish - 0.55f * wal;
  const float u = (p.x + san * p.y * 0.35f) / smax(0.12f, pw);
  const float v = (p.z + wal * p.y * 0.70f + san * p.x * 0.22f) / smax(0.30f, pl);
  const float cu = floorf(u), cv = floorf(v);
  const float lu = u - cu, lv = v - cv;
  const float seed = fx_hash<kParity>(cu, cv, 0.0f, 16.0f);
  const float macro = fx_hash<kParity>(floorf(p.x * 3.7f), floorf(p.y * 3.7f), floorf(p.z * 3.7f),
                                       31.0f + static_cast<float>(style));
  const float micro = fx_hash<kParity>(floorf(p.x * 34.0f), floorf(p.y * 34.0f), floorf(p.z * 34.0f),
                                       47.0f + static_cast<float>(style));
  const bool rot = par > 0.5f && fmodf(cu + cv, 2.0f) >= 1.0f;
  const float along = rot ? lv : lu, across = rot ? lu : lv;
  const float wobble = (macro - 0.5f) * (0.06f + rough * 0.12f + wal * 0.08f + san * 0.04f);
  const float wa = along + wobble + t_sin<kParity>(across * 6.0f + seed * 5.0f) * 0.018f;
  const float freq = 12.0f + rough * 8.0f + wal * 22.0f + san * 36.0f;
  const float wave = t_sin<kParity>((wa * freq + seed * 6.2831853f) +
                                    t_sin<kParity>(across * (6.0f + rough * 8.0f) + seed * 4.0f) *
                                        (0.25f + rough * 0.45f + wal * 0.45f));
  const float fine = t_sin<kParity>(wa * (55.0f + rough * 55.0f + san * 110.0f) + across * (9.0f + wal * 25.0f) +
                                    seed * 12.0f);
  const float fw = 0.10f + rough * 0.18f + wal * 0.18f + san * 0.22f;
  const float ring = fx_smooth(-0.35f + polish * 0.18f, 0.82f, wave) * (1.0f - fw) + (0.5f + 0.5f * fine) * fw;
  const float su = smin(lu, 1.0f - lu), sv = smin(lv, 1.0f - lv);
  const float seam = (1.0f - san) * (1.0f - fx_smooth(0.0f, 0.028f + polish * 0.018f, smin(su, sv)));
  const V3 dark = mul(base, 0.46f - rough * 0.10f - wal * 0.18f);
  const V3 amber = add(mul(base, 1.14f + coat * 0.22f + san * 0.18f),
                       mk(0.08f + san * 0.18f, 0.055f + san * 0.06f, 0.025f));
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

template <bool kParity>
__device__ __noinline__ V3 fx_albedo(const MaterialRec& m, V3 p, V3 n, V3 in) {
  V3 c = m.albedo;
  const uint32_t fx = m.effect;
  const float h = fx_hash<kParity>(p.x, p.y, p.z, static_cast<float>(fx));
  const float facing = dot(n, neg(in));
  switch (fx) {
    case 1u: {
      const float g = smax(0.0f, 1.0f - fabsf(facing));
      c = fx_lin(c, 0.65f + 0.25f * h, mk(0.25f, 0.22f, 0.28f), g * g * (0.4f + m.sheen));
      break;
    }
    case 2u:
      c = mul(c, 0.45f + 0.55f * (0.5f + 0.5f * t_sin<kParity>(p.x * 7.0f + p.z * 5.0f + h * 6.0f)));
      break;
    case 3u:
      c = mul(c, h > 0.72f ? 0.18f : 1.0f);
      break;
    case 4u: {
      const float vein = 0.5f + 0.5f * t_sin<kParity>((p.x + p.y * 0.4f + p.z * 0.7f) * 9.0f + h * 3.0f);
      c = fx_lin(c, 0.55f + 0.45f * vein, mk(0.18f, 0.20f, 0.23f), 1.0f - vein);
      break;
    }
    case 5u:
      c = fx_lin(c, 0.55f + 0.35f * h, mk(0.45f, 0.16f, 0.04f), 0.25f + 0.25f * h);
      break;
    case 6u:
      c = mul(c, 0.65f + 0.35f * h);
      break;
    case 7u:
      c = fx_lin(c, 0.78f, mk(1.0f, 0.62f, 0.42f), 0.16f);
      break;
    case 8u:
      c = fx_lin(c, 0.55f, mk(0.35f + 0.45f * h, 0.25f + 0.35f * (1.0f - h), 0.85f), 0.45f);
      break;
    case 9u:
      c = mul(c, fmodf(floorf(p.x * 4.0f) + floorf(p.z * 4.0f), 2.0f) < 0.5f ? 1.0f : 0.28f);
      break;
    case 10u:
      c = fx_lin(c, 0.45f, mk(1.0f, 0.35f + 0.3f * h, 0.08f), 0.55f);
      break;
    case 11u:
      c = mul(c, 0.55f + 0.45f * (0.5f + 0.5f * t_sin<kParity>(p.y * 18.0f + h * 5.0f)));
      break;
    case 12u: {
      const float f2 = smax(0.0f, facing) * smax(0.0f, facing);
      c = add(c, mul(mk(0.55f, 0.65f, 0.95f), f2 * f2 * f2));
      break;
    }
    case 13u:
      c = mul(c, 0.65f + 0.35f * fabsf(t_sin<kParity>(p.x * 10.0f) * t_cos<kParity>(p.z * 10.0f)));
      break;
    case 14u:
      c = mul(mk(0.15f, 0.75f, 1.0f), 0.2f + 0.8f * t_pow<kParity>(smax(0.0f, 1.0f - fabsf(facing)), 0.8f));
      break;
    case 15u: {
      const float bands = 0.5f + 0.5f * t_sin<kParity>(p.y * 11.0f + p.x * 3.0f + h * 7.0f);
      const float rim = t_pow<kParity>(smax(0.0f, 1.0f - fabsf(facing)), 1.5f);
      c = fx_lin(c, 0.25f + 0.45f * bands, mk(0.48f, 0.56f, 0.68f), 0.18f + 0.32f * rim);
      break;
    }
    case 16u:
    case 17u:
    case 18u:
    case 19u:
      c = fx_wood<kParity>(c, p, m.roughness, m.clearcoat, fx);
      break;
    default:
      break;
  }
  return mk(smin(1.5f, smax(0.0f, c.x)), smin(1.5f, smax(0.0f, c.y)), smin(1.5f, smax(0.0f, c.z)));
}

// kEffects = false compiles shading for scenes without procedural effects
// (every material's effect is 0), which keeps that code small.
template <bool kParity, bool kEffects>
__device__ __forceinline__ V3 surface_albedo(const MaterialRec& m, V3 p, V3 n, V3 in) {
  if constexpr (kEffects) return m.effect == 0u ? albedo_effect0(m) : fx_albedo<kParity>(m, p, n, in);
  else return albedo_effect0(m);
}

// ---------------------------------------------------- environment
// SampleSceneEnvironment (src/pathtracer/PathTracer.cpp:213-272): the constant
// environment colour, or a bilinear lookup in the equirectangular map
// (u from atan2(z, x), v from acos(y), texel grid wrapped in u and clamped
// in v), scaled.
template <bool kParity>
__device__ __forceinline__ V3 environment(const DevScene& s, V3 dir_in) {
  if (s.env_map == nullptr) return s.env;
  const float len_sq = dir_in.x * dir_in.x + dir_in.y * dir_in.y + dir_in.z * dir_in.z;
  if (len_sq <= 1.0e-12f) return s.env;
  const float inv_len = 1.0f / sqrtf(len_sq);
  const V3 dir = mk(dir_in.x * inv_len, dir_in.y * inv_len, dir_in.z * inv_len);
  float u = 0.5f + t_atan2<kParity>(dir.z, dir.x) * 0.15915494309189533577f;
  u -= floorf(u);
  const float v = t_acos<kParity>(sclamp(dir.y, -1.0f, 1.0f)) * 0.31830988618379067154f;
  const uint32_t W = s.env_w, H = s.env_h;
  const float x = u * static_cast<float>(W);
  const float y = sclamp(v, 0.0f, 1.0f) * static_cast<float>(H - 1u);
  const uint32_t x0 = static_cast<uint32_t>(floorf(x)) % W;
  const uint32_t x1 = (x0 + 1u) % W;
  const uint32_t y0 = static_cast<uint32_t>(floorf(y));
  const uint32_t y1 = y0 + 1u < H - 1u ? y0 + 1u : H - 1u;
  const float tx = x - floorf(x);
  const float ty = y - floorf(y);
  const float4 c00 = __ldg(s.env_map + static_cast<size_t>(y0) * W + x0);
  const float4 c10 = __ldg(s.env_map + static_cast<size_t>(y0) * W + x1);
  const float4 c01 = __ldg(s.env_map + static_cast<size_t>(y1) * W + x0);
  const float4 c11 = __ldg(s.env_map + static_cast<size_t>(y1) * W + x1);
  const V3 top = mk(c00.x + (c10.x - c00.x) * tx, c00.y + (c10.y - c00.y) * tx, c00.z + (c10.z - c00.z) * tx);
  const V3 bot = mk(c01.x + (c11.x - c01.x) * tx, c01.y + (c11.y - c01.y) * tx, c01.z + (c11.z - c01.z) * tx);
  V3 c = mk(top.x + (bot.x - top.x) * ty, top.y + (bot.y - top.y) * ty, top.z + (bot.z - top.z) * ty);
  c.x *= s.env_scale.x;
  c.y *= s.env_scale.y;
  c.z *= s.env_scale.z;
  return c;
}

// sample_direct_light without the visibility loop (which the shadow stage runs).
template <bool kParity, bool kEffects = true, bool kExotic = true>
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
    const float2 cs = t_cos_sin<kParity>(phi);
    lp = add(lp, mul(mk(r * cs.x, uz, r * cs.y), radius));
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
  const bool trans = kExotic && (m.model == 5u || m.transmission > 0.05f);
  const bool coat = kExotic && (m.model == 7u || m.clearcoat > 0.05f);
  const V3 alb = surface_albedo<kParity, kEffects>(m, p, n, neg(ldir));
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
  const float2 cs = t_cos_sin<kParity>(phi);
  const V3 loc = mk(r * cs.x, r * cs.y, sqrtf(smax(0.0f, u1)));
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
  const float2 cs = t_cos_sin<kParity>(phi);
  V3 out = unit(add(add(mul(t, sn * cs.x), mul(b, sn * cs.y)), mul(refl, ct)));
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
    // Polygonal aperture: the lens radius shrinks per blade sector
    // (ScalarCpuPathTracer::camera_rays, src/pathtracer/ScalarCpuPathTracer.Render.cpp:94-105).
    float boundary = 1.0f;
    if (s.iris_on) {
      const float local_phi = lphi - s.iris_rot;
      const float wrapped = local_phi - s.iris_sector * floorf(local_phi / s.iris_sector);
      const float centered = wrapped > s.iris_sector * 0.5f ? wrapped - s.iris_sector : wrapped;
      const float polygon = s.iris_cos_half / smax(0.1f, t_cos<kParity>(centered));
      boundary = polygon * s.iris_one_minus_round + s.iris_round;
    }
    const float rr = s.aperture * lr * boundary;
    const V3 off = add(mul(s.cam_right, rr * t_cos<kParity>(lphi) * s.squeeze), mul(s.cam_up, rr * t_sin<kParity>(lphi)));
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
  SdfCount sdf;       // SDF primitive tests of this bounce (extension and shadow)
};

// One bounce of the reference's trace loop for a path whose extension ray
// (P.o, P.d) hit triangle `prim` at distance `ht` (prim == kMiss: no triangle
// hit).  The scene's SDF primitives are tested here, after the triangles, as
// intersect_scene does; an SDF hit becomes prim = kSdfTag | index.  In a
// scene without transmissive materials the shadow query's SDF test runs here
// too: a query an SDF occludes is never queued for the triangle any-hit.
// kSdf = false compiles every SDF step out (for launches in which no scene
// has SDF primitives), and kExotic = false the transmissive, clear-coat,
// sheen and toon branches and the environment-map lookup (for launches whose
// scenes have none: the host classifies the material tables with the same
// tests), which keeps the shading kernel's hot code compact.
// sdf_staged: a load-balanced stage has already folded the SDF hits into
// (ht, prim) and tests the shadow queries itself (the loop driver).
template <bool kParity, bool kEffects = true, bool kSdf = true, bool kExotic = true>
__device__ __forceinline__ ShadeOut shade_bounce(const DevScene& s, const DevSettings& st, const float* lights,
                                               uint32_t depth, PathRegs& P, float ht, uint32_t prim,
                                               bool sdf_staged = false) {
  ShadeOut R;
  if constexpr (kSdf) {
    if (s.sdf_count != 0u && !sdf_staged) sdf_closest(s.sdf, s.sdf_count, P.o, P.d, ht, prim, R.sdf);
  }
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
    rad = add(rad, mulv(thr, kExotic ? environment<kParity>(s, d) : s.env));
  } else {
    const V3 hp = add(o, mul(d, ht));
    V3 gn;
    uint32_t mat_index;
    if (kSdf && (prim & kSdfTag)) {
      gn = sdf_hit_normal(s.sdf, prim & ~kSdfTag, o, d, ht);
      mat_index = sdf_material(s.sdf, prim & ~kSdfTag);
    } else {
      const float4 sh = __ldg(s.shade + prim);
      gn = mk(sh.x, sh.y, sh.z);
      mat_index = __float_as_uint(sh.w);
    }
    const bool entering = dot(d, gn) < 0.0f;
    const V3 nrm = entering ? gn : neg(gn);
    const uint32_t mi = mat_index < s.material_count - 1u ? mat_index : s.material_count - 1u;
    const MaterialRec m = load_material(s.materials + 16u * mi);
    const V3 alb = surface_albedo<kParity, kEffects>(m, hp, nrm, d);
    const float rough = clamp01(m.roughness);
    const bool emissive_any = m.emissive.x > 0.0f || m.emissive.y > 0.0f || m.emissive.z > 0.0f;
    const bool emissive_model = m.model == 1u || emissive_any;
    const bool mirror = m.model == 2u || rough <= 0.001f;
    const bool metal = m.model == 4u || m.metallic > 0.65f;
    const bool trans = kExotic && (m.model == 5u || m.transmission > 0.05f);
    const bool diffuse = rough >= 0.999f && !mirror && !metal && !trans;
    const bool sheen = kExotic && m.model == 6u;
    const bool coat = kExotic && (m.model == 7u || m.clearcoat > 0.05f);
    const bool toon = kExotic && m.model == 8u;

    if (!st.enable_nee || depth == 0u) {
      rad = add(rad, mulv(thr, m.emissive));
    } else if (st.enable_mis && emissive_model) {
      const float bp = smax(0.0f, dot(nrm, neg(d))) * kInvPi;
      const float lpdf = light_pdf_dir(s, lights, o, d);
      rad = add(rad, mul(mulv(thr, m.emissive), mis_weight(bp, lpdf)));
    }

    if (st.enable_nee && depth < st.max_depth - 1u) {
      const NeeQuery nq = nee_setup<kParity, kEffects, kExotic>(s, lights, hp, nrm, mat_index, neg(d), rng);
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
          R.shadow = !(kSdf && s.sdf_count != 0u && !s.has_transmissive && !sdf_staged &&
                       sdf_any(s.sdf, s.sdf_count, nq.origin, nq.dir, nq.remain, R.sdf));
          R.sh_o = nq.origin;
          R.sh_d = nq.dir;
          R.sh_t = nq.remain;
          R.sh_c = c;
        } else {
          rad = add(rad, c);   // no visibility test runs for so short a segment
        }
      }
    }

    // The last bounce samples no continuation: whatever it drew, the path ends
    // with the radiance it has (the reference draws and discards it).
    if (depth + 1u >= st.max_depth) {
      P.thr = thr;
      P.rad = rad;
      P.rng = rng;
      return R;
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
