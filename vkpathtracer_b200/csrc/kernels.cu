// kernels.cu -- wavefront path tracing and ray-query kernels (sm_100a).
//
// The integrator restates the reference's scalar CPU tracer:
//   camera_rays / shade_pixel   src/pathtracer/ScalarCpuPathTracer.Render.cpp:55-119, 228-284
//   trace                       src/pathtracer/ScalarCpuPathTracer.cpp:1148-1289
//   sample_direct_light         src/pathtracer/ScalarCpuPathTracer.cpp:1022-1118
//   light_pdf / MisWeight       src/pathtracer/ScalarCpuPathTracer.cpp:1120-1146
//   hemisphere / Phong lobe     src/pathtracer/ScalarCpuPathTracer.cpp:978-1020
//   FilmBuffer add / resolve    src/pathtracer/FilmBuffer.cpp:80-91, 160-214
// split into wavefront stages that exchange structure-of-arrays queues:
//   raygen -> for each depth: extend (closest hit) -> shade (material, NEE
//   set-up, BSDF sample, Russian roulette; appends shadow queries and the next
//   extension queue with warp-aggregated atomics) -> shadow (any hit) ->
//   accumulate into the film in sample order.
// The per-path RNG stream is keyed exactly as the reference keys it, so the
// wavefront reordering does not change any random number a path draws, and
// the stages add radiance terms in the reference's order (emission, then the
// NEE term of the same bounce, then the next bounce).
#include "kernels.cuh"
#include "traverse.cuh"

namespace vkptc {

size_t StackSmemBytes(int block, int cap) { return static_cast<size_t>(block) * cap * sizeof(int2); }

size_t SpillEntries(const LaunchShape& ls) {
  const int extra = ls.stack_cap - ls.smem_entries;
  return extra > 0 ? static_cast<size_t>(ls.grid) * ls.block * extra : 0u;
}

// ============================================================ query sources
// Each source supplies queries to persistent_traverse() and consumes results.
struct RaysSource {   // batched ray queries from a ray array
  const float* rays;
  const float* tmax;
  uint32_t* prim_out;
  float* t_out;
  bool any;
  __device__ __forceinline__ void load(uint32_t j, V3& o, V3& d, float& tm) const {
    const float2* rp = reinterpret_cast<const float2*>(rays + 6ull * j);
    const float2 a = __ldg(rp), b = __ldg(rp + 1), c = __ldg(rp + 2);
    o = mk(a.x, a.y, b.x);
    d = mk(b.y, c.x, c.y);
    tm = tmax ? __ldg(tmax + j) : kInf;
  }
  __device__ __forceinline__ void finish(uint32_t j, float t, uint32_t prim) const {
    prim_out[j] = prim;
    if (t_out) t_out[j] = any ? (prim ? 0.0f : kInf) : t;
  }
};

struct ExtendSource {  // closest hit for the queued paths of a wave
  const uint32_t* q;
  const float4* ray_o;
  const float4* ray_d;
  float2* hit;
  __device__ __forceinline__ void load(uint32_t j, V3& o, V3& d, float& tm) const {
    const uint32_t p = q[j];
    const float4 a = ray_o[p], b = ray_d[p];
    o = mk(a.x, a.y, a.z);
    d = mk(b.x, b.y, b.z);
    tm = kInf;
  }
  __device__ __forceinline__ void finish(uint32_t j, float t, uint32_t prim) const {
    hit[q[j]] = make_float2(t, __uint_as_float(prim));
  }
};

struct ShadowSource {  // any hit for the NEE queries; adds the term when visible
  const float4* sh_o;
  const float4* sh_d;
  const float4* sh_c;
  const uint32_t* sh_path;
  float4* rad;
  __device__ __forceinline__ void load(uint32_t j, V3& o, V3& d, float& tm) const {
    const float4 a = sh_o[j], b = sh_d[j];
    o = mk(a.x, a.y, a.z);
    d = mk(b.x, b.y, b.z);
    tm = a.w;
  }
  __device__ __forceinline__ void finish(uint32_t j, float, uint32_t occluded) const {
    if (occluded) return;
    const uint32_t p = sh_path[j];
    const float4 c = sh_c[j];
    float4 r = rad[p];
    r.x = r.x + c.x;
    r.y = r.y + c.y;
    r.z = r.z + c.z;
    rad[p] = r;
  }
};

template <class Src, bool kAny, bool kStats>
__device__ __forceinline__ void run_persistent(const DevScene& s, const Src& src, uint32_t n, uint32_t* fetch,
                                               int scap, int2* spill, int total, int steps,
                                               unsigned long long* c_nodes, unsigned long long* c_leaves,
                                               unsigned long long* c_tris, unsigned long long* c_rays, uint32_t* err) {
  extern __shared__ int2 smem_stack[];
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const int gstride = static_cast<int>(gridDim.x * blockDim.x);
  TwoLevelStack stk{smem_stack + threadIdx.x, static_cast<int>(blockDim.x), scap,
                    spill ? spill + gtid : nullptr, gstride, total};
  TraceStats st;
  uint32_t lerr = 0u;
  persistent_traverse<Src, kAny, kStats>(s, src, n, fetch, stk, steps, st, lerr);
  if (kStats) {
    warp_count(c_nodes, st.nodes);
    warp_count(c_leaves, st.leaves);
    warp_count(c_tris, st.tris);
    warp_count(c_rays, st.rays);
  }
  if (lerr) atomicOr(err, lerr);
}

// =============================================================== ray queries
template <bool kAny, bool kStats>
__global__ void __launch_bounds__(256) k_trace_rays(DevScene s, RaysSource src, uint32_t n, uint32_t* fetch, int scap,
                                                    int2* spill, int total, int steps, DevCounters* ctr, uint32_t* err) {
  run_persistent<RaysSource, kAny, kStats>(s, src, n, fetch, scap, spill, total, steps, &ctr->nodes, &ctr->leaves,
                                           &ctr->tris, &ctr->ext_rays, err);
}

cudaError_t LaunchTraceRays(const DevScene& s, const float* rays, const float* tmax, uint64_t n, bool any_hit,
                            uint32_t* prim_out, float* t_out, const LaunchShape& ls, DevCounters* ctr,
                            uint32_t* err, uint32_t* fetch) {
  if (n == 0) return cudaSuccess;
  const size_t smem = StackSmemBytes(ls.block, ls.smem_entries);
  cudaError_t e = cudaMemsetAsync(fetch, 0, sizeof(uint32_t), ls.stream);
  if (e != cudaSuccess) return e;
  const RaysSource src{rays, tmax, prim_out, t_out, any_hit};
  const uint32_t n32 = static_cast<uint32_t>(n);
#define VKPTC_TR(A, S) \
  k_trace_rays<A, S><<<ls.grid, ls.block, smem, ls.stream>>>(s, src, n32, fetch, ls.smem_entries, ls.spill, ls.stack_cap, ls.steps, ctr, err)
  if (any_hit) {
    if (ctr) VKPTC_TR(true, true);
    else VKPTC_TR(true, false);
  } else {
    if (ctr) VKPTC_TR(false, true);
    else VKPTC_TR(false, false);
  }
#undef VKPTC_TR
  return cudaGetLastError();
}

// ==================================================================== raygen
template <bool kParity>
__global__ void __launch_bounds__(256) k_raygen(DevScene s, DevSettings st, WaveState w, WaveTile tile) {
  const uint32_t tile_px = tile.w * tile.h;
  const uint32_t n = tile_px * tile.sample_count;
  const uint32_t W = st.width, H = st.height;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t sl = i / tile_px, pl = i - sl * tile_px;
    const uint32_t x = tile.x + pl % tile.w, y = tile.y + pl / tile.w;
    const uint32_t sample = tile.first_sample + sl;
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
    V3 o = s.cam_pos, d = dir;
    if (s.aperture > 0.0f && s.focus > kEps) {
      const float lr = sqrtf(next01(crng));
      const float lphi = 2.0f * kPi * next01(crng);
      const float rr = s.aperture * lr * 1.0f;
      const V3 off = add(mul(s.cam_right, rr * t_cos<kParity>(lphi) * 1.0f), mul(s.cam_up, rr * t_sin<kParity>(lphi)));
      const V3 fp = add(s.cam_pos, mul(dir, s.focus));
      o = add(s.cam_pos, off);
      d = unit(sub(fp, o));
    }
    w.rng[i] = stream_key(st.seed + sample_seed + cam_seed, st.frame, sample, path_id, 0u, 0u, sample_seed);
    w.ray_o[i] = make_float4(o.x, o.y, o.z, 0.0f);
    w.ray_d[i] = make_float4(d.x, d.y, d.z, 0.0f);
    w.thr[i] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    w.rad[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    w.q[0][i] = i;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    w.counts[0] = n;
    w.counts[1] = 0u;
    w.counts[2] = 0u;
    w.counts[3] = 0u;   // extension fetch counter
    w.counts[4] = 0u;   // shadow fetch counter
  }
}

// ==================================================================== extend
// Closest-hit traversal of the current extension queue (persistent warps).
// Zeroes the next queue's and the shadow queue's sizes for the shade stage.
template <bool kStats>
__global__ void __launch_bounds__(256) k_extend(DevScene s, WaveState w, uint32_t cur, int scap, int2* spill,
                                                int total, int steps, DevCounters* ctr, uint32_t* err) {
  const uint32_t n = w.counts[cur];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    w.counts[cur ^ 1u] = 0u;
    w.counts[2] = 0u;
  }
  const ExtendSource src{w.q[cur], w.ray_o, w.ray_d, w.hit};
  run_persistent<ExtendSource, false, kStats>(s, src, n, &w.counts[3], scap, spill, total, steps, &ctr->nodes,
                                              &ctr->leaves, &ctr->tris, &ctr->ext_rays, err);
}

// ===================================================================== shade
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

constexpr uint32_t kSmemLights = 64;   // lights staged in shared memory by the shade stage

template <bool kParity>
__global__ void __launch_bounds__(256) k_shade(DevScene s, DevSettings st, WaveState w, uint32_t cur,
                                               uint32_t depth, DevCounters* ctr) {
  __shared__ float sm_lights[16 * kSmemLights];
  const bool staged = s.light_count <= kSmemLights;
  if (staged) {
    for (uint32_t k = threadIdx.x; k < 16u * s.light_count; k += blockDim.x) sm_lights[k] = s.lights[k];
    __syncthreads();
  }
  const float* lights = staged ? sm_lights : s.lights;
  const uint32_t n = w.counts[cur];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    w.counts[3] = 0u;   // the extension stage of the next depth fetches from 0
    w.counts[4] = 0u;   // the shadow stage of this depth fetches from 0
  }
  const uint32_t* q = w.q[cur];
  uint32_t* qn = w.q[cur ^ 1u];
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const uint32_t j = base + threadIdx.x;
    bool emit_next = false, emit_shadow = false;
    uint32_t p = 0u;
    uint32_t shadow_tests = 0u;
    // shadow query payload
    V3 sh_o = mk(0, 0, 0), sh_d = mk(0, 0, 0), sh_c = mk(0, 0, 0);
    float sh_t = 0.0f;
    if (j < n) {
      p = q[j];
      const float4 o4 = w.ray_o[p], d4 = w.ray_d[p], t4 = w.thr[p], r4 = w.rad[p];
      const float2 h2 = w.hit[p];
      V3 d = mk(d4.x, d4.y, d4.z);
      V3 o = mk(o4.x, o4.y, o4.z);
      V3 thr = mk(t4.x, t4.y, t4.z);
      V3 rad = mk(r4.x, r4.y, r4.z);
      const float segs = r4.w + 1.0f;
      uint64_t rng = w.rng[p];
      const uint32_t prim = __float_as_uint(h2.y);
      if (prim == kMiss) {
        rad = add(rad, mulv(thr, s.env));
      } else {
        const float ht = h2.x;
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
            shadow_tests = 1u;
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
              emit_shadow = true;
              sh_o = nq.origin;
              sh_d = nq.dir;
              sh_t = nq.remain;
              sh_c = c;
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
              const V3 no = add(hp, mul(out, 0.002f));
              w.ray_o[p] = make_float4(no.x, no.y, no.z, 0.0f);
              w.ray_d[p] = make_float4(out.x, out.y, out.z, 0.0f);
              w.thr[p] = make_float4(thr.x, thr.y, thr.z, 0.0f);
              w.rng[p] = rng;
              emit_next = depth + 1u < st.max_depth;
            }
          }
        }
      }
      w.rad[p] = make_float4(rad.x, rad.y, rad.z, segs);
    }
    // Warp-aggregated appends (the whole warp reaches these together).
    const uint32_t slot_n = warp_append(&w.counts[cur ^ 1u], emit_next);
    if (emit_next) qn[slot_n] = p;
    const uint32_t slot_s = warp_append(&w.counts[2], emit_shadow);
    if (emit_shadow) {
      w.sh_path[slot_s] = p;
      w.sh_o[slot_s] = make_float4(sh_o.x, sh_o.y, sh_o.z, sh_t);
      w.sh_d[slot_s] = make_float4(sh_d.x, sh_d.y, sh_d.z, 0.0f);
      w.sh_c[slot_s] = make_float4(sh_c.x, sh_c.y, sh_c.z, 0.0f);
    }
    warp_count(&ctr->shadow_tests, shadow_tests);
  }
}

// ==================================================================== shadow
// Any-hit visibility of the NEE queries (persistent warps); adds the NEE term
// of every visible query to its path's radiance.
template <bool kStats>
__global__ void __launch_bounds__(256) k_shadow(DevScene s, WaveState w, int scap, int2* spill, int total, int steps,
                                                DevCounters* ctr, uint32_t* err) {
  const uint32_t n = w.counts[2];
  const ShadowSource src{w.sh_o, w.sh_d, w.sh_c, w.sh_path, w.rad};
  run_persistent<ShadowSource, true, kStats>(s, src, n, &w.counts[4], scap, spill, total, steps, &ctr->shadow_nodes,
                                             &ctr->shadow_leaves, &ctr->shadow_tris, &ctr->shadow_rays, err);
}

// Scenes with transmissive materials: the reference's closest-hit loop that
// steps through up to 8 transmissive occluders (one query per thread).
template <bool kStats>
__global__ void __launch_bounds__(256) k_shadow_transmissive(DevScene s, WaveState w, int cap, DevCounters* ctr, uint32_t* err) {
  extern __shared__ int2 smem_stack[];
  SmemStack stk{smem_stack + threadIdx.x, static_cast<int>(blockDim.x), cap};
  const uint32_t n = w.counts[2];
  uint32_t local_err = 0u;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const uint32_t j = base + threadIdx.x;
    TraceStats st;
    if (j < n) {
      const float4 o4 = w.sh_o[j], d4 = w.sh_d[j];
      V3 so = mk(o4.x, o4.y, o4.z);
      const V3 sd = mk(d4.x, d4.y, d4.z);
      float remain = o4.w;
      bool visible = true;
      if (!s.has_transmissive) {
        const RayPrep r = prep_ray(so, sd);
        visible = !trace_any<kStats>(s, r, remain, stk, st, local_err);
      } else {
        // Closest-hit loop that steps through up to 8 transmissive occluders
        // (src/pathtracer/ScalarCpuPathTracer.cpp:1067-1087).
        for (uint32_t skips = 0; skips < 8u && remain > 0.004f; ++skips) {
          const RayPrep r = prep_ray(so, sd);
          float t;
          uint32_t prim;
          trace_closest<kStats>(s, r, stk, t, prim, st, local_err);
          if (prim == kMiss || t >= remain) break;
          const uint32_t mat_index = __float_as_uint(__ldg(s.shade + prim).w);
          const uint32_t mi = mat_index < s.material_count - 1u ? mat_index : s.material_count - 1u;
          const float* mm = s.materials + 16u * mi;
          const bool tr = static_cast<uint32_t>(mm[7] + 0.5f) == 5u || mm[10] > 0.05f;
          if (!tr) {
            visible = false;
            break;
          }
          const float adv = t + 0.004f;
          so = add(so, mul(sd, adv));
          remain -= adv;
        }
      }
      if (visible) {
        const uint32_t p = w.sh_path[j];
        const float4 c = w.sh_c[j];
        float4 r = w.rad[p];
        r.x = r.x + c.x;
        r.y = r.y + c.y;
        r.z = r.z + c.z;
        w.rad[p] = r;
      }
    }
    if (kStats) {
      warp_count(&ctr->shadow_nodes, st.nodes);
      warp_count(&ctr->shadow_leaves, st.leaves);
      warp_count(&ctr->shadow_tris, st.tris);
      warp_count(&ctr->shadow_rays, j < n ? 1u : 0u);
    }
  }
  if (local_err) atomicOr(err, local_err);
}

// ================================================================ accumulate
__global__ void __launch_bounds__(256) k_accumulate(DevSettings st, WaveState w, WaveTile tile, Film film,
                                                    DevCounters* ctr) {
  const uint32_t tile_px = tile.w * tile.h;
  for (uint32_t base = blockIdx.x * blockDim.x; base < tile_px; base += gridDim.x * blockDim.x) {
    const uint32_t pl = base + threadIdx.x;
    uint32_t samples = 0u, segs = 0u, dropped = 0u;
    if (pl < tile_px) {
      const uint32_t x = tile.x + pl % tile.w, y = tile.y + pl / tile.w;
      const size_t px = static_cast<size_t>(y) * film.width + x;
      float4 acc = film.sum[px];
      uint32_t cnt = film.count[px];
      for (uint32_t sl = 0; sl < tile.sample_count; ++sl) {
        const float4 r = w.rad[sl * tile_px + pl];
        if (!(isfinite(r.x) && isfinite(r.y) && isfinite(r.z))) {
          ++dropped;   // dropped before the film, like the reference's shade_pixel
          continue;
        }
        float cx = r.x, cy = r.y, cz = r.z;
        if (st.firefly_clamp > 0.0f) {
          cx = smin(cx, st.firefly_clamp);
          cy = smin(cy, st.firefly_clamp);
          cz = smin(cz, st.firefly_clamp);
        }
        acc.x = acc.x + cx;
        acc.y = acc.y + cy;
        acc.z = acc.z + cz;
        ++cnt;
        ++samples;
        segs += static_cast<uint32_t>(r.w);
      }
      film.sum[px] = acc;
      film.count[px] = cnt;
    }
    warp_count(&ctr->samples, samples);
    warp_count(&ctr->rays, segs);
    warp_count(&ctr->dropped, dropped);
  }
}

cudaError_t LaunchWave(const DevScene& s, const DevSettings& st, const WaveState& w, const WaveTile& tile,
                       const Film& film, bool parity, bool stats, const LaunchShape& ls, DevCounters* ctr,
                       uint32_t* err, StageTimer* timer) {
  const size_t smem = StackSmemBytes(ls.block, ls.smem_entries);
  const size_t smem_full = StackSmemBytes(ls.block, ls.stack_cap);
  StageTimer dummy;
  StageTimer& tm = timer ? *timer : dummy;
  tm.begin(0, ls.stream);
  if (parity) k_raygen<true><<<ls.grid, ls.block, 0, ls.stream>>>(s, st, w, tile);
  else k_raygen<false><<<ls.grid, ls.block, 0, ls.stream>>>(s, st, w, tile);
  tm.end(ls.stream);
  uint32_t cur = 0u;
  for (uint32_t depth = 0; depth < st.max_depth; ++depth) {
    tm.begin(1, ls.stream);
    if (stats)
      k_extend<true><<<ls.grid, ls.block, smem, ls.stream>>>(s, w, cur, ls.smem_entries, ls.spill, ls.stack_cap,
                                                            ls.steps, ctr, err);
    else
      k_extend<false><<<ls.grid, ls.block, smem, ls.stream>>>(s, w, cur, ls.smem_entries, ls.spill, ls.stack_cap,
                                                             ls.steps, ctr, err);
    tm.end(ls.stream);
    tm.begin(2, ls.stream);
    if (parity) k_shade<true><<<ls.grid, ls.block, 0, ls.stream>>>(s, st, w, cur, depth, ctr);
    else k_shade<false><<<ls.grid, ls.block, 0, ls.stream>>>(s, st, w, cur, depth, ctr);
    tm.end(ls.stream);
    if (st.enable_nee) {
      tm.begin(3, ls.stream);
      if (s.has_transmissive) {
        if (stats) k_shadow_transmissive<true><<<ls.grid, ls.block, smem_full, ls.stream>>>(s, w, ls.stack_cap, ctr, err);
        else k_shadow_transmissive<false><<<ls.grid, ls.block, smem_full, ls.stream>>>(s, w, ls.stack_cap, ctr, err);
      } else {
        if (stats)
          k_shadow<true><<<ls.grid, ls.block, smem, ls.stream>>>(s, w, ls.smem_entries, ls.spill, ls.stack_cap,
                                                                ls.steps, ctr, err);
        else
          k_shadow<false><<<ls.grid, ls.block, smem, ls.stream>>>(s, w, ls.smem_entries, ls.spill, ls.stack_cap,
                                                                 ls.steps, ctr, err);
      }
      tm.end(ls.stream);
    }
    cur ^= 1u;
  }
  tm.begin(4, ls.stream);
  k_accumulate<<<ls.grid, ls.block, 0, ls.stream>>>(st, w, tile, film, ctr);
  tm.end(ls.stream);
  return cudaGetLastError();
}

// ==================================================================== film
__global__ void k_resolve_hdr(Film film, float* out) {
  const size_t npx = static_cast<size_t>(film.width) * film.height;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < npx;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const uint32_t c = film.count[i];
    const float inv = 1.0f / static_cast<float>(c > 1u ? c : 1u);
    const float4 v = film.sum[i];
    out[3 * i + 0] = v.x * inv;
    out[3 * i + 1] = v.y * inv;
    out[3 * i + 2] = v.z * inv;
  }
}

template <typename K>
static cudaError_t set_smem(K kernel, int bytes) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

cudaError_t ConfigureStackSmem(size_t bytes) {
  const int b = static_cast<int>(bytes);
  cudaError_t e = set_smem(k_trace_rays<true, true>, b);
  if (e == cudaSuccess) e = set_smem(k_trace_rays<true, false>, b);
  if (e == cudaSuccess) e = set_smem(k_trace_rays<false, true>, b);
  if (e == cudaSuccess) e = set_smem(k_trace_rays<false, false>, b);
  if (e == cudaSuccess) e = set_smem(k_extend<true>, b);
  if (e == cudaSuccess) e = set_smem(k_extend<false>, b);
  if (e == cudaSuccess) e = set_smem(k_shadow<true>, b);
  if (e == cudaSuccess) e = set_smem(k_shadow<false>, b);
  if (e == cudaSuccess) e = set_smem(k_shadow_transmissive<true>, b);
  if (e == cudaSuccess) e = set_smem(k_shadow_transmissive<false>, b);
  return e;
}

int ExtendBlocksPerSm(int block, size_t smem) {
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_extend<false>, block, smem) != cudaSuccess) return 1;
  return blocks > 0 ? blocks : 1;
}

cudaError_t LaunchResolveHdr(const Film& film, float* rgb_out, cudaStream_t stream) {
  k_resolve_hdr<<<592, 256, 0, stream>>>(film, rgb_out);
  return cudaGetLastError();
}

}  // namespace vkptc
