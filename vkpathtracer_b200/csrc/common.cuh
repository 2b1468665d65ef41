// common.cuh -- device records, float helpers and the counter-based RNG.
//
// All translation units of libvkpt_cuda are compiled with -fmad=false and
// IEEE division/sqrt: the integrator must evaluate every expression in the
// reference CPU tracer's operation order (an x86-64 -O2 build, which never
// contracts a*b+c), so hit ids and primary-path radiance are bit-exact.
// Fused multiply-adds appear only where written explicitly (__fmaf_rn).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace vkptc {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.31830988618f;
constexpr float kEps = 1e-4f;
constexpr uint32_t kMiss = 0xFFFFFFFFu;

// --------------------------------------------------------------- float3 math
struct V3 {
  float x, y, z;
};
__host__ __device__ __forceinline__ V3 mk(float x, float y, float z) { return V3{x, y, z}; }
__host__ __device__ __forceinline__ V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ __forceinline__ V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ __forceinline__ V3 neg(V3 a) { return {-a.x, -a.y, -a.z}; }
__host__ __device__ __forceinline__ V3 mul(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__host__ __device__ __forceinline__ V3 mulv(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__host__ __device__ __forceinline__ V3 divs(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__host__ __device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// std::max / std::min / std::clamp with their exact comparison order.
__host__ __device__ __forceinline__ float smax(float a, float b) { return (a < b) ? b : a; }
__host__ __device__ __forceinline__ float smin(float a, float b) { return (b < a) ? b : a; }
__host__ __device__ __forceinline__ float sclamp(float v, float lo, float hi) {
  return (v < lo) ? lo : ((hi < v) ? hi : v);
}
// normalize(): divide by the length; (0,1,0) when the length is <= 1e-4.
__host__ __device__ __forceinline__ V3 unit(V3 v) {
  const float l = sqrtf(dot(v, v));
  if (l <= kEps) return {0.0f, 1.0f, 0.0f};
  return divs(v, l);
}
__device__ __forceinline__ bool finitef(float v) { return isfinite(v); }
__device__ __forceinline__ float clamp01(float v) {
  if (!isfinite(v)) return 0.0f;
  return smin(1.0f, smax(0.0f, v));
}
__host__ __device__ __forceinline__ float pow5(float v) {
  const float v2 = v * v;
  return v2 * v2 * v;
}
__device__ __forceinline__ V3 ld3(const float* p) { return {p[0], p[1], p[2]}; }

// Transcendentals.  Parity mode evaluates in FP64 and rounds once, which
// lands on the correctly rounded float result (as glibc's sinf/cosf/powf do
// to within their sub-ulp error); fast mode uses the FP32 library calls.
// The FP64 routines are long, so each is one out-of-line function shared by
// all call sites of a kernel: the shading code stays small enough for the
// instruction cache.
static __device__ __noinline__ float parity_sin(float x) { return static_cast<float>(sin(static_cast<double>(x))); }
static __device__ __noinline__ float parity_cos(float x) { return static_cast<float>(cos(static_cast<double>(x))); }
static __device__ __noinline__ float parity_pow(float x, float y) {
  return static_cast<float>(pow(static_cast<double>(x), static_cast<double>(y)));
}
static __device__ __noinline__ float parity_atan2(float y, float x) {
  return static_cast<float>(atan2(static_cast<double>(y), static_cast<double>(x)));
}
static __device__ __noinline__ float parity_acos(float x) { return static_cast<float>(acos(static_cast<double>(x))); }
template <bool kParity>
__device__ __forceinline__ float t_atan2(float y, float x) {
  if constexpr (kParity) return parity_atan2(y, x);
  else return atan2f(y, x);
}
template <bool kParity>
__device__ __forceinline__ float t_acos(float x) {
  if constexpr (kParity) return parity_acos(x);
  else return acosf(x);
}
template <bool kParity>
__device__ __forceinline__ float t_sin(float x) {
  if constexpr (kParity) return parity_sin(x);
  else return sinf(x);
}
template <bool kParity>
__device__ __forceinline__ float t_cos(float x) {
  if constexpr (kParity) return parity_cos(x);
  else return cosf(x);
}
// cos and sin of one angle.  Parity mode: one FP64 sincos rounded to float
// per result, which gives the FP64 sin and cos rounded once, like t_cos/t_sin.
#ifndef VKPTC_SINCOS
#define VKPTC_SINCOS 1
#endif
#if VKPTC_SINCOS
static __device__ __noinline__ float2 parity_cos_sin(float x) {
  double s = 0.0, c = 0.0;
  sincos(static_cast<double>(x), &s, &c);
  return make_float2(static_cast<float>(c), static_cast<float>(s));
}
#endif
template <bool kParity>
__device__ __forceinline__ float2 t_cos_sin(float x) {
#if VKPTC_SINCOS
  if constexpr (kParity) return parity_cos_sin(x);
#else
  if constexpr (kParity) return make_float2(parity_cos(x), parity_sin(x));
#endif
  else return make_float2(cosf(x), sinf(x));
}
template <bool kParity>
__device__ __forceinline__ float t_pow(float x, float y) {
  if constexpr (kParity) return parity_pow(x, y);
  else return powf(x, y);
}

// ------------------------------------------------------------------ RNG
// splitmix64 and the keyed stream of the reference's Rng
// (src/pathtracer/ScalarCpuPathTracer.cpp:36-41, 383-393).
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ULL;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}
__host__ __device__ __forceinline__ uint64_t stream_key(uint64_t seed, uint64_t frame, uint64_t sample,
                                                        uint64_t path_id, uint64_t dim, uint64_t depth,
                                                        uint64_t pixel) {
  const uint64_t m = mix64(seed ^ mix64(frame) ^ mix64(sample) ^ mix64(path_id) ^ mix64(dim) ^ mix64(depth));
  return mix64(m + mix64(pixel));
}
__host__ __device__ __forceinline__ float next01(uint64_t& s) {
  s = mix64(s);
  return static_cast<float>(static_cast<uint32_t>((s >> 8) & 0x00ffffffu)) * (1.0f / 16777215.0f);
}

// --------------------------------------------------------------- records
// Material word map (16 floats) and light word map (16 floats); see vkptc.h.
struct MaterialRec {
  V3 albedo, emissive;
  float roughness, metallic, ior, transmission, clearcoat, sheen, alpha;
  uint32_t model, effect;
};
__device__ __forceinline__ MaterialRec load_material(const float* m) {
  MaterialRec r;
  r.albedo = ld3(m);
  r.emissive = ld3(m + 3);
  r.roughness = m[6];
  r.model = static_cast<uint32_t>(m[7] + 0.5f);
  r.metallic = m[8];
  r.ior = m[9];
  r.transmission = m[10];
  r.clearcoat = m[11];
  r.sheen = m[12];
  r.alpha = m[14];
  r.effect = static_cast<uint32_t>(m[15] + 0.5f) & 1023u;
  return r;
}

// Device view of one loaded scene (passed by value or read from a table).
struct DevScene {
  const float4* nodes;        // wide nodes, 8 float4 each
  const float4* tris;         // triangle records, 3 float4 each, leaf order
  const float4* shade;        // per primitive: normal xyz, material index bits
  const float4* tie;          // per binary node: lo3+parent, hi3+depth
  const float* materials;     // 16 floats each
  const float* lights;        // 16 floats each
  uint32_t material_count;
  uint32_t light_count;
  uint32_t prim_count;
  uint32_t has_transmissive;
  uint32_t has_effects;       // some material has a procedural effect (1..19)
  V3 env;
  const float4* env_map;      // equirectangular texels (rgb, w unused), or null
  uint32_t env_w, env_h;
  V3 env_scale;
  V3 cam_pos, cam_fwd, cam_right, cam_up;
  float tan_half_fov;
  float aperture, focus;
  // Lens shape, prepared on the host by the reference's own float expressions:
  // iris_on (3..64 blades, roundness below 0.999), the blade sector 2*pi/blades,
  // cos(sector/2), the rotation in radians, roundness and 1 - roundness, and
  // the anamorphic squeeze (non-finite: 1; else at least 0.01).
  uint32_t iris_on;
  float iris_sector, iris_cos_half, iris_rot, iris_round, iris_one_minus_round;
  float squeeze;
  uint32_t stack_required;
  uint32_t reference_tree;   // 1: the traversal tree is the reference's own tree
  uint32_t watertight;       // 1: triangle records hold vertices, tested watertight
  const float4* sdf;         // SDF primitive records (sdf.cuh), tested after the triangles
  uint32_t sdf_count;
};

// Render-wide integrator settings.
struct DevSettings {
  uint32_t width, height, max_depth;
  uint32_t enable_nee, enable_mis;
  uint32_t rr_start;
  float rr_min, rr_max;
  uint64_t seed;
  float firefly_clamp;
  uint32_t frame;
};

// Warp-aggregated append: one atomic per warp for all active lanes that want
// a slot; returns this lane's slot (or unspecified when !want).
__device__ __forceinline__ uint32_t warp_append(uint32_t* counter, bool want) {
  const unsigned active = __activemask();
  const unsigned mask = __ballot_sync(active, want);
  if (mask == 0u) return 0u;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(mask) - 1;
  uint32_t base = 0u;
  if (lane == leader) base = atomicAdd(counter, static_cast<uint32_t>(__popc(mask)));
  base = __shfl_sync(active, base, leader);
  return base + static_cast<uint32_t>(__popc(mask & ((1u << lane) - 1u)));
}

// Warp-reduced counter add: one 64-bit atomic per warp.
__device__ __forceinline__ void warp_count(unsigned long long* counter, uint32_t v) {
  const unsigned active = __activemask();
  const unsigned s = __reduce_add_sync(active, v);
  if ((threadIdx.x & 31) == (__ffs(active) - 1) && s != 0u) atomicAdd(counter, static_cast<unsigned long long>(s));
}

}  // namespace vkptc
