// traverse.cuh -- wide-BVH closest-hit and any-hit traversal for sm_100a.
//
// Semantics are those of the reference accelerator
// (src/pathtracer/CpuBvhAccelerator.cpp:113-154, 360-477) and its leaf test
// (src/cpu/BvhTriangleIntersector.cpp:25-74):
//  * Moller-Trumbore with |det| < 1e-4 rejected, no backface culling, a hit
//    accepted when 1e-4 < t < best; evaluated in the reference's exact
//    operation order without fused multiply-adds, so t is bit-identical.
//  * Box test: slab from t = 1e-4, an axis with |d| <= 1e-4 is "parallel" and
//    only checks that the origin lies inside the slab.  The node test here
//    uses a fused lo*inv - o*inv form for speed; every triangle box is padded
//    by 1e-4, which keeps a box that holds a valid hit inside the interval by
//    far more than the rounding difference, so the set of reachable hits, and
//    the parallel-axis culling, are the reference's.
//  * Exact distance ties: the reference keeps the first triangle it visits
//    (strict t < best), i.e. the earlier lane of one leaf, or for two leaves
//    the one under the nearer child of their lowest common binary ancestor
//    (left first when the entry distances are equal), since it traverses the
//    binary tree depth first, near child first.  tie_candidate_wins()
//    evaluates exactly that order from the binary tree kept beside the wide one.
// Nodes are 128-byte lines of which the traversal loads the bounds (three
// 256-bit loads) and the child refs (one 128-bit load; an unused slot's ref is
// kEmptyChild); triangles are three 128-bit loads.  The stack holds (child ref, entry distance) pairs in
// shared memory, interleaved per thread, and is sized on the host from the
// BVH's exact worst case so it cannot overflow.
#pragma once

#include "bvh_layout.h"
#include "common.cuh"

namespace vkptc {

#define kInf __int_as_float(0x7f800000)

// 1: the persistent traversal steps one node or one triangle at a time
// (lane_step_tri); 0: one node or one whole leaf (lane_step).
#ifndef VKPTC_TRI_STEP
#define VKPTC_TRI_STEP 1
#endif
#if VKPTC_TRI_STEP
#define VKPTC_LANE_STEP lane_step_tri<kAny, kStats, kWt>
#else
#define VKPTC_LANE_STEP lane_step<kAny, kStats, kWt>
#endif

struct RayPrep {
  float ox, oy, oz, dx, dy, dz;
  float ix, iy, iz;      // 1/d (0 on axes the node test treats with the inside rule)
  float nix, niy, niz;   // -o/d (for the fused node test)
  uint32_t par;          // bit k: |d_k| <= 1e-4, the reference's "parallel" axis
  uint32_t node_par;     // axes the node test handles with the origin-inside-slab rule
  uint32_t leaf_par;     // axes whose reference rule is applied at the leaf (reference leaf box)
};

// reference_tree: the traversal tree is the reference's own tree, so the
// reference's parallel-axis rule is applied exactly in every node test (it is
// monotone under box inclusion).  Otherwise nodes are tested geometrically
// (an exactly-zero component uses the inside rule, which is then exact) and
// the rule is applied where it decides the result: a hit on a triangle counts
// only if the origin lies inside its REFERENCE leaf's slab on those axes.
// watertight: no such rule anywhere.  The rule treats an axis with |d| <= 1e-4
// as parallel although the ray drifts up to 1e-4 t along it, more than the
// boxes' 1e-4 padding, so it can cull a box the ray enters; the watertight mode
// tests every box geometrically (only |d| < 1e-20 uses the inside rule).
__device__ __forceinline__ RayPrep prep_ray(V3 o, V3 d, bool reference_tree = true, bool watertight = false) {
  RayPrep r;
  r.ox = o.x; r.oy = o.y; r.oz = o.z;
  r.dx = d.x; r.dy = d.y; r.dz = d.z;
  r.par = (fabsf(d.x) <= kEps ? 1u : 0u) | (fabsf(d.y) <= kEps ? 2u : 0u) | (fabsf(d.z) <= kEps ? 4u : 0u);
  if (watertight) {
    r.par = (fabsf(d.x) < 1e-20f ? 1u : 0u) | (fabsf(d.y) < 1e-20f ? 2u : 0u) | (fabsf(d.z) < 1e-20f ? 4u : 0u);
    r.node_par = r.par;
    r.leaf_par = 0u;
  } else if (reference_tree) {
    r.node_par = r.par;
    r.leaf_par = 0u;
  } else {
    r.node_par = (fabsf(d.x) < 1e-20f ? 1u : 0u) | (fabsf(d.y) < 1e-20f ? 2u : 0u) | (fabsf(d.z) < 1e-20f ? 4u : 0u);
    r.leaf_par = r.par;
  }
  r.ix = (r.node_par & 1u) ? 0.0f : __fdiv_rn(1.0f, d.x);
  r.iy = (r.node_par & 2u) ? 0.0f : __fdiv_rn(1.0f, d.y);
  r.iz = (r.node_par & 4u) ? 0.0f : __fdiv_rn(1.0f, d.z);
  r.nix = -(o.x * r.ix);
  r.niy = -(o.y * r.iy);
  r.niz = -(o.z * r.iz);
  return r;
}

// The reference's parallel-axis rule for a hit in reference leaf `leaf`.
__device__ __forceinline__ bool leaf_rule_ok(const float4* tie, uint32_t leaf, const RayPrep& r) {
  if (r.leaf_par == 0u) return true;
  const float4 a = __ldg(tie + 2 * leaf);
  const float4 b = __ldg(tie + 2 * leaf + 1);
  if ((r.leaf_par & 1u) && (r.ox < a.x || r.ox > b.x)) return false;
  if ((r.leaf_par & 2u) && (r.oy < a.y || r.oy > b.y)) return false;
  if ((r.leaf_par & 4u) && (r.oz < a.z || r.oz > b.z)) return false;
  return true;
}

// The reference's slab test verbatim (no fusion); returns the entry distance.
__device__ __forceinline__ bool ref_slab(const float lo[3], const float hi[3], const RayPrep& r, float tmax_in,
                                         float& tnear) {
  const float o[3] = {r.ox, r.oy, r.oz};
  const float iv[3] = {r.ix, r.iy, r.iz};
  float t_min = kEps, t_max = tmax_in;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (r.par & (1u << a)) {
      if (o[a] < lo[a] || o[a] > hi[a]) return false;
      continue;
    }
    float t0 = __fmul_rn(__fsub_rn(lo[a], o[a]), iv[a]);
    float t1 = __fmul_rn(__fsub_rn(hi[a], o[a]), iv[a]);
    if (t0 > t1) {
      const float tmp = t0;
      t0 = t1;
      t1 = tmp;
    }
    t_min = smax(t_min, t0);
    t_max = smin(t_max, t1);
    if (t_min > t_max) return false;
  }
  tnear = t_min;
  return t_max > kEps;
}

// The six bound words of a wide node.  With VKPTC_NODE_LD256 (the default)
// three 256-bit read-only loads (ld.global.nc.v8, sm_100) instead of six
// 128-bit ones; node records are 128-byte lines of allocations whose base the
// host checks for 32-byte alignment.
#ifndef VKPTC_NODE_LD256
#define VKPTC_NODE_LD256 1
#endif
__device__ __forceinline__ void ldg256(const float4* p, float4& a, float4& b) {
  asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
      : "l"(p));
}
__device__ __forceinline__ void load_node_bounds(const float4* np, float4& lx, float4& hx, float4& ly, float4& hy,
                                                 float4& lz, float4& hz) {
#if VKPTC_NODE_LD256
  ldg256(np, lx, hx);
  ldg256(np + 2, ly, hy);
  ldg256(np + 4, lz, hz);
#else
  lx = __ldg(np + 0);
  hx = __ldg(np + 1);
  ly = __ldg(np + 2);
  hy = __ldg(np + 3);
  lz = __ldg(np + 4);
  hz = __ldg(np + 5);
#endif
}

// Fused node test of one child slot; exact parallel-axis rule.
__device__ __forceinline__ bool node_slab(float lx, float hx, float ly, float hy, float lz, float hz,
                                          const RayPrep& r, float tmax_in, float& tnear) {
  float ax0 = __fmaf_rn(lx, r.ix, r.nix), ax1 = __fmaf_rn(hx, r.ix, r.nix);
  float ay0 = __fmaf_rn(ly, r.iy, r.niy), ay1 = __fmaf_rn(hy, r.iy, r.niy);
  float az0 = __fmaf_rn(lz, r.iz, r.niz), az1 = __fmaf_rn(hz, r.iz, r.niz);
  float nx = fminf(ax0, ax1), fx = fmaxf(ax0, ax1);
  float ny = fminf(ay0, ay1), fy = fmaxf(ay0, ay1);
  float nz = fminf(az0, az1), fz = fmaxf(az0, az1);
  if (r.node_par) {
    if (r.node_par & 1u) {
      const bool in = !(r.ox < lx || r.ox > hx);
      nx = in ? -kInf : kInf;
      fx = kInf;
    }
    if (r.node_par & 2u) {
      const bool in = !(r.oy < ly || r.oy > hy);
      ny = in ? -kInf : kInf;
      fy = kInf;
    }
    if (r.node_par & 4u) {
      const bool in = !(r.oz < lz || r.oz > hz);
      nz = in ? -kInf : kInf;
      fz = kInf;
    }
  }
  const float tn = fmaxf(fmaxf(nx, ny), fmaxf(nz, kEps));
  const float tf = fminf(fminf(fx, fy), fminf(fz, tmax_in));
  tnear = tn;
  return tn <= tf && tf > kEps;
}

// Moller-Trumbore in the reference's operation order; returns t or -1.
__device__ __forceinline__ float mt_test(const float4 a, const float4 b, const float4 c, const RayPrep& r) {
  const float v0x = a.x, v0y = a.y, v0z = a.z;
  const float e1x = a.w, e1y = b.x, e1z = b.y;
  const float e2x = b.z, e2y = b.w, e2z = c.x;
  const float hx = __fsub_rn(__fmul_rn(r.dy, e2z), __fmul_rn(r.dz, e2y));
  const float hy = __fsub_rn(__fmul_rn(r.dz, e2x), __fmul_rn(r.dx, e2z));
  const float hz = __fsub_rn(__fmul_rn(r.dx, e2y), __fmul_rn(r.dy, e2x));
  const float det = __fadd_rn(__fadd_rn(__fmul_rn(e1x, hx), __fmul_rn(e1y, hy)), __fmul_rn(e1z, hz));
  if (fabsf(det) < kEps) return -1.0f;
  const float inv = __fdiv_rn(1.0f, det);
  const float sx = __fsub_rn(r.ox, v0x), sy = __fsub_rn(r.oy, v0y), sz = __fsub_rn(r.oz, v0z);
  const float u = __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(sx, hx), __fmul_rn(sy, hy)), __fmul_rn(sz, hz)), inv);
  if (u < 0.0f || u > 1.0f) return -1.0f;
  const float qx = __fsub_rn(__fmul_rn(sy, e1z), __fmul_rn(sz, e1y));
  const float qy = __fsub_rn(__fmul_rn(sz, e1x), __fmul_rn(sx, e1z));
  const float qz = __fsub_rn(__fmul_rn(sx, e1y), __fmul_rn(sy, e1x));
  const float v = __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(r.dx, qx), __fmul_rn(r.dy, qy)), __fmul_rn(r.dz, qz)), inv);
  if (v < 0.0f || __fadd_rn(u, v) > 1.0f) return -1.0f;
  const float t = __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(e2x, qx), __fmul_rn(e2y, qy)), __fmul_rn(e2z, qz)), inv);
  return t;
}

// Per-ray constants of the watertight test (Woop, Benthin and Wald, "Watertight
// Ray/Triangle Intersection", JCGT 2(1), 2013): kz is the axis of the largest
// |d| (the first on ties), kx and ky follow it cyclically and are swapped when
// d[kz] < 0, which keeps the triangles' winding; the shear maps the ray onto
// +z: sx = d[kx]/d[kz], sy = d[ky]/d[kz], sz = 1/d[kz].
struct WtRay {
  int kx, ky, kz;
  float sx, sy, sz;
};

__device__ __forceinline__ float axis_of(float x, float y, float z, int k) { return k == 0 ? x : (k == 1 ? y : z); }

__device__ __forceinline__ WtRay prep_wt(const RayPrep& r) {
  const float ax = fabsf(r.dx), ay = fabsf(r.dy), az = fabsf(r.dz);
  int kz = 0;
  float m = ax;
  if (ay > m) {
    kz = 1;
    m = ay;
  }
  if (az > m) kz = 2;
  int kx = kz == 2 ? 0 : kz + 1;
  int ky = kx == 2 ? 0 : kx + 1;
  const float dz = axis_of(r.dx, r.dy, r.dz, kz);
  if (dz < 0.0f) {
    const int t = kx;
    kx = ky;
    ky = t;
  }
  WtRay w;
  w.kx = kx;
  w.ky = ky;
  w.kz = kz;
  w.sx = __fdiv_rn(axis_of(r.dx, r.dy, r.dz, kx), dz);
  w.sy = __fdiv_rn(axis_of(r.dx, r.dy, r.dz, ky), dz);
  w.sz = __fdiv_rn(1.0f, dz);
  return w;
}

// The watertight test without back-face culling on a record holding the
// vertices (a, b, c) in the slots of (v0, e1, e2).  The three edge functions
// of the sheared 2D triangle are computed from the vertices themselves, so two
// triangles sharing an edge evaluate it identically (up to sign) and no ray
// passes between them; an edge function that rounds to exactly 0 is redone in
// double (the products are exact there).  Returns t = T/det, or -1 on a miss.
__device__ __forceinline__ float wt_test(const float4 p, const float4 q, const float4 s, const RayPrep& r,
                                         const WtRay& w) {
  const float ax = __fsub_rn(p.x, r.ox), ay = __fsub_rn(p.y, r.oy), az = __fsub_rn(p.z, r.oz);
  const float bx = __fsub_rn(p.w, r.ox), by = __fsub_rn(q.x, r.oy), bz = __fsub_rn(q.y, r.oz);
  const float cx = __fsub_rn(q.z, r.ox), cy = __fsub_rn(q.w, r.oy), cz = __fsub_rn(s.x, r.oz);
  const float akz = axis_of(ax, ay, az, w.kz), bkz = axis_of(bx, by, bz, w.kz), ckz = axis_of(cx, cy, cz, w.kz);
  const float Ax = __fsub_rn(axis_of(ax, ay, az, w.kx), __fmul_rn(w.sx, akz));
  const float Ay = __fsub_rn(axis_of(ax, ay, az, w.ky), __fmul_rn(w.sy, akz));
  const float Bx = __fsub_rn(axis_of(bx, by, bz, w.kx), __fmul_rn(w.sx, bkz));
  const float By = __fsub_rn(axis_of(bx, by, bz, w.ky), __fmul_rn(w.sy, bkz));
  const float Cx = __fsub_rn(axis_of(cx, cy, cz, w.kx), __fmul_rn(w.sx, ckz));
  const float Cy = __fsub_rn(axis_of(cx, cy, cz, w.ky), __fmul_rn(w.sy, ckz));
  float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
  float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
  float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
  if (U == 0.0f || V == 0.0f || W == 0.0f) {
    U = __double2float_rn(__dsub_rn(__dmul_rn(Cx, By), __dmul_rn(Cy, Bx)));
    V = __double2float_rn(__dsub_rn(__dmul_rn(Ax, Cy), __dmul_rn(Ay, Cx)));
    W = __double2float_rn(__dsub_rn(__dmul_rn(Bx, Ay), __dmul_rn(By, Ax)));
  }
  if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return -1.0f;
  const float det = __fadd_rn(__fadd_rn(U, V), W);
  if (det == 0.0f) return -1.0f;
  const float Az = __fmul_rn(w.sz, akz), Bz = __fmul_rn(w.sz, bkz), Cz = __fmul_rn(w.sz, ckz);
  const float T = __fadd_rn(__fadd_rn(__fmul_rn(U, Az), __fmul_rn(V, Bz)), __fmul_rn(W, Cz));
  return __fdiv_rn(T, det);
}

// The configured triangle test: the reference's Moller-Trumbore, or watertight.
template <bool kWt>
__device__ __forceinline__ float tri_test(const float4 a, const float4 b, const float4 c, const RayPrep& r,
                                          const WtRay& w) {
  if constexpr (kWt) return wt_test(a, b, c, r, w);
  else return mt_test(a, b, c, r);
}

__device__ __forceinline__ void tie_box(const float4* tie, int32_t id, float lo[3], float hi[3]) {
  const float4 a = __ldg(tie + 2 * id);
  const float4 b = __ldg(tie + 2 * id + 1);
  lo[0] = a.x; lo[1] = a.y; lo[2] = a.z;
  hi[0] = b.x; hi[1] = b.y; hi[2] = b.z;
}
__device__ __forceinline__ int32_t tie_parent(const float4* tie, int32_t id) {
  return __float_as_int(__ldg(tie + 2 * id).w);
}
__device__ __forceinline__ int32_t tie_depth(const float4* tie, int32_t id) {
  return __float_as_int(__ldg(tie + 2 * id + 1).w);
}

// True when the candidate (leaf_b, lane_b) is visited before the incumbent
// (leaf_a, lane_a) by the reference's depth-first near-first traversal.
// Takes the ray by value (origin, reciprocal direction, parallel mask) so the
// caller's ray state can stay in registers across this rarely taken call.
__device__ __forceinline__ bool tie_candidate_wins_v(const float4* tie, float ox, float oy, float oz, float ix, float iy,
                                                  float iz, uint32_t par, uint32_t leaf_a, uint32_t lane_a,
                                                  uint32_t leaf_b, uint32_t lane_b) {
  if (leaf_a == leaf_b) return lane_b < lane_a;
  RayPrep r;
  r.ox = ox; r.oy = oy; r.oz = oz;
  r.ix = ix; r.iy = iy; r.iz = iz;
  r.par = par;
  int32_t a = static_cast<int32_t>(leaf_a), b = static_cast<int32_t>(leaf_b);
  int32_t da = tie_depth(tie, a), db = tie_depth(tie, b);
  while (da > db && a > 0) { a = tie_parent(tie, a); --da; }
  while (db > da && b > 0) { b = tie_parent(tie, b); --db; }
  // Climb together to the children of the lowest common ancestor; the root
  // (id 0, parent -1) ends the walk on malformed input.
  while (a > 0 && b > 0 && tie_parent(tie, a) != tie_parent(tie, b)) {
    a = tie_parent(tie, a);
    b = tie_parent(tie, b);
  }
  if (a <= 0 || b <= 0) return false;
  float lo[3], hi[3];
  float ta = 0.0f, tb = 0.0f;
  tie_box(tie, a, lo, hi);
  ref_slab(lo, hi, r, kInf, ta);
  tie_box(tie, b, lo, hi);
  ref_slab(lo, hi, r, kInf, tb);
  // Sibling ids are allocated (left, right) consecutively: left is the smaller.
  const bool a_left = a < b;
  const float t_left = a_left ? ta : tb, t_right = a_left ? tb : ta;
  const bool left_first = t_left <= t_right;
  const bool a_first = (a_left == left_first);
  return !a_first;
}

__device__ __forceinline__ bool tie_candidate_wins(const float4* tie, const RayPrep& r, uint32_t leaf_a,
                                                   uint32_t lane_a, uint32_t leaf_b, uint32_t lane_b) {
  return tie_candidate_wins_v(tie, r.ox, r.oy, r.oz, r.ix, r.iy, r.iz, r.par, leaf_a, lane_a, leaf_b, lane_b);
}

struct TraceStats {
  uint32_t nodes = 0, leaves = 0, tris = 0, rays = 0;
};

// Shared-memory stack, interleaved so consecutive threads hit distinct banks.
struct SmemStack {
  int2* base;     // entry i of this thread at base[i * stride]
  int stride;
  int cap;
};

__device__ __forceinline__ int32_t leaf_first(int32_t ref) { return static_cast<int32_t>((~ref) >> 3); }
__device__ __forceinline__ int32_t leaf_count(int32_t ref) { return ((~ref) & 7) + 1; }

// Closest hit.  best_t = +inf and prim = kMiss on a miss.  `err` receives 1 on
// a stack overflow (which the host-side sizing rules out).
template <bool kStats, bool kWt = false>
__device__ __forceinline__ void trace_closest(const DevScene& s, const RayPrep& r, SmemStack stk, float& best_t,
                                              uint32_t& best_prim, TraceStats& st, uint32_t& err) {
  WtRay w{};
  if constexpr (kWt) w = prep_wt(r);
  best_t = kInf;
  best_prim = kMiss;
  uint32_t best_leaf = 0u, best_lane = 0u;
  int sp = 0;
  int32_t ref = 0;
  if (s.prim_count == 0u) return;
  while (true) {
    if (ref >= 0) {
      const float4* np = s.nodes + 8 * ref;
      float4 lx, hx, ly, hy, lz, hz;
      load_node_bounds(np, lx, hx, ly, hy, lz, hz);
      const int4 ch = __ldg(reinterpret_cast<const int4*>(np + 6));
      if (kStats) ++st.nodes;
      float t[4];
      int32_t c[4] = {ch.x, ch.y, ch.z, ch.w};
      bool h0 = node_slab(lx.x, hx.x, ly.x, hy.x, lz.x, hz.x, r, best_t, t[0]);
      bool h1 = node_slab(lx.y, hx.y, ly.y, hy.y, lz.y, hz.y, r, best_t, t[1]) && c[1] != kEmptyChild;
      bool h2 = node_slab(lx.z, hx.z, ly.z, hy.z, lz.z, hz.z, r, best_t, t[2]) && c[2] != kEmptyChild;
      bool h3 = node_slab(lx.w, hx.w, ly.w, hy.w, lz.w, hz.w, r, best_t, t[3]) && c[3] != kEmptyChild;
      t[0] = h0 ? t[0] : kInf;
      t[1] = h1 ? t[1] : kInf;
      t[2] = h2 ? t[2] : kInf;
      t[3] = h3 ? t[3] : kInf;
      const int hits = int(h0) + int(h1) + int(h2) + int(h3);
      // Sort (t, c) ascending with a 5-comparator network; misses sink (t = inf).
#define VKPTC_CSWAP(i, j)                         \
  if (t[j] < t[i]) {                              \
    const float tt = t[i]; t[i] = t[j]; t[j] = tt; \
    const int32_t cc = c[i]; c[i] = c[j]; c[j] = cc; \
  }
      VKPTC_CSWAP(0, 1) VKPTC_CSWAP(2, 3) VKPTC_CSWAP(0, 2) VKPTC_CSWAP(1, 3) VKPTC_CSWAP(1, 2)
#undef VKPTC_CSWAP
      if (hits > 0) {
        // Push the farther hits, farthest first, continue with the nearest.
#pragma unroll
        for (int k = 3; k >= 1; --k) {
          if (k < hits) {
            if (sp < stk.cap) {
              stk.base[sp * stk.stride] = make_int2(c[k], __float_as_int(t[k]));
              ++sp;
            } else {
              err = 1u;
            }
          }
        }
        ref = c[0];
        continue;
      }
    } else {
      const int32_t first = leaf_first(ref);
      const int32_t count = leaf_count(ref);
      if (kStats) {
        ++st.leaves;
        st.tris += static_cast<uint32_t>(count);
      }
      for (int32_t i = 0; i < count; ++i) {
        const float4* tp = s.tris + 3 * (first + i);
        const float4 a = __ldg(tp), b = __ldg(tp + 1), cc = __ldg(tp + 2);
        const float th = tri_test<kWt>(a, b, cc, r, w);
        if (th <= kEps) continue;   // also rejects the -1 miss code
        if (r.leaf_par != 0u && !leaf_rule_ok(s.tie, __float_as_uint(cc.z), r)) continue;
        if (th < best_t) {
          best_t = th;
          best_prim = __float_as_uint(cc.y);
          best_leaf = __float_as_uint(cc.z);
          best_lane = __float_as_uint(cc.w);
        } else if (th == best_t &&
                   tie_candidate_wins(s.tie, r, best_leaf, best_lane, __float_as_uint(cc.z), __float_as_uint(cc.w))) {
          best_prim = __float_as_uint(cc.y);
          best_leaf = __float_as_uint(cc.z);
          best_lane = __float_as_uint(cc.w);
        }
      }
    }
    // Pop the next entry that can still hold a hit no farther than best_t.
    bool found = false;
    while (sp > 0) {
      --sp;
      const int2 e = stk.base[sp * stk.stride];
      if (__int_as_float(e.y) <= best_t) {
        ref = e.x;
        found = true;
        break;
      }
    }
    if (!found) break;
  }
}

// Any hit with 1e-4 < t < tmax.  Returns true when occluded.
template <bool kStats, bool kWt = false>
__device__ __forceinline__ bool trace_any(const DevScene& s, const RayPrep& r, float tmax, SmemStack stk,
                                          TraceStats& st, uint32_t& err) {
  if (s.prim_count == 0u || !(tmax > kEps)) return false;
  WtRay w{};
  if constexpr (kWt) w = prep_wt(r);
  int sp = 0;
  int32_t ref = 0;
  while (true) {
    if (ref >= 0) {
      const float4* np = s.nodes + 8 * ref;
      float4 lx, hx, ly, hy, lz, hz;
      load_node_bounds(np, lx, hx, ly, hy, lz, hz);
      const int4 ch = __ldg(reinterpret_cast<const int4*>(np + 6));
      if (kStats) ++st.nodes;
      float t0, t1, t2, t3;
      const bool h0 = node_slab(lx.x, hx.x, ly.x, hy.x, lz.x, hz.x, r, tmax, t0);
      const bool h1 = node_slab(lx.y, hx.y, ly.y, hy.y, lz.y, hz.y, r, tmax, t1) && ch.y != kEmptyChild;
      const bool h2 = node_slab(lx.z, hx.z, ly.z, hy.z, lz.z, hz.z, r, tmax, t2) && ch.z != kEmptyChild;
      const bool h3 = node_slab(lx.w, hx.w, ly.w, hy.w, lz.w, hz.w, r, tmax, t3) && ch.w != kEmptyChild;
      int32_t next = 0;
      bool have = false;
      const int32_t cs[4] = {ch.x, ch.y, ch.z, ch.w};
      const bool hs[4] = {h0, h1, h2, h3};
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (!hs[k]) continue;
        if (!have) {
          next = cs[k];
          have = true;
        } else if (sp < stk.cap) {
          stk.base[sp * stk.stride] = make_int2(cs[k], 0);
          ++sp;
        } else {
          err = 1u;
        }
      }
      if (have) {
        ref = next;
        continue;
      }
    } else {
      const int32_t first = leaf_first(ref);
      const int32_t count = leaf_count(ref);
      if (kStats) {
        ++st.leaves;
        st.tris += static_cast<uint32_t>(count);
      }
      for (int32_t i = 0; i < count; ++i) {
        const float4* tp = s.tris + 3 * (first + i);
        const float4 tc = __ldg(tp + 2);
        const float th = tri_test<kWt>(__ldg(tp), __ldg(tp + 1), tc, r, w);
        if (th > kEps && th < tmax && (r.leaf_par == 0u || leaf_rule_ok(s.tie, __float_as_uint(tc.z), r))) return true;
      }
    }
    if (sp == 0) break;
    --sp;
    ref = stk.base[sp * stk.stride].x;
  }
  return false;
}


// ================================================================ persistent
// Lane-level traversal state machine for the persistent kernels: one call of
// lane_step() processes one wide node or one leaf, so a warp can re-converge
// every few steps and hand finished lanes new rays (dynamic ray fetch).

// Stack of (ref, entry distance): the first `scap` entries in shared memory
// (interleaved per thread), the rest in a per-thread slab in global memory.
struct TwoLevelStack {
  int2* smem;     // this thread's entry 0; entry i at smem[i * sstride]
  int sstride;
  int scap;
  int2* spill;    // this thread's spill entry 0; entry i at spill[i * gstride]
  int gstride;
  int total;      // scap + spill entries
  __device__ __forceinline__ void put(int i, int2 e) const {
    if (i < scap) smem[i * sstride] = e;
    else spill[(i - scap) * gstride] = e;
  }
  __device__ __forceinline__ int2 get(int i) const {
    return i < scap ? smem[i * sstride] : spill[(i - scap) * gstride];
  }
};

// Geometry a lane traverses (one launch may serve several scenes).
struct GeoView {
  const float4* nodes;
  const float4* tris;
  const float4* tie;
  uint32_t prim_count;
  uint32_t reference_tree;   // 1: traversal tree is the reference tree
};

__host__ __device__ __forceinline__ GeoView geo_of(const DevScene& s) {
  return GeoView{s.nodes, s.tris, s.tie, s.prim_count, s.reference_tree};
}

struct LaneState {
  GeoView g;
  RayPrep r;
  WtRay w;          // watertight test constants (unused by the Moller-Trumbore kernels)
  float t;          // closest: best distance so far; any: the query's upper bound
  uint32_t prim;    // closest: primitive; any: 1 when occluded
  uint32_t leaf, lane;
  int32_t ref;
  int sp;
  int32_t tri, tri_end;   // lane_step_tri: triangle records of the leaf being tested, [tri, tri_end)
};

template <bool kWt = false>
__device__ __forceinline__ void lane_begin(LaneState& L, V3 o, V3 d, float tmax, bool any) {
  L.r = prep_ray(o, d, L.g.reference_tree != 0u, kWt);
  if constexpr (kWt) L.w = prep_wt(L.r);
  L.t = any ? tmax : kInf;
  L.prim = any ? 0u : kMiss;
  L.leaf = L.lane = 0u;
  L.ref = 0;
  L.sp = 0;
  L.tri = L.tri_end = 0;
}

// Returns true when the query has finished.
template <bool kAny, bool kStats, bool kWt = false>
__device__ __forceinline__ bool lane_step(LaneState& L, const TwoLevelStack& stk, TraceStats& st, uint32_t& err) {
  if (L.ref >= 0) {
    const float4* np = L.g.nodes + 8 * L.ref;
    float4 lx, hx, ly, hy, lz, hz;
    load_node_bounds(np, lx, hx, ly, hy, lz, hz);
    const int4 ch = __ldg(reinterpret_cast<const int4*>(np + 6));
    if (kStats) ++st.nodes;
    float t[4];
    int32_t c[4] = {ch.x, ch.y, ch.z, ch.w};
    const bool h0 = node_slab(lx.x, hx.x, ly.x, hy.x, lz.x, hz.x, L.r, L.t, t[0]);
    const bool h1 = node_slab(lx.y, hx.y, ly.y, hy.y, lz.y, hz.y, L.r, L.t, t[1]) && c[1] != kEmptyChild;
    const bool h2 = node_slab(lx.z, hx.z, ly.z, hy.z, lz.z, hz.z, L.r, L.t, t[2]) && c[2] != kEmptyChild;
    const bool h3 = node_slab(lx.w, hx.w, ly.w, hy.w, lz.w, hz.w, L.r, L.t, t[3]) && c[3] != kEmptyChild;
    t[0] = h0 ? t[0] : kInf;
    t[1] = h1 ? t[1] : kInf;
    t[2] = h2 ? t[2] : kInf;
    t[3] = h3 ? t[3] : kInf;
    const int hits = int(h0) + int(h1) + int(h2) + int(h3);
#define VKPTC_CSWAP(i, j)                            \
  if (t[j] < t[i]) {                                 \
    const float tt = t[i]; t[i] = t[j]; t[j] = tt;   \
    const int32_t cc = c[i]; c[i] = c[j]; c[j] = cc; \
  }
    VKPTC_CSWAP(0, 1) VKPTC_CSWAP(2, 3) VKPTC_CSWAP(0, 2) VKPTC_CSWAP(1, 3) VKPTC_CSWAP(1, 2)
#undef VKPTC_CSWAP
    if (hits > 0) {
#pragma unroll
      for (int k = 3; k >= 1; --k) {
        if (k < hits) {
          if (L.sp < stk.total) {
            stk.put(L.sp, make_int2(c[k], __float_as_int(t[k])));
            ++L.sp;
          } else {
            err = 1u;
          }
        }
      }
      L.ref = c[0];
      return false;
    }
  } else {
    const int32_t first = leaf_first(L.ref);
    const int32_t count = leaf_count(L.ref);
    if (kStats) {
      ++st.leaves;
      st.tris += static_cast<uint32_t>(count);
    }
    for (int32_t i = 0; i < count; ++i) {
      const float4* tp = L.g.tris + 3 * (first + i);
      const float4 a = __ldg(tp), b = __ldg(tp + 1), cc = __ldg(tp + 2);
      const float th = tri_test<kWt>(a, b, cc, L.r, L.w);
      if (th <= kEps) continue;
      if (L.r.leaf_par != 0u && !leaf_rule_ok(L.g.tie, __float_as_uint(cc.z), L.r)) continue;
      if (kAny) {
        if (th < L.t) {
          L.prim = 1u;
          return true;
        }
      } else if (th < L.t) {
        L.t = th;
        L.prim = __float_as_uint(cc.y);
        L.leaf = __float_as_uint(cc.z);
        L.lane = __float_as_uint(cc.w);
      } else if (th == L.t &&
                 tie_candidate_wins(L.g.tie, L.r, L.leaf, L.lane, __float_as_uint(cc.z), __float_as_uint(cc.w))) {
        L.prim = __float_as_uint(cc.y);
        L.leaf = __float_as_uint(cc.z);
        L.lane = __float_as_uint(cc.w);
      }
    }
  }
  while (L.sp > 0) {
    --L.sp;
    const int2 e = stk.get(L.sp);
    if (kAny || __int_as_float(e.y) <= L.t) {
      L.ref = e.x;
      return false;
    }
  }
  return true;
}

// The same traversal with a step of one wide node OR one triangle: a leaf
// reached by a step is tested one triangle per later step.  A warp's lanes
// diverge between node and leaf work at every step; with whole leaves per
// step a lane in a leaf holds the warp for up to eight triangle tests while
// its neighbours wait, with single triangles the two branches cost about the
// same.  Triangles are tested in the same order with the same rules, so hits
// (and ties) are identical to lane_step's.  Returns true when the query has
// finished.
template <bool kAny, bool kStats, bool kWt = false>
__device__ __forceinline__ void lane_enter(LaneState& L, int32_t ref, TraceStats& st) {
  L.ref = ref;
  if (ref < 0) {
    L.tri = leaf_first(ref);
    L.tri_end = L.tri + leaf_count(ref);
    if (kStats) {
      ++st.leaves;
      st.tris += static_cast<uint32_t>(L.tri_end - L.tri);
    }
  }
}

template <bool kAny, bool kStats, bool kWt = false>
__device__ __forceinline__ bool lane_step_tri(LaneState& L, const TwoLevelStack& stk, TraceStats& st,
                                              uint32_t& err) {
  if (L.tri < L.tri_end) {
    const float4* tp = L.g.tris + 3 * L.tri;
    ++L.tri;
    const float4 a = __ldg(tp), b = __ldg(tp + 1), cc = __ldg(tp + 2);
    const float th = tri_test<kWt>(a, b, cc, L.r, L.w);
    if (th > kEps && (L.r.leaf_par == 0u || leaf_rule_ok(L.g.tie, __float_as_uint(cc.z), L.r))) {
      if (kAny) {
        if (th < L.t) {
          L.prim = 1u;
          return true;
        }
      } else if (th < L.t) {
        L.t = th;
        L.prim = __float_as_uint(cc.y);
        L.leaf = __float_as_uint(cc.z);
        L.lane = __float_as_uint(cc.w);
      } else if (th == L.t &&
                 tie_candidate_wins(L.g.tie, L.r, L.leaf, L.lane, __float_as_uint(cc.z), __float_as_uint(cc.w))) {
        L.prim = __float_as_uint(cc.y);
        L.leaf = __float_as_uint(cc.z);
        L.lane = __float_as_uint(cc.w);
      }
    }
    if (L.tri < L.tri_end) return false;
  } else {
    const float4* np = L.g.nodes + 8 * L.ref;
    float4 lx, hx, ly, hy, lz, hz;
    load_node_bounds(np, lx, hx, ly, hy, lz, hz);
    const int4 ch = __ldg(reinterpret_cast<const int4*>(np + 6));
    if (kStats) ++st.nodes;
    float t[4];
    int32_t c[4] = {ch.x, ch.y, ch.z, ch.w};
    const bool h0 = node_slab(lx.x, hx.x, ly.x, hy.x, lz.x, hz.x, L.r, L.t, t[0]);
    const bool h1 = node_slab(lx.y, hx.y, ly.y, hy.y, lz.y, hz.y, L.r, L.t, t[1]) && c[1] != kEmptyChild;
    const bool h2 = node_slab(lx.z, hx.z, ly.z, hy.z, lz.z, hz.z, L.r, L.t, t[2]) && c[2] != kEmptyChild;
    const bool h3 = node_slab(lx.w, hx.w, ly.w, hy.w, lz.w, hz.w, L.r, L.t, t[3]) && c[3] != kEmptyChild;
    t[0] = h0 ? t[0] : kInf;
    t[1] = h1 ? t[1] : kInf;
    t[2] = h2 ? t[2] : kInf;
    t[3] = h3 ? t[3] : kInf;
    const int hits = int(h0) + int(h1) + int(h2) + int(h3);
#define VKPTC_CSWAP(i, j)                            \
  if (t[j] < t[i]) {                                 \
    const float tt = t[i]; t[i] = t[j]; t[j] = tt;   \
    const int32_t cc = c[i]; c[i] = c[j]; c[j] = cc; \
  }
    VKPTC_CSWAP(0, 1) VKPTC_CSWAP(2, 3) VKPTC_CSWAP(0, 2) VKPTC_CSWAP(1, 3) VKPTC_CSWAP(1, 2)
#undef VKPTC_CSWAP
    if (hits > 0) {
#pragma unroll
      for (int k = 3; k >= 1; --k) {
        if (k < hits) {
          if (L.sp < stk.total) {
            stk.put(L.sp, make_int2(c[k], __float_as_int(t[k])));
            ++L.sp;
          } else {
            err = 1u;
          }
        }
      }
      lane_enter<kAny, kStats, kWt>(L, c[0], st);
      return false;
    }
  }
  while (L.sp > 0) {
    --L.sp;
    const int2 e = stk.get(L.sp);
    if (kAny || __int_as_float(e.y) <= L.t) {
      lane_enter<kAny, kStats, kWt>(L, e.x, st);
      return false;
    }
  }
  return true;
}

// Persistent traversal over `n` queries supplied by Src:
//   Src::load(j, o, d, tmax) and Src::finish(j, t, prim) (any-hit: prim = occluded).
// Each warp keeps its lanes busy: whenever lanes are idle it claims that many
// query ids with one atomic (warp-aggregated) and refills them.  `steps`
// packs two limits: the low 16 bits are the most traversal steps between
// refills; the high bits, when non-zero, a refill threshold -- the warp
// leaves the step loop for a refill as soon as that many lanes are idle
// (checked after every step).  Without a threshold the lanes run the full
// number of steps between refills.
template <class Src, bool kAny, bool kStats, bool kWt = false>
__device__ __forceinline__ void persistent_traverse(const Src& src, uint32_t n, uint32_t* fetch,
                                                    TwoLevelStack stk, int steps, TraceStats& st, uint32_t& err) {
  const unsigned lane_id = threadIdx.x & 31u;
  const int max_steps = steps & 0xFFFF;
  const int refill_min = steps >> 16;
  LaneState L;
  bool active = false;
  bool exhausted = false;
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
          V3 o, d;
          float tmax;
          src.load(j, o, d, tmax, L.g);
          lane_begin<kWt>(L, o, d, tmax, kAny);
          if (L.g.prim_count == 0u || (kAny && !(tmax > kEps))) {
            src.finish(j, L.t, L.prim);
            if (kStats) ++st.rays;
          } else {
            tag = j;
            active = true;
          }
        }
      }
    }
    if (!__any_sync(0xffffffffu, active)) break;
    if (refill_min == 0) {
      if (active) {
        for (int k = 0; k < max_steps; ++k) {
          if (VKPTC_LANE_STEP(L, stk, st, err)) {
            src.finish(tag, L.t, L.prim);
            if (kStats) ++st.rays;
            active = false;
            break;
          }
        }
      }
    } else {
      for (int k = 0; k < max_steps; ++k) {
        if (active && VKPTC_LANE_STEP(L, stk, st, err)) {
          src.finish(tag, L.t, L.prim);
          if (kStats) ++st.rays;
          active = false;
        }
        const unsigned idle_now = __ballot_sync(0xffffffffu, !active);
        if (idle_now == 0xffffffffu || (!exhausted && __popc(idle_now) >= refill_min)) break;
      }
    }
  }
}

}  // namespace vkptc
