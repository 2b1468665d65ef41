// adjoint.cu -- forward / loss / backward kernels of differentiable rendering.
//
// Forward: one thread per (sample, pixel) path, inline closest-hit and
// any-hit traversal, the float instantiation of the vertex math (adjoint.cuh)
// in the reference's operation order, so each sample's radiance equals the
// renderer's (the film test pins this bit-for-bit).
//
// Backward ("re-trace from the seed"): the same path is replayed from its RNG
// key, recording per vertex the ray, hit, throughput, roulette divisor, RNG
// state and decision flags (64 bytes, at most 8 vertices), then swept in
// reverse.  Each vertex's local Jacobian with respect to (ray origin, ray
// direction, roughness) comes from the dual-number instantiation of the same
// vertex math; albedo and emission enter affinely and are handled in closed
// form.  Per-vertex parameter gradients are combined across the warp (lanes
// grouped by material, butterfly sums) into per-warp shared-memory slots,
// then per-block partials, then a fixed-order FP64 reduction: the gradient is
// deterministic for a given launch shape.
#include "adjoint.cuh"
#include <algorithm>

#include "adjoint_launch.h"
#include "traverse.cuh"

namespace vkptc {

namespace {

struct AdjRec {
  float4 a;   // origin xyz, hit distance
  float4 b;   // direction xyz, primitive bits (kMiss on a miss)
  float4 c;   // throughput at the vertex xyz, roulette divisor applied after it
  uint4 e;    // RNG state lo, hi at the vertex, flags, material index
};
static_assert(sizeof(AdjRec) == kAdjRecordFloat4s * sizeof(float4), "record layout of the backward buffers");
static_assert(kAdjVertexSlots == kAdjMaxDepth, "record slots per path");

__device__ __forceinline__ uint32_t mat_slot(const DevScene& s, uint32_t mat_index) {
  return mat_index < s.material_count - 1u ? mat_index : s.material_count - 1u;
}

// The primal path of pixel (x, y), sample `sample`.  kRecord keeps the
// vertex records for the reverse sweep: vertex k at rec[k * rec_stride].  Returns radiance xyz and, in w, the
// bits of a 32-bit hash of the path's discrete decisions (hit primitives and
// vertex flags): two evaluations with equal hashes took the same branches.
template <bool kParity, bool kRecord>
__device__ __forceinline__ float4 adj_primal(const DevScene& s, const DevSettings& st, const float* mat0,
                                             uint32_t x, uint32_t y, uint32_t sample, SmemStack stk,
                                             uint32_t& err, AdjRec* rec, uint32_t& nrec, uint32_t rec_stride = 1u) {
  V3 o, d;
  uint64_t rng;
  camera_path<kParity>(s, st, x, y, sample, o, d, rng);
  V3 thr = mk(1.0f, 1.0f, 1.0f), thr0 = thr, rad = mk(0.0f, 0.0f, 0.0f);
  uint64_t sig = 0u;
  nrec = 0u;
  const float* lights = s.lights;
  TraceStats ts;
  for (uint32_t depth = 0; depth < st.max_depth; ++depth) {
    float t;
    uint32_t prim;
    trace_closest<false>(s, prep_ray(o, d, s.reference_tree != 0u), stk, t, prim, ts, err);
    if (prim == kMiss) {
      rad = add(rad, mulv(thr, s.env));
      sig = mix64(sig ^ 0xFFFFFFFFull);
      if (kRecord) {
        AdjRec& r = rec[static_cast<size_t>(nrec++) * rec_stride];
        r.a = make_float4(o.x, o.y, o.z, 0.0f);
        r.b = make_float4(d.x, d.y, d.z, __uint_as_float(kMiss));
        r.c = make_float4(thr.x, thr.y, thr.z, 1.0f);
        r.e = make_uint4(0u, 0u, kVfMiss, 0u);
      }
      break;
    }
    const uint64_t rng_at = rng;
    const V3 o_at = o, d_at = d;
    const float4 sh = __ldg(s.shade + prim);
    const V3 gn = mk(sh.x, sh.y, sh.z);
    const uint32_t mi = mat_slot(s, __float_as_uint(sh.w));
    const MaterialRec m = load_material(s.materials + 16u * mi);
    uint32_t flags = 0u;
    AdjVertex<float, V3> R;
    adj_vertex<float, V3, kParity, false>(s, st, lights, depth, o, d, t, gn, m, clamp01(m.roughness), rng, flags, R);
    // emission, then the next-event term, in the renderer's order
    const bool emissive_model = m.model == 1u || m.emissive.x > 0.0f || m.emissive.y > 0.0f || m.emissive.z > 0.0f;
    if (!st.enable_nee || depth == 0u) rad = add(rad, mulv(thr, m.emissive));
    else if (st.enable_mis && emissive_model) rad = add(rad, mul(mulv(thr, m.emissive), R.w_e));
    if (R.nee) {
      const V3 c = st.enable_mis ? mul(mulv(thr, R.q.radiance), R.w_n) : mulv(thr, R.q.radiance);
      bool vis = true;
      if (R.q.remain > 0.004f) vis = !trace_any<false>(s, prep_ray(R.q.origin, R.q.dir, s.reference_tree != 0u),
                                                       R.q.remain, stk, ts, err);
      if (vis) {
        rad = add(rad, c);
        flags |= kVfNeeVis;
      }
    }
    const V3 thr_at = thr;
    float rr = 1.0f;
    bool cont = false;
    if (R.scattered) {
      const V3 wgt = albedo_effect0(m);
      const V3 wgt0 = albedo_effect0(load_material(mat0 + 16u * mi));
      thr = mulv(thr, wgt);
      thr0 = mulv(thr0, wgt0);
      const float tmx = smax(thr0.x, smax(thr0.y, thr0.z));
      if (!(tmx < 0.001f)) {
        rr = smin(st.rr_max, smax(st.rr_min, tmx));
        if (!(depth >= st.rr_start && next01(rng) > rr)) {
          thr = divs(thr, rr);
          thr0 = divs(thr0, rr);
          cont = depth + 1u < st.max_depth;
          o = add(R.hp, mul(R.out, 0.002f));
          d = R.out;
        }
      }
    }
    sig = mix64(sig ^ (static_cast<uint64_t>(prim + 1u) | (static_cast<uint64_t>(flags | (cont ? kVfCont : 0u)) << 32)));
    if (kRecord) {
      AdjRec& r = rec[static_cast<size_t>(nrec++) * rec_stride];
      r.a = make_float4(o_at.x, o_at.y, o_at.z, t);
      r.b = make_float4(d_at.x, d_at.y, d_at.z, __uint_as_float(prim));
      r.c = make_float4(thr_at.x, thr_at.y, thr_at.z, rr);
      r.e = make_uint4(static_cast<uint32_t>(rng_at), static_cast<uint32_t>(rng_at >> 32),
                       flags | (cont ? kVfCont : 0u), mi);
    }
    if (!cont) break;
  }
  return make_float4(rad.x, rad.y, rad.z, __uint_as_float(static_cast<uint32_t>(sig ^ (sig >> 32))));
}

// 102 registers (5 blocks of 128 threads per SM): 1.98 -> 1.87 ms per forward pass.
// kRecord: the forward also writes every path's vertex records (recs, the
// backward's layout with all paths as one chunk) and their count (nrec), so
// a backward over the same paths needs no replay.
template <bool kParity, bool kRecord>
__global__ void __launch_bounds__(128, 5) k_adj_forward(DevScene s, DevSettings st, const float* mat0, uint32_t spp,
                                                     uint32_t first_sample, int cap, float4* rad, AdjRec* recs,
                                                     uint32_t* nrec_out, uint32_t* err) {
  extern __shared__ int2 smem_stack[];
  SmemStack stk{smem_stack + threadIdx.x, static_cast<int>(blockDim.x), cap};
  const uint32_t npx = st.width * st.height;
  const uint64_t n = static_cast<uint64_t>(npx) * spp;
  uint32_t local_err = 0u;
  for (uint64_t j = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; j < n;
       j += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint32_t sl = static_cast<uint32_t>(j / npx), p = static_cast<uint32_t>(j % npx);
    uint32_t nrec = 0u;
    if (kRecord) {
      rad[j] = adj_primal<kParity, true>(s, st, mat0, p % st.width, p / st.width, first_sample + sl, stk, local_err,
                                         recs + j, nrec, static_cast<uint32_t>(n));
      nrec_out[j] = nrec;
    } else {
      rad[j] = adj_primal<kParity, false>(s, st, mat0, p % st.width, p / st.width, first_sample + sl, stk, local_err,
                                          nullptr, nrec);
    }
  }
  if (local_err) atomicOr(err, local_err);
}

// Per pixel: film accumulation in sample order (non-finite samples dropped,
// optional firefly clamp), resolve, squared error (FP64) and the adjoint of
// each sample's radiance, 2 (img - target) / (3 W H) / count.
__global__ void __launch_bounds__(256) k_adj_loss(DevSettings st, uint32_t spp, const float4* rad, const float* target,
                                                  float* image, float4* adj, double* loss_part) {
  __shared__ double red[256];
  const uint32_t npx = st.width * st.height;
  double local = 0.0;
  const float scale = 2.0f / (3.0f * static_cast<float>(npx));
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < npx; p += gridDim.x * blockDim.x) {
    float ax = 0.0f, ay = 0.0f, az = 0.0f;
    uint32_t cnt = 0u;
    for (uint32_t sl = 0; sl < spp; ++sl) {
      const float4 r = rad[static_cast<size_t>(sl) * npx + p];
      if (!(isfinite(r.x) && isfinite(r.y) && isfinite(r.z))) continue;
      float cx = r.x, cy = r.y, cz = r.z;
      if (st.firefly_clamp > 0.0f) {
        cx = smin(cx, st.firefly_clamp);
        cy = smin(cy, st.firefly_clamp);
        cz = smin(cz, st.firefly_clamp);
      }
      ax = ax + cx;
      ay = ay + cy;
      az = az + cz;
      ++cnt;
    }
    const float inv = 1.0f / static_cast<float>(cnt > 1u ? cnt : 1u);
    const float ix = ax * inv, iy = ay * inv, iz = az * inv;
    image[3 * p + 0] = ix;
    image[3 * p + 1] = iy;
    image[3 * p + 2] = iz;
    float4 g = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (target) {
      const float dx = ix - target[3 * p + 0], dy = iy - target[3 * p + 1], dz = iz - target[3 * p + 2];
      local += static_cast<double>(dx) * dx + static_cast<double>(dy) * dy + static_cast<double>(dz) * dz;
      g = make_float4(scale * dx * inv, scale * dy * inv, scale * dz * inv, 0.0f);
    }
    adj[p] = g;
  }
  red[threadIdx.x] = local;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (static_cast<int>(threadIdx.x) < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) loss_part[blockIdx.x] = red[0];
}

__global__ void k_adj_loss_final(const double* part, int n, double scale, double* loss) {
  __shared__ double red[256];
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += part[i];
  red[threadIdx.x] = v;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (static_cast<int>(threadIdx.x) < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *loss = red[0] * scale;
}

__device__ __forceinline__ DV3 seed3(V3 v, int first) {
  DV3 r = lift<DV3>(v);
  r.x.g[first] = 1.0f;
  r.y.g[first + 1] = 1.0f;
  r.z.g[first + 2] = 1.0f;
  return r;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Reverse sweep of one path.  `g` is dL/d(path radiance).  The warp runs the
// vertex loop in lockstep (k from the longest path's last vertex down) so the
// per-vertex gradients can be combined across lanes.
template <bool kParity>
__device__ __forceinline__ void adj_reverse(const DevScene& s, const DevSettings& st, const AdjRec* rec,
                                            uint32_t rec_stride, uint32_t nrec, bool lane_on, V3 g,
                                            float* warp_grad) {
  const uint32_t kmax = __reduce_max_sync(0xffffffffu, lane_on ? nrec : 0u);
  const int lane = threadIdx.x & 31;
  V3 aT = mk(0.0f, 0.0f, 0.0f), aO = aT, aD = aT;
  for (int k = static_cast<int>(kmax) - 1; k >= 0; --k) {
    const bool act = lane_on && k < static_cast<int>(nrec);
    uint32_t mat = kMiss;
    float gv[kAdjParams] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    if (act) {
      const AdjRec r = rec[static_cast<size_t>(k) * rec_stride];
      const uint32_t flags = r.e.z;
      const V3 T = mk(r.c.x, r.c.y, r.c.z);
      if (flags & kVfMiss) {
        aT = mulv(g, s.env);
        aO = aD = mk(0.0f, 0.0f, 0.0f);
      } else {
        const uint32_t prim = __float_as_uint(r.b.w);
        const float4 sh = __ldg(s.shade + prim);
        const V3 gn = mk(sh.x, sh.y, sh.z);
        mat = r.e.w;
        const MaterialRec m = load_material(s.materials + 16u * mat);
        const V3 ov = mk(r.a.x, r.a.y, r.a.z), dv = mk(r.b.x, r.b.y, r.b.z);
        const float th = r.a.w;
        // Seeds: origin (0..2), direction (3..5), roughness (6).
        const DV3 od = seed3(ov, 0), dd = seed3(dv, 3);
        Dual rough = dconst(clamp01(m.roughness));
        rough.g[6] = (m.roughness > 0.0f && m.roughness < 1.0f) ? 1.0f : 0.0f;
        // Hit distance on the hit triangle's plane: t = (v0 - o).n / (d.n).
        Dual tt = dconst(th);
        const float dn = dot(dv, gn);
        if (dn != 0.0f) {
          tt.g[0] = -gn.x / dn;
          tt.g[1] = -gn.y / dn;
          tt.g[2] = -gn.z / dn;
          tt.g[3] = -th * gn.x / dn;
          tt.g[4] = -th * gn.y / dn;
          tt.g[5] = -th * gn.z / dn;
        }
        uint64_t rng = static_cast<uint64_t>(r.e.x) | (static_cast<uint64_t>(r.e.y) << 32);
        uint32_t fl = flags;
        AdjVertex<Dual, DV3> R;
        adj_vertex<Dual, DV3, kParity, true>(s, st, s.lights, static_cast<uint32_t>(k), od, dd, tt, gn, m, rough,
                                             rng, fl, R);
        float xb[kAdjN];
#pragma unroll
        for (int i = 0; i < kAdjN; ++i) xb[i] = 0.0f;
        V3 aTk = mk(0.0f, 0.0f, 0.0f);
        const V3 amask = mk((m.albedo.x > 0.0f && m.albedo.x < 1.5f) ? 1.0f : 0.0f,
                            (m.albedo.y > 0.0f && m.albedo.y < 1.5f) ? 1.0f : 0.0f,
                            (m.albedo.z > 0.0f && m.albedo.z < 1.5f) ? 1.0f : 0.0f);
        // emission: (T * Le) * w_e
        {
          const float we = R.w_e.v;
          const float se = g.x * T.x * m.emissive.x + g.y * T.y * m.emissive.y + g.z * T.z * m.emissive.z;
#pragma unroll
          for (int i = 0; i < kAdjN; ++i) xb[i] += se * R.w_e.g[i];
          gv[4] = g.x * T.x * we;
          gv[5] = g.y * T.y * we;
          gv[6] = g.z * T.z * we;
          aTk = mk(g.x * m.emissive.x * we, g.y * m.emissive.y * we, g.z * m.emissive.z * we);
        }
        // next-event term: (T * R) * w_n when it was added
        if (R.nee && (flags & kVfNeeVis)) {
          const float wn = R.w_n.v;
          const V3 q = mk(g.x * T.x, g.y * T.y, g.z * T.z);
          const float sr = q.x * R.q.radiance.x.v + q.y * R.q.radiance.y.v + q.z * R.q.radiance.z.v;
#pragma unroll
          for (int i = 0; i < kAdjN; ++i)
            xb[i] += wn * (q.x * R.q.radiance.x.g[i] + q.y * R.q.radiance.y.g[i] + q.z * R.q.radiance.z.g[i]) +
                     sr * R.w_n.g[i];
          gv[0] += q.x * wn * R.q.p_alb.x * amask.x;
          gv[1] += q.y * wn * R.q.p_alb.y * amask.y;
          gv[2] += q.z * wn * R.q.p_alb.z * amask.z;
          aTk = add(aTk, mk(g.x * R.q.radiance.x.v * wn, g.y * R.q.radiance.y.v * wn, g.z * R.q.radiance.z.v * wn));
        }
        // throughput T' = T * albedo / rr (rr held constant) and the next ray
        if (flags & kVfCont) {
          const float inv_rr = 1.0f / r.c.w;
          const V3 W = albedo_effect0(m);
          aTk = add(aTk, mk(aT.x * W.x * inv_rr, aT.y * W.y * inv_rr, aT.z * W.z * inv_rr));
          gv[0] += aT.x * T.x * inv_rr * amask.x;
          gv[1] += aT.y * T.y * inv_rr * amask.y;
          gv[2] += aT.z * T.z * inv_rr * amask.z;
          const DV3 o2 = add(R.hp, mul(R.out, 0.002f));
#pragma unroll
          for (int i = 0; i < kAdjN; ++i)
            xb[i] += aO.x * o2.x.g[i] + aO.y * o2.y.g[i] + aO.z * o2.z.g[i] + aD.x * R.out.x.g[i] +
                     aD.y * R.out.y.g[i] + aD.z * R.out.z.g[i];
        }
        gv[3] = xb[6];
        aT = aTk;
        aO = mk(xb[0], xb[1], xb[2]);
        aD = mk(xb[3], xb[4], xb[5]);
      }
    }
    // Combine lanes that hit the same material, one group at a time.
    unsigned pending = __ballot_sync(0xffffffffu, mat != kMiss);
    while (pending) {
      const int leader = __ffs(pending) - 1;
      const uint32_t gm = __shfl_sync(0xffffffffu, mat, leader);
      const bool mine = mat == gm;
#pragma unroll
      for (int i = 0; i < static_cast<int>(kAdjParams); ++i) {
        const float v = warp_sum(mine ? gv[i] : 0.0f);
        if (lane == leader) warp_grad[gm * kAdjParams + i] += v;
      }
      pending &= ~__ballot_sync(0xffffffffu, mine);
    }
  }
}

// The backward runs as two kernels per chunk of paths: the replay (the
// primal path again, with the traversal) writes every path's vertex records
// and its radiance adjoint to device memory, and the reverse sweep (the dual-
// number vertex code) reads them.  Split, each kernel's code is small enough
// for the instruction cache -- the fused kernel's warps waited on instruction
// fetch more than on anything else -- and each gets its own register budget.
// Records: vertex k of chunk path i at recs[k * count + i] (lanes of a warp
// touch consecutive records).
template <bool kParity>
__global__ void __launch_bounds__(128, 5) k_adj_replay(DevScene s, DevSettings st, const float* mat0,
                                                    uint32_t first_sample, int cap, const float4* adj,
                                                    const float* path_weight, uint64_t base, uint32_t count,
                                                    AdjRec* recs, float4* gout, uint32_t* err) {
  extern __shared__ int2 smem_dyn[];
  SmemStack stk{smem_dyn + threadIdx.x, static_cast<int>(blockDim.x), cap};
  const uint32_t npx = st.width * st.height;
  uint32_t local_err = 0u;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const uint64_t j = base + i;
    const uint32_t sl = static_cast<uint32_t>(j / npx), p = static_cast<uint32_t>(j % npx);
    float4 a = adj[p];
    if (path_weight) {
      const float pw = path_weight[j];
      a = make_float4(a.x * pw, a.y * pw, a.z * pw, 0.0f);
    }
    V3 g = mk(0.0f, 0.0f, 0.0f);
    uint32_t nrec = 0u;
    if (a.x != 0.0f || a.y != 0.0f || a.z != 0.0f) {
      // The replayed radiance decides what the film would have dropped or
      // clamped (the replay may use other samples than the forward's).
      const float4 rv = adj_primal<kParity, true>(s, st, mat0, p % st.width, p / st.width, first_sample + sl, stk,
                                                  local_err, recs + i, nrec, count);
      const float fc = st.firefly_clamp;
      g = mk((fc > 0.0f && rv.x > fc) ? 0.0f : a.x, (fc > 0.0f && rv.y > fc) ? 0.0f : a.y,
             (fc > 0.0f && rv.z > fc) ? 0.0f : a.z);
      if (!(isfinite(rv.x) && isfinite(rv.y) && isfinite(rv.z))) nrec = 0u;
    }
    gout[i] = make_float4(g.x, g.y, g.z, __uint_as_float(nrec));
  }
  if (local_err) atomicOr(err, local_err);
}

// What the replay hands the reverse sweep, for paths the forward recorded
// (the same paths): each path's radiance adjoint (zero where the film
// dropped or clamped the sample, the path's weight applied) and its record
// count (0: nothing to sweep).
__global__ void __launch_bounds__(256) k_adj_gout(DevSettings st, const float4* adj, const float* path_weight,
                                                  const float4* rad, const uint32_t* nrec_fwd, uint32_t count,
                                                  float4* gout) {
  const uint32_t npx = st.width * st.height;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    float4 a = adj[i % npx];
    if (path_weight) {
      const float pw = path_weight[i];
      a = make_float4(a.x * pw, a.y * pw, a.z * pw, 0.0f);
    }
    V3 g = mk(0.0f, 0.0f, 0.0f);
    uint32_t nrec = 0u;
    if (a.x != 0.0f || a.y != 0.0f || a.z != 0.0f) {
      const float4 rv = rad[i];
      const float fc = st.firefly_clamp;
      g = mk((fc > 0.0f && rv.x > fc) ? 0.0f : a.x, (fc > 0.0f && rv.y > fc) ? 0.0f : a.y,
             (fc > 0.0f && rv.z > fc) ? 0.0f : a.z);
      nrec = (isfinite(rv.x) && isfinite(rv.y) && isfinite(rv.z)) ? nrec_fwd[i] : 0u;
    }
    gout[i] = make_float4(g.x, g.y, g.z, __uint_as_float(nrec));
  }
}

// The reverse sweep of one chunk: per-warp gradient slots in shared memory,
// then one partial per block, added to the partials of the earlier chunks
// (accumulate) in a fixed order, so the gradient is deterministic.
#ifndef VKPTC_ADJ_REVERSE_BLOCKS
#define VKPTC_ADJ_REVERSE_BLOCKS 4
#endif
template <bool kParity>
__global__ void __launch_bounds__(128, VKPTC_ADJ_REVERSE_BLOCKS) k_adj_reverse(DevScene s, DevSettings st, uint32_t count,
                                                     const AdjRec* recs, const float4* gout, float* grad_part,
                                                     int accumulate) {
  extern __shared__ float grads[];
  const int warps = blockDim.x >> 5;
  const uint32_t stride = s.material_count * kAdjParams;
  for (uint32_t i = threadIdx.x; i < stride * warps; i += blockDim.x) grads[i] = 0.0f;
  __syncthreads();
  float* warp_grad = grads + (threadIdx.x >> 5) * stride;
  for (uint32_t base = blockIdx.x * blockDim.x; base < count; base += gridDim.x * blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    V3 g = mk(0.0f, 0.0f, 0.0f);
    uint32_t nrec = 0u;
    if (i < count) {
      const float4 gv = gout[i];
      g = mk(gv.x, gv.y, gv.z);
      nrec = __float_as_uint(gv.w);
    }
    adj_reverse<kParity>(s, st, recs + (i < count ? i : 0u), count, nrec, nrec != 0u, g, warp_grad);
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < stride; i += blockDim.x) {
    float v = 0.0f;
    for (int w = 0; w < warps; ++w) v += grads[w * stride + i];
    float* dst = grad_part + static_cast<size_t>(blockIdx.x) * stride + i;
    *dst = accumulate ? *dst + v : v;
  }
}

__global__ void k_adj_grad_reduce(const float* part, int blocks, uint32_t stride, float* grad) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < stride; i += gridDim.x * blockDim.x) {
    double v = 0.0;
    for (int b = 0; b < blocks; ++b) v += part[static_cast<size_t>(b) * stride + i];
    grad[i] = static_cast<float>(v);
  }
}

}  // namespace

size_t AdjForwardSmem(int block, int stack_cap) { return static_cast<size_t>(block) * stack_cap * sizeof(int2); }

size_t AdjBackwardSmem(int block, int stack_cap, uint32_t materials) {
  return std::max(AdjForwardSmem(block, stack_cap), AdjReverseSmem(block, materials));
}

size_t AdjReverseSmem(int block, uint32_t materials) {
  return static_cast<size_t>(block / 32) * materials * kAdjParams * sizeof(float);
}

int AdjBlocksPerSm(AdjKernel k, int block, size_t smem, bool parity) {
  int n = 0;
  switch (k) {
    case AdjKernel::kForward:
      if (parity) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_adj_forward<true, false>, block, smem);
      else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_adj_forward<false, false>, block, smem);
      break;
    case AdjKernel::kReplay:
      if (parity) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_adj_replay<true>, block, smem);
      else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_adj_replay<false>, block, smem);
      break;
    case AdjKernel::kReverse:
      if (parity) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_adj_reverse<true>, block, smem);
      else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_adj_reverse<false>, block, smem);
      break;
  }
  return n > 0 ? n : 1;
}

cudaError_t ConfigureAdjSmem(size_t bytes) {
  const int b = static_cast<int>(bytes);
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(k_adj_forward<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, b))) return e;
  if ((e = cudaFuncSetAttribute(k_adj_forward<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, b))) return e;
  if ((e = cudaFuncSetAttribute(k_adj_forward<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, b))) return e;
  if ((e = cudaFuncSetAttribute(k_adj_forward<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, b))) return e;
  if ((e = cudaFuncSetAttribute(k_adj_replay<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, b))) return e;
  if ((e = cudaFuncSetAttribute(k_adj_replay<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, b))) return e;
  if ((e = cudaFuncSetAttribute(k_adj_reverse<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, b))) return e;
  return cudaFuncSetAttribute(k_adj_reverse<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
}

cudaError_t LaunchAdjForward(const DevScene& s, const DevSettings& st, const float* mat0, const AdjLaunch& l,
                             float4* rad, uint32_t* err, float4* recs, uint32_t* nrec) {
  const size_t smem = AdjForwardSmem(l.block, l.stack_cap);
  AdjRec* r = reinterpret_cast<AdjRec*>(recs);
  const bool rec = recs != nullptr && nrec != nullptr;
  if (l.parity && rec)
    k_adj_forward<true, true><<<l.grid, l.block, smem, l.stream>>>(s, st, mat0, l.spp, l.first_sample, l.stack_cap, rad,
                                                                   r, nrec, err);
  else if (l.parity)
    k_adj_forward<true, false><<<l.grid, l.block, smem, l.stream>>>(s, st, mat0, l.spp, l.first_sample, l.stack_cap,
                                                                    rad, nullptr, nullptr, err);
  else if (rec)
    k_adj_forward<false, true><<<l.grid, l.block, smem, l.stream>>>(s, st, mat0, l.spp, l.first_sample, l.stack_cap,
                                                                    rad, r, nrec, err);
  else
    k_adj_forward<false, false><<<l.grid, l.block, smem, l.stream>>>(s, st, mat0, l.spp, l.first_sample, l.stack_cap,
                                                                     rad, nullptr, nullptr, err);
  return cudaGetLastError();
}

cudaError_t LaunchAdjLoss(const DevSettings& st, uint32_t spp, const float4* rad, const float* target, float* image,
                          float4* adj, double* loss_part, double* loss, int grid, cudaStream_t stream) {
  k_adj_loss<<<grid, 256, 0, stream>>>(st, spp, rad, target, image, adj, loss_part);
  const double npx = static_cast<double>(st.width) * st.height;
  k_adj_loss_final<<<1, 256, 0, stream>>>(loss_part, grid, 1.0 / (3.0 * npx), loss);
  return cudaGetLastError();
}

cudaError_t LaunchAdjBackward(const DevScene& s, const DevSettings& st, const float* mat0, const AdjLaunch& l,
                              const float4* adj, const float* path_weight, float4* recs, float4* gout,
                              float* grad_part, float* grad, uint32_t* err, const float4* fwd_rad,
                              const uint32_t* fwd_nrec) {
  const size_t smem_replay = AdjForwardSmem(l.block, l.stack_cap);
  const size_t smem_rev = AdjReverseSmem(l.block, s.material_count);
  const uint64_t n = static_cast<uint64_t>(st.width) * st.height * l.spp;
  AdjRec* r = reinterpret_cast<AdjRec*>(recs);
  if (fwd_rad != nullptr && fwd_nrec != nullptr && n <= kAdjChunkPaths) {
    // the forward recorded these paths: no replay
    const uint32_t count = static_cast<uint32_t>(n);
    k_adj_gout<<<static_cast<int>(std::min<uint64_t>(4096, (n + 255) / 256)), 256, 0, l.stream>>>(
        st, adj, path_weight, fwd_rad, fwd_nrec, count, gout);
    if (l.parity) k_adj_reverse<true><<<l.grid_reverse, l.block, smem_rev, l.stream>>>(s, st, count, r, gout, grad_part, 0);
    else k_adj_reverse<false><<<l.grid_reverse, l.block, smem_rev, l.stream>>>(s, st, count, r, gout, grad_part, 0);
    const uint32_t stride = s.material_count * kAdjParams;
    k_adj_grad_reduce<<<(stride + 127) / 128, 128, 0, l.stream>>>(grad_part, l.grid_reverse, stride, grad);
    return cudaGetLastError();
  }
  for (uint64_t base = 0; base < n; base += kAdjChunkPaths) {
    const uint32_t count = static_cast<uint32_t>(std::min<uint64_t>(kAdjChunkPaths, n - base));
    const int acc = base > 0 ? 1 : 0;
    if (l.parity) {
      k_adj_replay<true><<<l.grid, l.block, smem_replay, l.stream>>>(s, st, mat0, l.first_sample, l.stack_cap, adj,
                                                                   path_weight, base, count, r, gout, err);
      k_adj_reverse<true><<<l.grid_reverse, l.block, smem_rev, l.stream>>>(s, st, count, r, gout, grad_part, acc);
    } else {
      k_adj_replay<false><<<l.grid, l.block, smem_replay, l.stream>>>(s, st, mat0, l.first_sample, l.stack_cap, adj,
                                                                    path_weight, base, count, r, gout, err);
      k_adj_reverse<false><<<l.grid_reverse, l.block, smem_rev, l.stream>>>(s, st, count, r, gout, grad_part, acc);
    }
  }
  const uint32_t stride = s.material_count * kAdjParams;
  k_adj_grad_reduce<<<(stride + 127) / 128, 128, 0, l.stream>>>(grad_part, l.grid_reverse, stride, grad);
  return cudaGetLastError();
}

}  // namespace vkptc
