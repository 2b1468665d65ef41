// batch.cu -- the persistent batched renderer.
//
// Many render jobs of uneven triangle count, resolution, spp and depth run in
// ONE cooperative launch.  The launch owns a pool of path slots; a device
// work queue (one 64-bit counter over all jobs' paths, job-major then sample-
// major) refills every slot whose path has ended, so the GPU stays full until
// the last path of the last job.  Each iteration runs the wavefront stages
// over the whole pool, separated by a grid barrier:
//   REGEN   free slots take the next path ids; camera ray + RNG key
//   EXTEND  closest-hit traversal of the extension queue (persistent warps)
//   SHADE   one bounce of the reference integrator per path; appends the
//           shadow queue, the next extension queue, or the finished list
//   SHADOW  any-hit traversal of the NEE queries; adds visible NEE terms
//   FINISH  finished paths write their radiance to the job's staging slot
//           (sample, pixel) and return their slot to the free list
// The stagings are then added to each job's film in sample order, so the film
// is bit-identical to rendering the job one sample (one launch) at a time.
//
// The grid barrier is a counter/generation barrier whose wait is bounded: a
// block that waits longer than its bound (BatchPool::barrier_spins sleeps of
// ~128 ns, ~8.6 s by default) sets an abort word, and every block leaves the
// loop at its next barrier; the host reports a timeout.  The
// launch is cooperative, so all blocks are co-resident by construction.
#include <cooperative_groups.h>

#include "batch.cuh"
#include "integrator.cuh"
#include "traverse.cuh"

namespace vkptc {

namespace {

// Control words of BatchPool::ctl.
constexpr int kCtlExt0 = 0, kCtlExt1 = 1, kCtlShadow = 2, kCtlFin = 3, kCtlFree = 4;
constexpr int kCtlFetchExt = 5, kCtlFetchShadow = 6;
constexpr int kCtlWork = 8;      // 64-bit path counter (words 8, 9)
constexpr int kCtlBarCount = 12, kCtlBarGen = 13, kCtlAbort = 15;
constexpr int kCtlIter = kBatchCtlIterations;

// spin_limit: sleeps of ~128 ns a block waits before it raises the abort word.
__device__ __forceinline__ bool grid_barrier(uint32_t* ctl, uint32_t spin_limit) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile uint32_t* gen_p = ctl + kCtlBarGen;
    volatile uint32_t* abort_p = ctl + kCtlAbort;
    const uint32_t gen = *gen_p;
    __threadfence();
    const uint32_t arrived = atomicAdd(ctl + kCtlBarCount, 1u);
    if (arrived == gridDim.x - 1u) {
      atomicExch(ctl + kCtlBarCount, 0u);
      __threadfence();
      atomicAdd(ctl + kCtlBarGen, 1u);
    } else {
      unsigned spins = 0u;
      while (*gen_p == gen && *abort_p == 0u) {
        if (++spins > spin_limit) {
          atomicExch(ctl + kCtlAbort, 1u);
          break;
        }
        __nanosleep(128);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return *reinterpret_cast<volatile uint32_t*>(ctl + kCtlAbort) == 0u;
}

__device__ __forceinline__ GeoView job_geo(const DevJob* jobs, uint32_t j) { return geo_of(jobs[j].scene); }

struct BatchExtendSource {
  const DevJob* jobs;
  const uint32_t* q;
  const uint32_t* job;
  const float4* ray_o;
  const float4* ray_d;
  float2* hit;
  __device__ __forceinline__ void load(uint32_t j, V3& o, V3& d, float& tm, GeoView& g) const {
    const uint32_t slot = q[j];
    g = job_geo(jobs, job[slot]);
    const float4 a = ray_o[slot], b = ray_d[slot];
    o = mk(a.x, a.y, a.z);
    d = mk(b.x, b.y, b.z);
    tm = kInf;
  }
  __device__ __forceinline__ void finish(uint32_t j, float t, uint32_t prim) const {
    hit[q[j]] = make_float2(t, __uint_as_float(prim));
  }
};

struct BatchShadowSource {
  const DevJob* jobs;
  const uint32_t* q;
  const uint32_t* job;
  const float4* sh_o;
  const float4* sh_d;
  const float4* sh_c;
  float4* rad;
  __device__ __forceinline__ void load(uint32_t j, V3& o, V3& d, float& tm, GeoView& g) const {
    const uint32_t slot = q[j];
    g = job_geo(jobs, job[slot]);
    const float4 a = sh_o[j], b = sh_d[j];
    o = mk(a.x, a.y, a.z);
    d = mk(b.x, b.y, b.z);
    tm = a.w;
  }
  __device__ __forceinline__ void finish(uint32_t j, float, uint32_t occluded) const {
    if (occluded) return;
    const uint32_t slot = q[j];
    const float4 c = sh_c[j];
    float4 r = rad[slot];
    r.x = r.x + c.x;
    r.y = r.y + c.y;
    r.z = r.z + c.z;
    rad[slot] = r;
  }
};

// ------------------------------------------------------------------ phases
// The five stages of one iteration over the pool, separated by grid
// barriers in the persistent kernel.  Each is grid-stride over a device-side
// count.

// REGEN: free slots take the next path ids of the work queue, generate the
// camera ray and append to the extension queue `cur`.
template <bool kParity>
__device__ __forceinline__ void phase_regen(const DevJob* __restrict__ jobs, uint32_t job_count,
                                            unsigned long long total, const BatchPool& P, uint32_t cur) {
  const uint32_t gthreads = gridDim.x * blockDim.x;
  const unsigned lane = threadIdx.x & 31u;
  unsigned long long* work_next = reinterpret_cast<unsigned long long*>(P.ctl + kCtlWork);
  const uint32_t nfree = P.ctl[kCtlFree];
  for (uint32_t base = blockIdx.x * blockDim.x; base < nfree; base += gthreads) {
    const uint32_t j = base + threadIdx.x;
    const bool want = j < nfree;
    const unsigned mask = __ballot_sync(0xffffffffu, want);
    unsigned long long g0 = 0ull;
    const int lead = __ffs(mask) - 1;
    if (mask != 0u && static_cast<int>(lane) == lead) g0 = atomicAdd(work_next, static_cast<unsigned long long>(__popc(mask)));
    g0 = __shfl_sync(0xffffffffu, g0, lead < 0 ? 0 : lead);
    const unsigned long long g = g0 + static_cast<unsigned long long>(__popc(mask & ((1u << lane) - 1u)));
    const bool ok = want && g < total;
    uint32_t slot = 0u;
    if (ok) {
      slot = P.freel[j];
      const uint32_t jb = find_job(jobs, job_count, g);
      const DevJob& J = jobs[jb];
      const uint32_t local = static_cast<uint32_t>(g - J.path_base);
      const uint32_t sl = local / J.pixels, px = local - sl * J.pixels;
      const uint32_t W = J.settings.width;
      V3 o, d;
      uint64_t rng;
      camera_path<kParity>(J.scene, J.settings, px % W, px / W, J.first_sample + sl, o, d, rng);
      P.job[slot] = jb;
      P.local[slot] = local;
      P.depth[slot] = 0u;
      P.rng[slot] = rng;
      P.ray_o[slot] = make_float4(o.x, o.y, o.z, 0.0f);
      P.ray_d[slot] = make_float4(d.x, d.y, d.z, 0.0f);
      P.thr[slot] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
      P.rad[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    const uint32_t qi = warp_append(&P.ctl[cur], ok);
    if (ok) P.ext[cur][qi] = slot;
  }
}

// SHADE: one bounce of the integrator for every path of extension queue
// `cur`; appends to the next extension queue, the shadow queue, or the
// finished list.  Returns this thread's shadow-test count.
template <bool kParity>
__device__ __forceinline__ uint32_t phase_shade(const DevJob* __restrict__ jobs, const BatchPool& P, uint32_t cur,
                                                uint32_t n_ext) {
  const uint32_t gthreads = gridDim.x * blockDim.x;
  uint32_t shadow_tests = 0u;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n_ext; base += gthreads) {
    const uint32_t j = base + threadIdx.x;
    bool next = false, shadow = false, fin = false;
    uint32_t slot = 0u;
    ShadeOut R;
    if (j < n_ext) {
      slot = P.ext[cur][j];
      const DevJob& J = jobs[P.job[slot]];
      const uint32_t depth = P.depth[slot];
      const float4 o4 = P.ray_o[slot], d4 = P.ray_d[slot], t4 = P.thr[slot], r4 = P.rad[slot];
      const float2 h2 = P.hit[slot];
      PathRegs pr;
      pr.o = mk(o4.x, o4.y, o4.z);
      pr.d = mk(d4.x, d4.y, d4.z);
      pr.thr = mk(t4.x, t4.y, t4.z);
      pr.rad = mk(r4.x, r4.y, r4.z);
      pr.segs = r4.w;
      pr.rng = P.rng[slot];
      R = shade_bounce<kParity>(J.scene, J.settings, J.scene.lights, depth, pr, h2.x, __float_as_uint(h2.y));
      if (R.next) {
        P.ray_o[slot] = make_float4(pr.o.x, pr.o.y, pr.o.z, 0.0f);
        P.ray_d[slot] = make_float4(pr.d.x, pr.d.y, pr.d.z, 0.0f);
        P.thr[slot] = make_float4(pr.thr.x, pr.thr.y, pr.thr.z, 0.0f);
        P.rng[slot] = pr.rng;
        P.depth[slot] = depth + 1u;
      }
      P.rad[slot] = make_float4(pr.rad.x, pr.rad.y, pr.rad.z, pr.segs);
      next = R.next;
      fin = !R.next;
      shadow = R.shadow;
      shadow_tests += R.shadow_tests;
    }
    const uint32_t qn = warp_append(&P.ctl[cur ^ 1u], next);
    if (next) P.ext[cur ^ 1u][qn] = slot;
    const uint32_t qf = warp_append(&P.ctl[kCtlFin], fin);
    if (fin) P.fin[qf] = slot;
    const uint32_t qs = warp_append(&P.ctl[kCtlShadow], shadow);
    if (shadow) {
      P.shq[qs] = slot;
      P.sh_o[qs] = make_float4(R.sh_o.x, R.sh_o.y, R.sh_o.z, R.sh_t);
      P.sh_d[qs] = make_float4(R.sh_d.x, R.sh_d.y, R.sh_d.z, 0.0f);
      P.sh_c[qs] = make_float4(R.sh_c.x, R.sh_c.y, R.sh_c.z, 0.0f);
    }
  }
  return shadow_tests;
}

// FINISH: finished paths write their radiance to the job's staging slot and
// return their slot to the free list.
__device__ __forceinline__ void phase_finish(const DevJob* __restrict__ jobs, const BatchPool& P) {
  const uint32_t gthreads = gridDim.x * blockDim.x;
  const uint32_t n_fin = P.ctl[kCtlFin];
  for (uint32_t base = blockIdx.x * blockDim.x; base < n_fin; base += gthreads) {
    const uint32_t j = base + threadIdx.x;
    const bool ok = j < n_fin;
    uint32_t slot = 0u;
    if (ok) {
      slot = P.fin[j];
      const DevJob& J = jobs[P.job[slot]];
      J.staging[P.local[slot]] = P.rad[slot];
    }
    const uint32_t qi = warp_append(&P.ctl[kCtlFree], ok);
    if (ok) P.freel[qi] = slot;
  }
}

__device__ __forceinline__ TwoLevelStack batch_stack(int2* smem_stack, int scap, int2* spill, int total_cap) {
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t gthreads = gridDim.x * blockDim.x;
  return TwoLevelStack{smem_stack + threadIdx.x, static_cast<int>(blockDim.x), scap,
                       spill ? spill + gtid : nullptr, static_cast<int>(gthreads), total_cap};
}

template <bool kStats>
__device__ __forceinline__ void flush_traversal_stats(DevCounters* ctr, const TraceStats& st_e, const TraceStats& st_s) {
  if (kStats) {
    warp_count(&ctr->nodes, st_e.nodes);
    warp_count(&ctr->leaves, st_e.leaves);
    warp_count(&ctr->tris, st_e.tris);
    warp_count(&ctr->ext_rays, st_e.rays);
    warp_count(&ctr->shadow_nodes, st_s.nodes);
    warp_count(&ctr->shadow_leaves, st_s.leaves);
    warp_count(&ctr->shadow_tris, st_s.tris);
    warp_count(&ctr->shadow_rays, st_s.rays);
  }
}

}  // namespace

// ------------------------------------------------------- persistent driver
// kMinBlocks: resident 256-thread blocks per SM the register allocation must
// allow (0 = compiler's choice); the autotuner picks the occupancy/spill trade-off.
template <bool kParity, bool kStats, int kMinBlocks, bool kWt>
__global__ void __launch_bounds__(256, kMinBlocks) k_batch(const DevJob* __restrict__ jobs, uint32_t job_count,
                                                           unsigned long long total, BatchPool P, int scap,
                                                           int2* spill, int total_cap, int steps, DevCounters* ctr,
                                                           uint32_t* err) {
  extern __shared__ int2 smem_stack[];
  const TwoLevelStack stk = batch_stack(smem_stack, scap, spill, total_cap);
  TraceStats st_e, st_s;
  uint32_t lerr = 0u;
  uint32_t shadow_tests = 0u;
  uint32_t cur = 0u;
  const bool leader = blockIdx.x == 0 && threadIdx.x == 0;

  while (true) {
    if (leader) P.ctl[kCtlFetchExt] = 0u;
    phase_regen<kParity>(jobs, job_count, total, P, cur);
    if (!grid_barrier(P.ctl, P.barrier_spins)) break;

    const uint32_t n_ext = P.ctl[cur];
    if (n_ext == 0u) break;   // no live path and no work left (same value in every block)
    if (leader) {
      P.ctl[cur ^ 1u] = 0u;
      P.ctl[kCtlShadow] = 0u;
      P.ctl[kCtlFin] = 0u;
      P.ctl[kCtlFree] = 0u;
      P.ctl[kCtlFetchShadow] = 0u;
    }
    {
      const BatchExtendSource src{jobs, P.ext[cur], P.job, P.ray_o, P.ray_d, P.hit};
      persistent_traverse<BatchExtendSource, false, kStats, kWt>(src, n_ext, &P.ctl[kCtlFetchExt], stk, steps, st_e, lerr);
    }
    if (!grid_barrier(P.ctl, P.barrier_spins)) break;

    shadow_tests += phase_shade<kParity>(jobs, P, cur, n_ext);
    if (!grid_barrier(P.ctl, P.barrier_spins)) break;

    {
      const uint32_t n_sh = P.ctl[kCtlShadow];
      const BatchShadowSource src{jobs, P.shq, P.job, P.sh_o, P.sh_d, P.sh_c, P.rad};
      persistent_traverse<BatchShadowSource, true, kStats, kWt>(src, n_sh, &P.ctl[kCtlFetchShadow], stk, steps, st_s, lerr);
    }
    if (!grid_barrier(P.ctl, P.barrier_spins)) break;

    phase_finish(jobs, P);
    if (leader) P.ctl[kCtlIter] += 1u;
    if (!grid_barrier(P.ctl, P.barrier_spins)) break;
    cur ^= 1u;
  }

  warp_count(&ctr->shadow_tests, shadow_tests);
  flush_traversal_stats<kStats>(ctr, st_e, st_s);
  if (lerr) atomicOr(err, lerr);
  if (threadIdx.x == 0 && blockIdx.x == 0 && *reinterpret_cast<volatile uint32_t*>(P.ctl + kCtlAbort) != 0u) {
    atomicOr(err, 2u);   // barrier timeout
  }
}

// Adds one job's stagings to its film, sample by sample (the reference's order).
__global__ void __launch_bounds__(256) k_staging_accumulate(const DevJob* jobs, uint32_t jb, DevCounters* ctr) {
  const DevJob& J = jobs[jb];
  const float clampv = J.settings.firefly_clamp;
  for (uint32_t base = blockIdx.x * blockDim.x; base < J.pixels; base += gridDim.x * blockDim.x) {
    const uint32_t px = base + threadIdx.x;
    uint32_t samples = 0u, segs = 0u, dropped = 0u;
    if (px < J.pixels) {
      float4 acc = J.film.sum[px];
      uint32_t cnt = J.film.count[px];
      for (uint32_t sl = 0; sl < J.spp; ++sl) {
        const float4 r = J.staging[static_cast<size_t>(sl) * J.pixels + px];
        if (!(isfinite(r.x) && isfinite(r.y) && isfinite(r.z))) {
          ++dropped;
          continue;
        }
        float cx = r.x, cy = r.y, cz = r.z;
        if (clampv > 0.0f) {
          cx = smin(cx, clampv);
          cy = smin(cy, clampv);
          cz = smin(cz, clampv);
        }
        acc.x = acc.x + cx;
        acc.y = acc.y + cy;
        acc.z = acc.z + cz;
        ++cnt;
        ++samples;
        segs += static_cast<uint32_t>(r.w);
      }
      J.film.sum[px] = acc;
      J.film.count[px] = cnt;
    }
    warp_count(&ctr->samples, samples);
    warp_count(&ctr->rays, segs);
    warp_count(&ctr->dropped, dropped);
  }
}

// Pool reset before a run: every slot free, all queues and counters zero.
__global__ void k_batch_init(BatchPool P) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kBatchCtlWords) P.ctl[i] = (i == static_cast<uint32_t>(kCtlFree)) ? P.capacity : 0u;
  for (uint32_t k = i; k < P.capacity; k += gridDim.x * blockDim.x) P.freel[k] = k;
}

cudaError_t LaunchBatchInit(const BatchPool& pool, cudaStream_t stream) {
  k_batch_init<<<592, 256, 0, stream>>>(pool);
  return cudaGetLastError();
}

namespace {
template <typename K>
cudaError_t set_smem_attr(K kernel, int bytes) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}
}  // namespace

// Kernel variant table: [triangle test][parity][stats][occupancy variant].
namespace {
using BatchFn = void (*)(const DevJob*, uint32_t, unsigned long long, BatchPool, int, int2*, int, int, DevCounters*,
                         uint32_t*);
constexpr int kOccVariants = 4;   // minBlocks 1, 2, 3, 4
template <bool kWt>
BatchFn batch_fn_of(bool parity, bool stats, int o) {
  static const BatchFn table[2][2][kOccVariants] = {
      {{k_batch<false, false, 1, kWt>, k_batch<false, false, 2, kWt>, k_batch<false, false, 3, kWt>,
        k_batch<false, false, 4, kWt>},
       {k_batch<false, true, 1, kWt>, k_batch<false, true, 1, kWt>, k_batch<false, true, 1, kWt>,
        k_batch<false, true, 1, kWt>}},
      {{k_batch<true, false, 1, kWt>, k_batch<true, false, 2, kWt>, k_batch<true, false, 3, kWt>,
        k_batch<true, false, 4, kWt>},
       {k_batch<true, true, 1, kWt>, k_batch<true, true, 1, kWt>, k_batch<true, true, 1, kWt>,
        k_batch<true, true, 1, kWt>}}};
  return table[parity ? 1 : 0][stats ? 1 : 0][o];
}
BatchFn batch_fn(bool parity, bool stats, int occ, bool wt) {
  const int o = occ < 0 ? 0 : (occ >= kOccVariants ? kOccVariants - 1 : occ);
  return wt ? batch_fn_of<true>(parity, stats, o) : batch_fn_of<false>(parity, stats, o);
}
}  // namespace

cudaError_t ConfigureBatchSmem(size_t bytes) {
  const int b = static_cast<int>(bytes);
  cudaError_t e = cudaSuccess;
  for (int wt = 0; wt < 2 && e == cudaSuccess; ++wt)
    for (int p = 0; p < 2 && e == cudaSuccess; ++p)
      for (int st = 0; st < 2 && e == cudaSuccess; ++st)
        for (int o = 0; o < kOccVariants && e == cudaSuccess; ++o)
          e = set_smem_attr(batch_fn(p != 0, st != 0, o, wt != 0), b);
  return e;
}

int BatchBlocksPerSm(int block, size_t smem, bool parity, bool stats, int occ, bool watertight) {
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, batch_fn(parity, stats, occ, watertight), block, smem) !=
      cudaSuccess)
    return 0;
  return blocks;
}

cudaError_t LaunchBatchPersistent(const DevJob* d_jobs, uint32_t job_count, unsigned long long total_paths,
                                  const BatchPool& pool, const BatchLaunch& bl, DevCounters* ctr, uint32_t* err) {
  const size_t smem = StackSmemBytes(bl.block, bl.smem_entries);
  const DevJob* jobs = d_jobs;
  uint32_t jc = job_count;
  unsigned long long total = total_paths;
  BatchPool P = pool;
  int scap = bl.smem_entries, tcap = bl.stack_cap, steps = bl.steps;
  int2* spill = bl.spill;
  void* args[] = {&jobs, &jc, &total, &P, &scap, &spill, &tcap, &steps, &ctr, &err};
  const void* fn = reinterpret_cast<const void*>(batch_fn(bl.parity, bl.stats, bl.occupancy, bl.watertight));
  return cudaLaunchCooperativeKernel(fn, dim3(bl.grid), dim3(bl.block), args, smem, bl.stream);
}

cudaError_t LaunchStagingAccumulate(const DevJob* d_jobs, uint32_t job_count, unsigned long long,
                                    cudaStream_t stream, DevCounters* ctr) {
  for (uint32_t j = 0; j < job_count; ++j) {
    k_staging_accumulate<<<296, 256, 0, stream>>>(d_jobs, j, ctr);
  }
  return cudaGetLastError();
}

}  // namespace vkptc

