// context.cu -- the C ABI of libvkpt_cuda (include/vkptc.h).
//
// One vkptc_ctx is one IPathTracer instance (src/pathtracer/PathTracer.h:1069-1184):
// it follows that interface's state machine (Uninitialized -> Configured ->
// SceneLoaded -> Ready; reset is film-only and keeps the acceleration
// structure), returns its StatusCode values, and keeps a last-error string.
// All device memory (scene, wide BVH, film, wave queues) belongs to the context.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/vkptc.h"
#include "adjoint_launch.h"
#include "bvh_build.h"
#include "bvh_host.h"
#include "batch.cuh"
#include "kernels.cuh"
#include "sdf.cuh"

using namespace vkptc;

namespace {

template <typename T>
struct DevBuf {
  T* ptr = nullptr;
  size_t count = 0;
  bool pooled = false;            // from the builder's stream-ordered pool (adopt_pooled)
  cudaStream_t pool_stream = nullptr;
  ~DevBuf() { release(); }
  void release() {
    if (ptr && pooled) {
      // after the queued work of the stream that used it; if that stream is gone, after all work
      if (cudaFreeAsync(ptr, pool_stream) != cudaSuccess) {
        cudaGetLastError();
        cudaDeviceSynchronize();
        cudaFreeAsync(ptr, nullptr);
      }
    } else if (ptr) {
      cudaFree(ptr);
    }
    ptr = nullptr;
    count = 0;
    pooled = false;
  }
  cudaError_t alloc(size_t n) {
    if (n <= count && ptr) return cudaSuccess;
    release();
    if (n == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&ptr), n * sizeof(T));
    if (e == cudaSuccess) count = n;
    else ptr = nullptr;
    return e;
  }
  size_t bytes() const { return count * sizeof(T); }
  void adopt(T* p, size_t n) {
    release();
    ptr = p;
    count = p ? n : 0;
  }
  void adopt_pooled(T* p, size_t n, cudaStream_t s) {
    adopt(p, n);
    pooled = p != nullptr;
    pool_stream = s;
  }
};

struct HostCamera {
  float pos[3], target[3], up[3];
  float fov, aperture, focus;
  uint32_t iris_blades = 0u;                // lens shape (RTCameraState defaults)
  float iris_rotation = 0.0f, iris_roundness = 1.0f, squeeze = 1.0f;
};

// Differentiable-rendering state of a context (vkptc_forward / vkptc_backward).
struct AdjointState {
  bool setup = false, forward_done = false, has_target = false;
  vkptc_adjoint_desc desc{};
  uint32_t width = 0, height = 0;
  std::vector<float> host_mat, host_mat0;   // 16 floats per material: params / roulette params applied
  DevBuf<float> mat, mat0;                 // device copies of the two tables
  DevBuf<float4> rad;                      // per-sample radiance of the last forward
  DevBuf<float4> adj;                      // per-pixel adjoint of a sample's radiance
  DevBuf<float> target, image;
  DevBuf<double> loss_part, loss;
  DevBuf<float> grad_part, grad;
  DevBuf<float4> recs, gout;               // backward: vertex records and radiance adjoints of a chunk
  DevBuf<uint32_t> fwd_nrec;               // records per path of a forward that recorded its paths
  bool recorded = false;                   // recs hold every path of the last forward (no replay needed)
  DevBuf<float> path_weight;
  int loss_grid = 0;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  vkptc_adjoint_stats stats{};
  ~AdjointState() {
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
  }
};

// Scratch of vkptc_render_tile_noalloc, one file-scope device array per GPU
// that loads the library, held until the process exits.  Path-state bytes per
// path: rng (8) + seven float4 arrays (ray_o, ray_d, thr, rad, sh_o, sh_d,
// sh_c: 112) + hit float2 (8) + three u32 queues (12); every array starts on
// a 256-byte boundary.
constexpr size_t kNoAllocPathBytes = 8 + 7 * 16 + 8 + 3 * 4;
constexpr size_t kNoAllocArrays = 12;
constexpr size_t kNoAllocBytes = VKPTC_NOALLOC_MAX_PATHS * kNoAllocPathBytes + (kNoAllocArrays + 1) * 256;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Live contexts per device (a batch's jobs are contexts too): when the last
// one goes, the device build pool's kept memory is returned to the driver.
std::atomic<int> g_live_contexts[64];

// Makes `device` current for the scope and restores the caller's device after.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int device) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    cudaSetDevice(device);
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
  DeviceGuard(const DeviceGuard&) = delete;
  DeviceGuard& operator=(const DeviceGuard&) = delete;
};

}  // namespace

struct vkptc_ctx {
  vkptc_config config{};
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;      // stream all work is enqueued on
  cudaStream_t own_stream = nullptr;  // the context's own stream
  // Two events made with the context: they order kernels a call enqueues on a
  // caller's stream against the work queued on `stream` (no allocation per call).
  cudaEvent_t order_ev[2] = {nullptr, nullptr};
  // Device address of g_noalloc_scratch on this context's device, looked up
  // once when the context is created (its device current then).
  unsigned char* noalloc_scratch = nullptr;
  cudaError_t noalloc_lookup = cudaSuccess;
  std::string last_error;
  // per-stage timing
  StageTimer timer;
  std::vector<cudaEvent_t> timer_events;
  double stage_ms[StageTimer::kStages] = {0, 0, 0, 0, 0};
  uint64_t stage_launches[StageTimer::kStages] = {0, 0, 0, 0, 0};
  bool configured = false, has_scene = false, accel_valid = false;
  uint32_t current_sample = 0;
  uint64_t last_sample_us = 0, accumulation_gen = 0;
  vkptc_render_settings settings{};

  // scene (host copies needed to rebuild)
  SceneGeometry geo;                      // flattened on the host (host build, external BVHs)
  bool geo_ready = false;
  DevBuf<float> d_raw_vertices;           // the scene's arrays, for the device build
  DevBuf<uint32_t> d_raw_indices;
  uint32_t raw_vertex_count = 0, raw_index_count = 0;
  std::vector<uint32_t> raw_instances;
  DevBuf<float> d_raw_local_vertices;     // dynamic instances (empty without)
  DevBuf<uint32_t> d_raw_local_indices;
  uint32_t raw_local_vertex_count = 0, raw_local_index_count = 0;
  std::vector<uint32_t> raw_instance_local;
  std::vector<float> raw_instance_transforms;
  std::vector<uint32_t> raw_local_indices_host;   // for checking transform updates
  DeviceRefitState* refit = nullptr;      // device build of a scene with dynamic local geometry
  BinNode* d_ref_nodes = nullptr;         // its reference tree, kept for refits
  uint32_t* d_ref_order = nullptr;
  uint32_t ref_count = 0;
  uint32_t prim_count = 0;                // flattened primitives of the built accelerator
  uint32_t instance_count = 0;            // the loaded scene's instances
  std::vector<uint32_t> instance_material;   // per instance: its material index (scene deltas)
  std::vector<uint32_t> inst_prims;       // built accelerator: first primitive per instance, then the total
  DevBuf<uint4> d_delta_ranges;           // scene deltas: instance ranges whose material changes
  std::vector<float> materials, lights;
  float env[3] = {0, 0, 0};
  uint32_t env_w = 0, env_h = 0;          // environment map size (0: constant environment)
  float env_scale[3] = {1, 1, 1};
  DevBuf<float4> d_env;
  uint32_t sdf_count = 0;                 // SDF primitives (records of kSdfWords float4)
  DevBuf<float4> d_sdf;
  HostCamera cam{};
  bool has_transmissive = false;
  bool has_effects = false;
  bool has_exotic = false;      // a transmissive, clear-coat, sheen or toon material (shading variants)

  // device scene
  DevBuf<float4> d_nodes, d_tris, d_shade, d_tie;
  DevBuf<float> d_materials, d_lights;
  WideBvh wide;
  vkptc_accel_info accel{};

  DevBuf<float> d_pack;                   // film sums packed to rgb for host readback
  // split LDR readback (request / poll)
  DevBuf<uint8_t> d_ldr;
  uint8_t* h_ldr = nullptr;               // pinned, 4 bytes per pixel
  size_t h_ldr_bytes = 0;
  cudaEvent_t ldr_event = nullptr;
  uint64_t ldr_token = 0, ldr_next_token = 1;
  uint32_t ldr_width = 0, ldr_height = 0;

  // film
  DevBuf<float4> d_film_sum;
  DevBuf<uint32_t> d_film_count;
  DevBuf<float> d_film_invalid;

  // wave state
  DevBuf<uint64_t> w_rng;
  DevBuf<float4> w_ray_o, w_ray_d, w_thr, w_rad, w_sh_o, w_sh_d, w_sh_c;
  DevBuf<float2> w_hit;
  DevBuf<uint32_t> w_q0, w_q1, w_sh_path, w_counts;
  uint32_t wave_capacity = 0;
  size_t smem_configured = 48 * 1024;

  // counters, error word, fetch counter of the ray-query kernel, stack spill
  DevBuf<DevCounters> d_ctr;
  DevBuf<uint32_t> d_err;
  DevBuf<uint32_t> d_fetch;
  DevBuf<int2> d_spill;

  // ray-query scratch for host-buffer calls
  DevBuf<float> q_rays, q_tmax, q_t;
  DevBuf<uint32_t> q_prim;

  AdjointState adj;
};

namespace {

int32_t fail(vkptc_ctx* ctx, int32_t code, const std::string& msg) {
  if (ctx) ctx->last_error = msg;
  return code;
}

int32_t cuda_fail(vkptc_ctx* ctx, cudaError_t e, const char* what) {
  const int32_t code = (e == cudaErrorMemoryAllocation) ? VKPTC_ALLOC_FAILED : VKPTC_INTERNAL_ERROR;
  return fail(ctx, code, std::string(what) + ": " + cudaGetErrorString(e));
}

#define VKPTC_CUDA(ctx, call, what)            \
  do {                                         \
    cudaError_t e_ = (call);                   \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, what); \
  } while (0)

vkptc_lifecycle lifecycle(const vkptc_ctx* c) {
  if (!c->configured) return VKPTC_UNINITIALIZED;
  if (!c->has_scene) return VKPTC_CONFIGURED;
  if (!c->accel_valid) return VKPTC_SCENE_LOADED;
  return VKPTC_READY;
}

// Camera basis and tan(fov/2) computed on the host exactly as the reference
// does (compute_camera_basis, ScalarCpuPathTracer.cpp:139-152; camera_rays,
// ScalarCpuPathTracer.Render.cpp:78) so primary rays are bit-identical.
void camera_basis(const HostCamera& c, V3& fwd, V3& right, V3& up) {
  fwd = unit(sub(mk(c.target[0], c.target[1], c.target[2]), mk(c.pos[0], c.pos[1], c.pos[2])));
  right = unit(cross(fwd, mk(c.up[0], c.up[1], c.up[2])));
  if (dot(right, right) <= kEps * kEps) right = mk(1.0f, 0.0f, 0.0f);
  up = unit(cross(right, fwd));
  if (dot(up, up) <= kEps * kEps) up = mk(0.0f, 1.0f, 0.0f);
}

DevScene dev_scene(const vkptc_ctx* c) {
  DevScene s{};
  s.nodes = c->d_nodes.ptr;
  s.tris = c->d_tris.ptr;
  s.shade = c->d_shade.ptr;
  s.tie = c->d_tie.ptr;
  s.materials = c->d_materials.ptr;
  s.lights = c->d_lights.ptr;
  s.material_count = static_cast<uint32_t>(c->materials.size() / 16);
  s.light_count = static_cast<uint32_t>(c->lights.size() / 16);
  s.prim_count = c->prim_count;
  s.has_transmissive = c->has_transmissive ? 1u : 0u;
  s.has_effects = c->has_effects ? 1u : 0u;
  s.env = mk(c->env[0], c->env[1], c->env[2]);
  s.env_map = c->env_w ? c->d_env.ptr : nullptr;
  s.env_w = c->env_w;
  s.env_h = c->env_h;
  s.env_scale = mk(c->env_scale[0], c->env_scale[1], c->env_scale[2]);
  s.cam_pos = mk(c->cam.pos[0], c->cam.pos[1], c->cam.pos[2]);
  camera_basis(c->cam, s.cam_fwd, s.cam_right, s.cam_up);
  const float radians = c->cam.fov * (kPi / 180.0f);
  s.tan_half_fov = std::tan(0.5f * radians);
  s.aperture = c->cam.aperture > 0.0f ? c->cam.aperture : c->settings.camera_aperture_radius;
  s.focus = c->cam.focus > 0.0f ? c->cam.focus : c->settings.camera_focus_distance;
  // Lens shape: the same float expressions as ScalarCpuPathTracer::camera_rays
  // (src/pathtracer/ScalarCpuPathTracer.Render.cpp:44-49, 95-110), evaluated once.
  const uint32_t blades = std::min(c->cam.iris_blades, 64u);
  const float rd = c->cam.iris_roundness;
  const float roundness = std::isfinite(rd) ? std::min(1.0f, std::max(0.0f, rd)) : 0.0f;
  s.iris_on = (blades >= 3u && roundness < 0.999f) ? 1u : 0u;
  s.iris_sector = s.iris_on ? 2.0f * kPi / static_cast<float>(blades) : 1.0f;
  s.iris_cos_half = std::cos(s.iris_sector * 0.5f);
  s.iris_rot = c->cam.iris_rotation * (kPi / 180.0f);
  s.iris_round = roundness;
  s.iris_one_minus_round = 1.0f - roundness;
  s.squeeze = std::isfinite(c->cam.squeeze) ? std::max(0.01f, c->cam.squeeze) : 1.0f;
  s.stack_required = c->wide.stack_required;
  s.reference_tree = c->wide.reference_topology ? 1u : 0u;
  s.watertight = c->config.triangle_test == VKPTC_TRIANGLE_WATERTIGHT ? 1u : 0u;
  s.sdf = c->sdf_count ? c->d_sdf.ptr : nullptr;
  s.sdf_count = c->sdf_count;
  return s;
}

DevSettings dev_settings(const vkptc_ctx* c, uint32_t frame) {
  DevSettings st{};
  st.width = c->settings.width;
  st.height = c->settings.height;
  st.max_depth = c->settings.max_depth;
  st.enable_nee = c->settings.enable_nee;
  st.enable_mis = c->settings.enable_mis;
  st.rr_start = c->settings.rr_start_depth;
  st.rr_min = c->settings.rr_min_survival;
  st.rr_max = c->settings.rr_max_survival;
  st.seed = c->settings.seed;
  st.firefly_clamp = c->settings.firefly_clamp;
  st.frame = frame;
  return st;
}

int block_size(const vkptc_ctx* c) {
  const uint32_t b = c->config.block_size;
  if (b == 0) return 128;
  return static_cast<int>(std::min<uint32_t>(256u, std::max<uint32_t>(32u, (b + 31u) / 32u * 32u)));
}

int stack_cap(const vkptc_ctx* c) {
  return static_cast<int>(std::max<uint32_t>(1u, c->wide.stack_required));
}

constexpr int kDefaultSmemEntries = 16;
constexpr int kDefaultSteps = 4;

int32_t ensure_stack_smem(vkptc_ctx* c, const LaunchShape& ls);

// The traversal's step word: low 16 bits the steps between refills (0: the
// default), high 16 bits the refill threshold in idle lanes (at most 32).
int steps_word(uint32_t v, int default_steps) {
  const uint32_t low = v & 0xFFFFu, refill = std::min<uint32_t>(32u, v >> 16);
  return static_cast<int>((low ? low : static_cast<uint32_t>(default_steps)) | (refill << 16));
}

// Block size, stack split (shared-memory entries + global spill), steps between
// warp refills, and a grid of (resident blocks per SM) x SMs: the traversal
// kernels are persistent.  allow_spill = false keeps the whole stack in
// shared memory (no spill buffer is needed, none is allocated).
int32_t launch_shape(vkptc_ctx* c, cudaStream_t stream, LaunchShape& ls, bool allow_spill = true) {
  ls.block = block_size(c);
  ls.stack_cap = stack_cap(c);
  const int asked = c->config.stack_depth ? static_cast<int>(c->config.stack_depth) : kDefaultSmemEntries;
  ls.smem_entries = allow_spill ? std::min(ls.stack_cap, std::max(1, asked)) : ls.stack_cap;
  ls.steps = steps_word(c->config.steps, kDefaultSteps);
  ls.stream = stream;
  ls.spill = nullptr;
  const int32_t rc = ensure_stack_smem(c, ls);
  if (rc != VKPTC_OK) return rc;
  const size_t smem = StackSmemBytes(ls.block, ls.smem_entries);
  const int per_sm = ExtendBlocksPerSm(ls.block, smem, c->config.triangle_test == VKPTC_TRIANGLE_WATERTIGHT);
  ls.grid = c->sm_count * per_sm;
  const size_t spill = SpillEntries(ls);
  if (spill > 0) {
    if (c->d_spill.count < spill) VKPTC_CUDA(c, c->d_spill.alloc(spill), "stack spill alloc");
    ls.spill = c->d_spill.ptr;
  }
  return VKPTC_OK;
}

int32_t ensure_stack_smem(vkptc_ctx* c, const LaunchShape& ls) {
  const size_t smem = StackSmemBytes(ls.block, ls.smem_entries);
  // The transmissive shadow kernel keeps its whole stack in shared memory.
  const size_t smem_full = c->has_transmissive ? StackSmemBytes(ls.block, ls.stack_cap) : smem;
  const size_t need = std::max(smem, smem_full);
  int max_optin = 0;
  cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
  if (need > static_cast<size_t>(max_optin)) {
    return fail(c, VKPTC_UNSUPPORTED, "traversal stack does not fit in shared memory (BVH too deep for this block size)");
  }
  if (need > c->smem_configured) {
    VKPTC_CUDA(c, ConfigureStackSmem(need), "shared memory limit");
    c->smem_configured = need;
  }
  return VKPTC_OK;
}

int32_t ensure_wave(vkptc_ctx* c, uint32_t paths) {
  if (paths <= c->wave_capacity) return VKPTC_OK;
  const size_t n = paths;
  VKPTC_CUDA(c, c->w_rng.alloc(n), "wave alloc");
  VKPTC_CUDA(c, c->w_ray_o.alloc(n), "wave alloc");
  VKPTC_CUDA(c, c->w_ray_d.alloc(n), "wave alloc");
  VKPTC_CUDA(c, c->w_thr.alloc(n), "wave alloc");
  VKPTC_CUDA(c, c->w_rad.alloc(n), "wave alloc");
  VKPTC_CUDA(c, c->w_hit.alloc(n), "wave alloc");
  VKPTC_CUDA(c, c->w_q0.alloc(n), "wave alloc");
  VKPTC_CUDA(c, c->w_q1.alloc(n), "wave alloc");
  VKPTC_CUDA(c, c->w_sh_path.alloc(n), "wave alloc");
  VKPTC_CUDA(c, c->w_sh_o.alloc(n), "wave alloc");
  VKPTC_CUDA(c, c->w_sh_d.alloc(n), "wave alloc");
  VKPTC_CUDA(c, c->w_sh_c.alloc(n), "wave alloc");
  VKPTC_CUDA(c, c->w_counts.alloc(8), "wave alloc");
  c->wave_capacity = paths;
  return VKPTC_OK;
}

WaveState wave_state(vkptc_ctx* c) {
  WaveState w{};
  w.rng = c->w_rng.ptr;
  w.ray_o = c->w_ray_o.ptr;
  w.ray_d = c->w_ray_d.ptr;
  w.thr = c->w_thr.ptr;
  w.rad = c->w_rad.ptr;
  w.hit = c->w_hit.ptr;
  w.sh_path = c->w_sh_path.ptr;
  w.sh_o = c->w_sh_o.ptr;
  w.sh_d = c->w_sh_d.ptr;
  w.sh_c = c->w_sh_c.ptr;
  w.q[0] = c->w_q0.ptr;
  w.q[1] = c->w_q1.ptr;
  w.counts = c->w_counts.ptr;
  w.capacity = c->wave_capacity;
  return w;
}

Film film_of(vkptc_ctx* c) {
  Film f{};
  f.sum = c->d_film_sum.ptr;
  f.count = c->d_film_count.ptr;
  f.invalid = c->d_film_invalid.ptr;
  f.width = c->settings.width;
  f.height = c->settings.height;
  return f;
}

// Orders the kernels a call enqueues on a caller's stream `st` against the
// context's stream: before the launch `st` waits for the work already queued
// on the context's stream (a rebuild, scene reload or upload the kernels must
// not overtake), and after it the context's stream waits for the launch, so
// later work there (which may free or rewrite the arrays these kernels read)
// cannot overtake them.  Nothing is inserted when `st` is the context's
// stream, or while either stream is being captured: an event recorded in a
// capture and waited on by a stream outside it would pull that stream into
// the capture.  *active tells order_end whether to close the pair.
int32_t order_begin(vkptc_ctx* c, cudaStream_t st, bool* active) {
  *active = false;
  if (st == c->stream) return VKPTC_OK;
  cudaStreamCaptureStatus a = cudaStreamCaptureStatusNone, b = cudaStreamCaptureStatusNone;
  VKPTC_CUDA(c, cudaStreamIsCapturing(st, &a), "stream capture status");
  VKPTC_CUDA(c, cudaStreamIsCapturing(c->stream, &b), "stream capture status");
  if (a != cudaStreamCaptureStatusNone || b != cudaStreamCaptureStatusNone) return VKPTC_OK;
  VKPTC_CUDA(c, cudaEventRecord(c->order_ev[0], c->stream), "stream ordering");
  VKPTC_CUDA(c, cudaStreamWaitEvent(st, c->order_ev[0], 0), "stream ordering");
  *active = true;
  return VKPTC_OK;
}

// Calls that rewrite or free device arrays the kernels read (scene and BVH
// uploads, rebuilds, film writes) first wait for the work queued on the
// context's stream: their synchronous copies run on the legacy stream, which
// does not wait for the context's non-blocking stream.
cudaError_t drain(vkptc_ctx* c) { return cudaStreamSynchronize(c->stream); }

int32_t order_end(vkptc_ctx* c, cudaStream_t st, bool active) {
  if (!active) return VKPTC_OK;
  VKPTC_CUDA(c, cudaEventRecord(c->order_ev[1], st), "stream ordering");
  VKPTC_CUDA(c, cudaStreamWaitEvent(c->stream, c->order_ev[1], 0), "stream ordering");
  return VKPTC_OK;
}

int32_t check_device_error(vkptc_ctx* c) {
  uint32_t err = 0;
  VKPTC_CUDA(c, cudaMemcpyAsync(&err, c->d_err.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream), "error word");
  VKPTC_CUDA(c, cudaStreamSynchronize(c->stream), "synchronize");
  if (err != 0u) return fail(c, VKPTC_INTERNAL_ERROR, "device traversal stack overflow");
  return VKPTC_OK;
}

// Flags the kernels take from the material table: a transmissive material
// (model 5 or transmission above 0.05) and a procedural effect.
void scan_materials(vkptc_ctx* c) {
  c->has_transmissive = false;
  c->has_effects = false;
  c->has_exotic = false;
  for (size_t i = 0; i < c->materials.size() / 16; ++i) {
    const float* m = &c->materials[16 * i];
    if (static_cast<uint32_t>(m[7] + 0.5f) == 5u || m[10] > 0.05f) c->has_transmissive = true;
    if ((static_cast<uint32_t>(m[15] + 0.5f) & 1023u) != 0u) c->has_effects = true;
    // The shading stage's tests (models 5..8, transmission, clear coat); a model
    // word outside the plain range counts as exotic so no branch is dropped.
    const float mw = m[7];
    const bool plain_model = mw >= 0.0f && mw < 4.5f;
    if (!plain_model || m[10] > 0.05f || m[11] > 0.05f) c->has_exotic = true;
  }
}

int32_t upload_accel(vkptc_ctx* c, const std::vector<BinNode>& bin, const std::vector<uint32_t>& prim_indices,
                     double build_ms) {
  // The reference tree always supplies tie order and the parallel-axis rule;
  // the traversal tree is either that same tree or a binned-SAH tree.
  if (c->config.bvh_mode == VKPTC_BVH_SAH) {
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<BinNode> sah;
    std::vector<uint32_t> sah_prims;
    BuildSahBvh(c->geo, 4u, sah, sah_prims);
    CollapseToWide(c->geo, sah, sah_prims, bin, prim_indices, c->wide);
    build_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  } else {
    CollapseToWide(c->geo, bin, prim_indices, bin, prim_indices, c->wide);
  }
  const WideBvh& w = c->wide;
  VKPTC_CUDA(c, c->d_nodes.alloc(std::max<size_t>(1, w.nodes.size() * 8)), "bvh alloc");
  VKPTC_CUDA(c, c->d_tris.alloc(std::max<size_t>(1, w.tris.size() * 3)), "bvh alloc");
  VKPTC_CUDA(c, c->d_tie.alloc(std::max<size_t>(1, w.tie_nodes.size() * 2)), "bvh alloc");
  VKPTC_CUDA(c, c->d_shade.alloc(std::max<size_t>(1, c->geo.prims.size())), "bvh alloc");
  if (!w.nodes.empty()) {
    VKPTC_CUDA(c, cudaMemcpy(c->d_nodes.ptr, w.nodes.data(), w.nodes.size() * sizeof(WideNode), cudaMemcpyHostToDevice), "bvh upload");
    VKPTC_CUDA(c, cudaMemcpy(c->d_tris.ptr, w.tris.data(), w.tris.size() * sizeof(TriRecord), cudaMemcpyHostToDevice), "bvh upload");
    VKPTC_CUDA(c, cudaMemcpy(c->d_tie.ptr, w.tie_nodes.data(), w.tie_nodes.size() * sizeof(TieNode), cudaMemcpyHostToDevice), "bvh upload");
  }
  std::vector<float4> shade(c->geo.prims.size());
  for (size_t i = 0; i < c->geo.prims.size(); ++i) {
    const HostPrim& p = c->geo.prims[i];
    float m;
    std::memcpy(&m, &p.material, 4);
    shade[i] = make_float4(p.n[0], p.n[1], p.n[2], m);
  }
  if (!shade.empty())
    VKPTC_CUDA(c, cudaMemcpy(c->d_shade.ptr, shade.data(), shade.size() * sizeof(float4), cudaMemcpyHostToDevice), "bvh upload");
  c->prim_count = static_cast<uint32_t>(c->geo.prims.size());
  c->inst_prims.assign(c->geo.inst_first.begin(), c->geo.inst_first.end());
  c->inst_prims.push_back(c->prim_count);
  c->accel = vkptc_accel_info{};
  c->accel.primitive_count = static_cast<uint32_t>(c->geo.prims.size());
  c->accel.binary_node_count = w.binary_nodes;
  c->accel.binary_leaf_count = w.binary_leaves;
  c->accel.wide_node_count = static_cast<uint32_t>(w.nodes.size());
  c->accel.wide_depth = w.depth;
  c->accel.stack_required = w.stack_required;
  c->accel.build_ms = build_ms;
  c->accel.device_bytes = w.nodes.size() * sizeof(WideNode) + w.tris.size() * sizeof(TriRecord);
  c->accel_valid = true;
  return VKPTC_OK;
}

int32_t run_wave(vkptc_ctx* c, const WaveTile& tile, uint32_t frame) {
  const uint32_t paths = tile.w * tile.h * tile.sample_count;
  int32_t rc = ensure_wave(c, paths);
  if (rc != VKPTC_OK) return rc;
  LaunchShape ls;
  rc = launch_shape(c, c->stream, ls);
  if (rc != VKPTC_OK) return rc;
  const DevScene s = dev_scene(c);
  const DevSettings st = dev_settings(c, frame);
  StageTimer* timer = c->config.stage_timing ? &c->timer : nullptr;
  VKPTC_CUDA(c, LaunchWave(s, st, wave_state(c), tile, film_of(c), c->config.math_mode == 0u,
                           c->config.collect_stats != 0u, ls, c->d_ctr.ptr, c->d_err.ptr, timer),
             "wave launch");
  if (timer) {
    // Fold this wave's event pairs into the per-stage totals.
    VKPTC_CUDA(c, cudaStreamSynchronize(c->stream), "timer sync");
    for (int k = 0; k < timer->used; ++k) {
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, timer->events[2 * k], timer->events[2 * k + 1]);
      c->stage_ms[timer->stage_of[k]] += ms;
      c->stage_launches[timer->stage_of[k]] += 1;
    }
    timer->used = 0;
  }
  return VKPTC_OK;
}

constexpr uint32_t kDefaultWavePaths = 1u << 22;

uint32_t wave_paths(const vkptc_ctx* c) {
  return c->config.wave_paths ? c->config.wave_paths : kDefaultWavePaths;
}

}  // namespace

extern "C" {

uint32_t vkptc_abi_version(void) { return VKPTC_ABI_VERSION; }

int32_t vkptc_create(const vkptc_config* config, vkptc_ctx** out_ctx) {
  if (!out_ctx) return VKPTC_INVALID_ARGUMENT;
  *out_ctx = nullptr;
  auto* c = new (std::nothrow) vkptc_ctx();
  if (!c) return VKPTC_ALLOC_FAILED;
  if (config) c->config = *config;
  if (c->config.triangle_test > VKPTC_TRIANGLE_WATERTIGHT) {
    delete c;
    return VKPTC_INVALID_ARGUMENT;
  }
  c->device = c->config.device;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    delete c;
    return VKPTC_UNSUPPORTED;
  }
  if (c->device < 0 || c->device >= count) {
    delete c;
    return VKPTC_INVALID_ARGUMENT;
  }
  if (cudaSetDevice(c->device) != cudaSuccess || cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return VKPTC_INTERNAL_ERROR;
  }
  c->stream = c->own_stream;
  if (c->config.stage_timing) {
    c->timer_events.resize(2 * 4096);
    for (auto& e : c->timer_events) cudaEventCreate(&e);
    c->timer.events = c->timer_events.data();
    c->timer.capacity = 4096;
  }
  cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, c->device);
  if (c->d_ctr.alloc(1) != cudaSuccess || c->d_err.alloc(1) != cudaSuccess || c->d_fetch.alloc(1) != cudaSuccess ||
      cudaMemset(c->d_ctr.ptr, 0, sizeof(DevCounters)) != cudaSuccess ||
      cudaMemset(c->d_err.ptr, 0, sizeof(uint32_t)) != cudaSuccess) {
    cudaStreamDestroy(c->stream);
    delete c;
    return VKPTC_ALLOC_FAILED;
  }
  for (auto& ev : c->order_ev) {
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
      for (auto& e2 : c->order_ev)
        if (e2) cudaEventDestroy(e2);
      cudaStreamDestroy(c->stream);
      delete c;
      return VKPTC_INTERNAL_ERROR;
    }
  }
  // The allocation-free entry point's scratch: host code cannot use the
  // array's name as a device address, so its address on this device is looked
  // up here, with the device current.  A failure is reported by that entry
  // point; nothing else depends on it.
  void* scratch = nullptr;
  c->noalloc_lookup = cudaGetSymbolAddress(&scratch, g_noalloc_scratch);
  if (c->noalloc_lookup == cudaSuccess) c->noalloc_scratch = static_cast<unsigned char*>(scratch);
  else cudaGetLastError();
  if (c->device < 64) g_live_contexts[c->device].fetch_add(1);
  *out_ctx = c;
  return VKPTC_OK;
}

void release_refit(vkptc_ctx* c);

int32_t vkptc_destroy(vkptc_ctx* ctx) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  cudaStream_t s = ctx->own_stream;
  for (auto& e : ctx->timer_events) cudaEventDestroy(e);
  for (auto& e : ctx->order_ev)
    if (e) cudaEventDestroy(e);
  if (ctx->ldr_event) cudaEventDestroy(ctx->ldr_event);
  if (ctx->h_ldr) cudaFreeHost(ctx->h_ldr);
  release_refit(ctx);
  const int device = ctx->device;
  delete ctx;
  if (s) cudaStreamDestroy(s);
  if (device < 64 && g_live_contexts[device].fetch_sub(1) == 1) TrimBuildPool();
  return VKPTC_OK;
}

int32_t vkptc_configure(vkptc_ctx* ctx, const vkptc_render_settings* settings) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  if (!settings) return fail(ctx, VKPTC_INVALID_ARGUMENT, "settings is null");
  if (settings->max_depth > 1024u) return fail(ctx, VKPTC_INVALID_ARGUMENT, "max_depth above 1024");
  const uint64_t px = static_cast<uint64_t>(settings->width) * settings->height;
  if (px > (1ull << 28)) return fail(ctx, VKPTC_INVALID_ARGUMENT, "film larger than 2^28 pixels");
  cudaSetDevice(ctx->device);
  VKPTC_CUDA(ctx, drain(ctx), "waiting for the work queued on the context's stream");
  ctx->settings = *settings;
  VKPTC_CUDA(ctx, ctx->d_film_sum.alloc(std::max<uint64_t>(1, px)), "film alloc");
  VKPTC_CUDA(ctx, ctx->d_film_count.alloc(std::max<uint64_t>(1, px)), "film alloc");
  VKPTC_CUDA(ctx, ctx->d_film_invalid.alloc(std::max<uint64_t>(1, px)), "film alloc");
  VKPTC_CUDA(ctx, cudaMemsetAsync(ctx->d_film_sum.ptr, 0, ctx->d_film_sum.bytes(), ctx->stream), "film clear");
  VKPTC_CUDA(ctx, cudaMemsetAsync(ctx->d_film_count.ptr, 0, ctx->d_film_count.bytes(), ctx->stream), "film clear");
  VKPTC_CUDA(ctx, cudaMemsetAsync(ctx->d_film_invalid.ptr, 0, ctx->d_film_invalid.bytes(), ctx->stream), "film clear");
  VKPTC_CUDA(ctx, cudaMemsetAsync(ctx->d_ctr.ptr, 0, sizeof(DevCounters), ctx->stream), "counter clear");
  ctx->configured = true;
  ctx->has_scene = false;
  ctx->accel_valid = false;
  ctx->adj.setup = false;
  ctx->current_sample = 0;
  ctx->accumulation_gen = 0;
  ctx->last_error.clear();
  return VKPTC_OK;
}

int32_t vkptc_load_scene(vkptc_ctx* ctx, const vkptc_scene_view* scene) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  if (!ctx->configured) return fail(ctx, VKPTC_NOT_READY, "load_scene_snapshot called before configure");
  if (!scene) return fail(ctx, VKPTC_INVALID_ARGUMENT, "scene is null");
  if ((scene->vertex_count && !scene->vertices) || (scene->index_count && !scene->indices) ||
      (scene->material_count && !scene->materials) || (scene->light_count && !scene->lights)) {
    return fail(ctx, VKPTC_INVALID_ARGUMENT, "scene array pointer is null");
  }
  ctx->adj.setup = false;
  cudaSetDevice(ctx->device);
  VKPTC_CUDA(ctx, drain(ctx), "waiting for the work queued on the context's stream");
  if (scene->instance_count > 0 && scene->instances == nullptr)
    return fail(ctx, VKPTC_INVALID_ARGUMENT, "instances pointer is null");
  {
    uint64_t tris = 0;   // the instances' triangle ranges bound the flattened primitives
    for (uint32_t i = 0; i < scene->instance_count; ++i) tris += scene->instances[3 * i + 1];
    if (tris > kMaxTriangles)
      return fail(ctx, VKPTC_INVALID_ARGUMENT, "more than 2^28 - 8 triangles (the wide BVH's leaf references)");
  }
  const bool dyn = scene->instance_local != nullptr && scene->instance_transforms != nullptr;
  if ((scene->instance_local != nullptr) != (scene->instance_transforms != nullptr) ||
      (dyn && ((scene->local_vertex_count && !scene->local_vertices) || (scene->local_index_count && !scene->local_indices))))
    return fail(ctx, VKPTC_INVALID_ARGUMENT, "dynamic-instance array pointer is null");
  InstanceGeometry ig;
  if (dyn) {
    ig.instance_local = scene->instance_local;
    ig.instance_transforms = scene->instance_transforms;
    ig.local_vertices = scene->local_vertices;
    ig.local_vertex_count = scene->local_vertex_count;
    ig.local_indices = scene->local_indices;
    ig.local_index_count = scene->local_index_count;
  }
  if (ctx->config.build_mode == VKPTC_BUILD_HOST) {
    std::string err;
    SceneGeometry geo;
    if (!FlattenScene(scene->vertices, scene->vertex_count, scene->indices, scene->index_count, scene->instances,
                      scene->instance_count, geo, err, dyn ? &ig : nullptr)) {
      return fail(ctx, VKPTC_INVALID_ARGUMENT, err);
    }
    ctx->geo = std::move(geo);
    ctx->geo_ready = true;
    ctx->d_raw_vertices.release();
    ctx->d_raw_indices.release();
    ctx->raw_instances.clear();
  } else {
    // Flattened on the device by the build (or on the host for an external BVH).
    ctx->raw_vertex_count = scene->vertex_count;
    ctx->raw_index_count = scene->index_count;
    VKPTC_CUDA(ctx, ctx->d_raw_vertices.alloc(std::max<size_t>(1, 3ull * scene->vertex_count)), "scene alloc");
    VKPTC_CUDA(ctx, ctx->d_raw_indices.alloc(std::max<size_t>(1, scene->index_count)), "scene alloc");
    if (scene->vertex_count)
      VKPTC_CUDA(ctx, cudaMemcpy(ctx->d_raw_vertices.ptr, scene->vertices, 12ull * scene->vertex_count,
                                 cudaMemcpyHostToDevice), "scene upload");
    if (scene->index_count)
      VKPTC_CUDA(ctx, cudaMemcpy(ctx->d_raw_indices.ptr, scene->indices, 4ull * scene->index_count,
                                 cudaMemcpyHostToDevice), "scene upload");
    ctx->raw_instances.assign(scene->instances, scene->instances + 3 * static_cast<size_t>(scene->instance_count));
    ctx->raw_instance_local.clear();
    ctx->raw_instance_transforms.clear();
    ctx->raw_local_indices_host.clear();
    ctx->raw_local_vertex_count = ctx->raw_local_index_count = 0u;
    ctx->d_raw_local_vertices.release();
    ctx->d_raw_local_indices.release();
    if (dyn) {
      ctx->raw_instance_local.assign(scene->instance_local, scene->instance_local + 5 * static_cast<size_t>(scene->instance_count));
      ctx->raw_instance_transforms.assign(scene->instance_transforms,
                                          scene->instance_transforms + 10 * static_cast<size_t>(scene->instance_count));
      ctx->raw_local_vertex_count = scene->local_vertex_count;
      ctx->raw_local_index_count = scene->local_index_count;
      VKPTC_CUDA(ctx, ctx->d_raw_local_vertices.alloc(std::max<size_t>(1, 3ull * scene->local_vertex_count)), "scene alloc");
      VKPTC_CUDA(ctx, ctx->d_raw_local_indices.alloc(std::max<size_t>(1, scene->local_index_count)), "scene alloc");
      if (scene->local_vertex_count)
        VKPTC_CUDA(ctx, cudaMemcpy(ctx->d_raw_local_vertices.ptr, scene->local_vertices, 12ull * scene->local_vertex_count,
                                   cudaMemcpyHostToDevice), "scene upload");
      if (scene->local_index_count)
        VKPTC_CUDA(ctx, cudaMemcpy(ctx->d_raw_local_indices.ptr, scene->local_indices, 4ull * scene->local_index_count,
                                   cudaMemcpyHostToDevice), "scene upload");
      ctx->raw_local_indices_host.assign(scene->local_indices, scene->local_indices + scene->local_index_count);
    }
    ctx->geo = SceneGeometry{};
    ctx->geo_ready = false;
  }
  ctx->materials.assign(scene->materials, scene->materials + 16 * static_cast<size_t>(scene->material_count));
  if (ctx->materials.empty()) {
    // The reference substitutes one default RTMaterial (ScalarCpuPathTracer.cpp:468-470).
    const float def[16] = {1, 1, 1, 0, 0, 0, 1, 0, 0, 1.5f, 0, 0, 0, 0, 1, 0};
    ctx->materials.assign(def, def + 16);
  }
  ctx->lights.assign(scene->lights, scene->lights + 16 * static_cast<size_t>(scene->light_count));
  for (size_t i = 0; i < ctx->lights.size() / 16; ++i) ctx->lights[16 * i + 7] = std::max(0.0f, ctx->lights[16 * i + 7]);
  scan_materials(ctx);
  ctx->instance_count = scene->instance_count;
  ctx->instance_material.resize(scene->instance_count);
  for (uint32_t i = 0; i < scene->instance_count; ++i) ctx->instance_material[i] = scene->instances[3 * i + 2];
  ctx->inst_prims.clear();
  std::memcpy(ctx->env, scene->environment, sizeof(ctx->env));
  // Environment map: used when it holds width*height texels (as the reference checks).
  const uint64_t env_texels = static_cast<uint64_t>(scene->environment_map_width) * scene->environment_map_height;
  ctx->env_w = ctx->env_h = 0u;
  if (scene->environment_map && env_texels > 0) {
    if (env_texels > (1ull << 28)) return fail(ctx, VKPTC_INVALID_ARGUMENT, "environment map above 2^28 texels");
    std::vector<float4> texels(env_texels);
    for (uint64_t i = 0; i < env_texels; ++i) {
      const float* t = scene->environment_map + 3 * i;
      texels[i] = make_float4(t[0], t[1], t[2], 0.0f);
    }
    VKPTC_CUDA(ctx, ctx->d_env.alloc(env_texels), "environment alloc");
    VKPTC_CUDA(ctx, cudaMemcpy(ctx->d_env.ptr, texels.data(), env_texels * sizeof(float4), cudaMemcpyHostToDevice),
               "environment upload");
    ctx->env_w = scene->environment_map_width;
    ctx->env_h = scene->environment_map_height;
    const float* sc = scene->environment_map_scale;
    const bool unit_scale = std::max({sc[0], sc[1], sc[2]}) <= 1.0e-6f;
    for (int a = 0; a < 3; ++a) ctx->env_scale[a] = unit_scale ? 1.0f : sc[a];
  }
  // SDF primitives: one record of kSdfWords float4 each (sdf.cuh), with the
  // sines and cosines of the rotation angles taken once here, by the same
  // float sin/cos calls the reference makes per evaluation.
  ctx->sdf_count = 0u;
  if (scene->sdf_count) {
    if (!scene->sdf_primitives) return fail(ctx, VKPTC_INVALID_ARGUMENT, "scene array pointer is null");
    std::vector<float4> rec;
    for (uint32_t i = 0; i < scene->sdf_count; ++i) {
      const float* q = scene->sdf_primitives + 16 * static_cast<size_t>(i);
      if (!(q[0] >= 0.0f && q[0] < 5.5f)) continue;   // Unknown shape: never hits
      const uint32_t shape = static_cast<uint32_t>(q[0] + 0.5f);
      const float mat = q[10] >= 0.0f ? q[10] : 0.0f;
      const uint32_t material = mat < 4294967040.0f ? static_cast<uint32_t>(mat + 0.5f) : 0xFFFFFFFFu;
      const float rx = q[7], ry = q[8], rz = q[9];
      auto div = [](float v) { return v != 0.0f ? v : 1.0f; };
      auto bits = [](uint32_t v) {
        float f;
        std::memcpy(&f, &v, 4);
        return f;
      };
      rec.push_back(make_float4(q[1], q[2], q[3], bits(shape)));
      rec.push_back(make_float4(q[4], q[5], q[6], bits(material)));
      rec.push_back(make_float4(div(q[4]), div(q[5]), div(q[6]), q[11]));
      const bool unit_scale = div(q[4]) == 1.0f && div(q[5]) == 1.0f && div(q[6]) == 1.0f;
      const bool no_rotation = rx == 0.0f && ry == 0.0f && rz == 0.0f;
      rec.push_back(make_float4(q[12], q[13], bits((unit_scale ? 1u : 0u) | (no_rotation ? 2u : 0u)), 0.0f));
      rec.push_back(make_float4(std::sin(-rx), std::cos(-rx), std::sin(-ry), std::cos(-ry)));
      rec.push_back(make_float4(std::sin(-rz), std::cos(-rz), std::sin(rz), std::cos(rz)));
      rec.push_back(make_float4(std::sin(ry), std::cos(ry), std::sin(rx), std::cos(rx)));
      // Cull sphere of a marched shape: a bound on |local point| over the set
      // {distance <= 1e-4}, times the largest divisor (local = R^-1 (w - pos) / div).
      const double e = 1e-4, pa = q[12], rad = q[11];
      const double sx = std::fabs(q[4]), sy = std::fabs(q[5]), sz = std::fabs(q[6]);
      double rl = 0.0;   // 0: never culled
      if (shape == kSdfBox) rl = std::sqrt((sx + e) * (sx + e) + (sy + e) * (sy + e) + (sz + e) * (sz + e));
      if (shape == kSdfRoundedBox) {
        const double a = std::fabs(pa) + e;
        rl = std::sqrt((sx + a) * (sx + a) + (sy + a) * (sy + a) + (sz + a) * (sz + a));
      }
      if (shape == kSdfTorus) {
        const double ring = std::max(0.05, pa), tube = std::max(0.02, rad);
        rl = std::sqrt((ring + tube + e) * (ring + tube + e) + (tube + e) * (tube + e));
      }
      if (shape == kSdfCapsule) rl = std::fabs(pa) + std::max(0.0, rad + e);
      const double dmax = std::max({std::fabs(div(q[4])), std::fabs(div(q[5])), std::fabs(div(q[6]))});
      const double dmin = std::min({std::fabs(div(q[4])), std::fabs(div(q[5])), std::fabs(div(q[6]))});
      double cull_r = rl * dmax * (1.0 + 1e-5), cull_k = dmax / dmin;
      bool finite = std::isfinite(cull_r) && std::isfinite(cull_k) && cull_r < 1e30;
      for (int w = 1; w <= 13; ++w) finite = finite && std::isfinite(q[w]);
      if (!finite || rl == 0.0) cull_r = cull_k = 0.0;
      rec.push_back(make_float4(static_cast<float>(cull_r), static_cast<float>(cull_k), 0.0f, 0.0f));
    }
    if (!rec.empty()) {
      VKPTC_CUDA(ctx, ctx->d_sdf.alloc(rec.size()), "sdf alloc");
      VKPTC_CUDA(ctx, cudaMemcpy(ctx->d_sdf.ptr, rec.data(), rec.size() * sizeof(float4), cudaMemcpyHostToDevice),
                 "sdf upload");
      ctx->sdf_count = static_cast<uint32_t>(rec.size() / kSdfWords);
    }
  }
  std::memcpy(ctx->cam.pos, scene->camera_position, 12);
  std::memcpy(ctx->cam.target, scene->camera_target, 12);
  std::memcpy(ctx->cam.up, scene->camera_up, 12);
  ctx->cam.fov = scene->camera_fov_deg;
  ctx->cam.aperture = scene->camera_aperture_radius;
  ctx->cam.focus = scene->camera_focus_distance;
  ctx->cam.iris_blades = scene->camera_lens_set ? scene->camera_iris_blade_count : 0u;
  ctx->cam.iris_rotation = scene->camera_lens_set ? scene->camera_iris_rotation_degrees : 0.0f;
  ctx->cam.iris_roundness = scene->camera_lens_set ? scene->camera_iris_roundness : 1.0f;
  ctx->cam.squeeze = scene->camera_lens_set ? scene->camera_anamorphic_squeeze : 1.0f;
  VKPTC_CUDA(ctx, ctx->d_materials.alloc(ctx->materials.size()), "material alloc");
  VKPTC_CUDA(ctx, cudaMemcpy(ctx->d_materials.ptr, ctx->materials.data(), ctx->materials.size() * sizeof(float),
                             cudaMemcpyHostToDevice), "material upload");
  VKPTC_CUDA(ctx, ctx->d_lights.alloc(std::max<size_t>(16, ctx->lights.size())), "light alloc");
  if (!ctx->lights.empty())
    VKPTC_CUDA(ctx, cudaMemcpy(ctx->d_lights.ptr, ctx->lights.data(), ctx->lights.size() * sizeof(float),
                               cudaMemcpyHostToDevice), "light upload");
  ctx->has_scene = true;
  ctx->accel_valid = false;
  ctx->last_error.clear();
  return VKPTC_OK;
}

// Host flattening of the scene for the host build and external BVHs.
int32_t ensure_geo(vkptc_ctx* c) {
  if (c->geo_ready) return VKPTC_OK;
  std::vector<float> v(3ull * c->raw_vertex_count);
  std::vector<uint32_t> idx(c->raw_index_count);
  if (!v.empty())
    VKPTC_CUDA(c, cudaMemcpy(v.data(), c->d_raw_vertices.ptr, v.size() * 4, cudaMemcpyDeviceToHost), "scene read");
  if (!idx.empty())
    VKPTC_CUDA(c, cudaMemcpy(idx.data(), c->d_raw_indices.ptr, idx.size() * 4, cudaMemcpyDeviceToHost), "scene read");
  std::vector<float> lv(3ull * c->raw_local_vertex_count);
  std::vector<uint32_t> li(c->raw_local_index_count);
  if (!lv.empty())
    VKPTC_CUDA(c, cudaMemcpy(lv.data(), c->d_raw_local_vertices.ptr, lv.size() * 4, cudaMemcpyDeviceToHost), "scene read");
  if (!li.empty())
    VKPTC_CUDA(c, cudaMemcpy(li.data(), c->d_raw_local_indices.ptr, li.size() * 4, cudaMemcpyDeviceToHost), "scene read");
  InstanceGeometry ig;
  const bool dyn = !c->raw_instance_local.empty();
  if (dyn) {
    ig.instance_local = c->raw_instance_local.data();
    ig.instance_transforms = c->raw_instance_transforms.data();
    ig.local_vertices = lv.data();
    ig.local_vertex_count = c->raw_local_vertex_count;
    ig.local_indices = li.data();
    ig.local_index_count = c->raw_local_index_count;
  }
  std::string err;
  SceneGeometry geo;
  if (!FlattenScene(v.data(), c->raw_vertex_count, idx.data(), c->raw_index_count, c->raw_instances.data(),
                    static_cast<uint32_t>(c->raw_instances.size() / 3), geo, err, dyn ? &ig : nullptr)) {
    return fail(c, VKPTC_INVALID_ARGUMENT, err);
  }
  c->geo = std::move(geo);
  c->geo_ready = true;
  return VKPTC_OK;
}

void release_refit(vkptc_ctx* c) {
  FreeRefitState(c->refit, c->stream);
  FreeAccelArray(c->d_ref_nodes, c->stream);
  FreeAccelArray(c->d_ref_order, c->stream);
  c->d_ref_nodes = nullptr;
  c->d_ref_order = nullptr;
  c->ref_count = 0;
}

// Device build: every array the traversal reads, produced by CUDA kernels
// (bvh_build.cu).  Returns VKPTC_OK with *done = false when the scene needs
// the host path (non-finite primitive bounds).
int32_t build_on_device(vkptc_ctx* c, bool* done) {
  *done = false;
  const auto t0 = std::chrono::steady_clock::now();
  DeviceAccelOut out;
  DeviceSceneArrays a;
  a.vertices = c->d_raw_vertices.ptr;
  a.vertex_count = c->raw_vertex_count;
  a.indices = c->d_raw_indices.ptr;
  a.index_count = c->raw_index_count;
  a.instances = c->raw_instances.data();
  a.instance_count = static_cast<uint32_t>(c->raw_instances.size() / 3);
  if (!c->raw_instance_local.empty()) {
    a.local_vertices = c->d_raw_local_vertices.ptr;
    a.local_vertex_count = c->raw_local_vertex_count;
    a.local_indices = c->d_raw_local_indices.ptr;
    a.local_index_count = c->raw_local_index_count;
    a.instance_local = c->raw_instance_local.data();
    a.instance_transforms = c->raw_instance_transforms.data();
  }
  a.watertight = c->config.triangle_test == VKPTC_TRIANGLE_WATERTIGHT;
  const cudaError_t e = BuildAccelOnDevice(a, c->config.bvh_mode == VKPTC_BVH_SAH, c->stream, out);
  if (e != cudaSuccess) {
    FreeDeviceAccel(out, c->stream);
    return cuda_fail(c, e, "device BVH build");
  }
  if (out.fallback) return VKPTC_OK;
  const uint32_t n = out.prim_count;
  c->inst_prims = std::move(out.inst_first);
  c->d_shade.adopt_pooled(out.shade, std::max<uint32_t>(1, n), c->stream);
  if (n == 0u) {
    VKPTC_CUDA(c, c->d_nodes.alloc(1), "bvh alloc");
    VKPTC_CUDA(c, c->d_tris.alloc(1), "bvh alloc");
    VKPTC_CUDA(c, c->d_tie.alloc(1), "bvh alloc");
  } else {
    if (reinterpret_cast<uintptr_t>(out.nodes) % 32u == 0u) {
      c->d_nodes.adopt_pooled(out.nodes, 8ull * out.wide_nodes, c->stream);
    } else {
      // the traversal reads node bounds with 32-byte loads: move the nodes to an aligned allocation
      VKPTC_CUDA(c, c->d_nodes.alloc(8ull * out.wide_nodes), "bvh alloc");
      VKPTC_CUDA(c, cudaMemcpyAsync(c->d_nodes.ptr, out.nodes, 128ull * out.wide_nodes, cudaMemcpyDeviceToDevice,
                                    c->stream), "bvh copy");
      FreeAccelArray(out.nodes, c->stream);
    }
    c->d_tris.adopt_pooled(out.tris, 3ull * n, c->stream);
    c->d_tie.adopt_pooled(out.tie, 2ull * out.binary_nodes, c->stream);
  }
  release_refit(c);
  if (out.refit) {
    c->refit = out.refit;
    c->d_ref_nodes = out.ref_nodes;
    c->d_ref_order = out.ref_order;
    c->ref_count = out.binary_nodes;
    out.refit = nullptr;
  } else {
    FreeAccelArray(out.ref_nodes, c->stream);
    FreeAccelArray(out.ref_order, c->stream);
  }
  c->wide = WideBvh{};
  c->wide.binary_nodes = out.binary_nodes;
  c->wide.binary_leaves = out.binary_leaves;
  c->wide.depth = out.depth;
  c->wide.stack_required = out.stack_required;
  c->wide.reference_topology = out.reference_topology;
  c->prim_count = n;
  c->accel = vkptc_accel_info{};
  c->accel.primitive_count = n;
  c->accel.binary_node_count = out.binary_nodes;
  c->accel.binary_leaf_count = out.binary_leaves;
  c->accel.wide_node_count = out.wide_nodes;
  c->accel.wide_depth = out.depth;
  c->accel.stack_required = out.stack_required;
  c->accel.build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  c->accel.device_bytes = static_cast<uint64_t>(out.wide_nodes) * sizeof(WideNode) + static_cast<uint64_t>(n) * sizeof(TriRecord);
  c->accel_valid = true;
  *done = true;
  return VKPTC_OK;
}

int32_t vkptc_build_acceleration(vkptc_ctx* ctx) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  if (!ctx->has_scene) return fail(ctx, VKPTC_NOT_READY, "build_or_update_acceleration called before load_scene_snapshot");
  cudaSetDevice(ctx->device);
  VKPTC_CUDA(ctx, drain(ctx), "waiting for the work queued on the context's stream");
  const bool watertight = ctx->config.triangle_test == VKPTC_TRIANGLE_WATERTIGHT;
  if (watertight && ctx->config.build_mode == VKPTC_BUILD_HOST)
    return fail(ctx, VKPTC_UNSUPPORTED, "the watertight triangle test needs the device build");
  if (ctx->config.build_mode != VKPTC_BUILD_HOST) {
    bool done = false;
    const int32_t rc = build_on_device(ctx, &done);
    if (rc != VKPTC_OK) return rc;
    if (done) {
      ctx->last_error.clear();
      return VKPTC_OK;
    }
    // non-finite vertices: the host path builds Moller-Trumbore records only
    if (watertight) return fail(ctx, VKPTC_UNSUPPORTED, "the watertight triangle test needs finite vertices");
  }
  release_refit(ctx);
  int32_t grc = ensure_geo(ctx);
  if (grc != VKPTC_OK) return grc;
  const auto t0 = std::chrono::steady_clock::now();
  std::vector<BinNode> bin;
  std::vector<uint32_t> order;
  BuildBinaryBvh(ctx->geo, 4u, bin, order);
  const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  const int32_t rc = upload_accel(ctx, bin, order, ms);
  if (rc == VKPTC_OK) ctx->last_error.clear();
  return rc;
}

int32_t vkptc_load_bvh(vkptc_ctx* ctx, const vkptc_bvh_view* bvh) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  if (!ctx->has_scene) return fail(ctx, VKPTC_NOT_READY, "load_bvh called before load_scene_snapshot");
  if (!bvh || !bvh->nodes || !bvh->prim_indices) return fail(ctx, VKPTC_INVALID_ARGUMENT, "bvh view is null");
  if (ctx->config.triangle_test == VKPTC_TRIANGLE_WATERTIGHT)
    return fail(ctx, VKPTC_UNSUPPORTED, "the watertight triangle test needs the device build");
  cudaSetDevice(ctx->device);
  VKPTC_CUDA(ctx, drain(ctx), "waiting for the work queued on the context's stream");
  std::vector<BinNode> bin(bvh->node_count);
  for (uint32_t i = 0; i < bvh->node_count; ++i) {
    const uint32_t* w = bvh->nodes + 10 * static_cast<size_t>(i);
    std::memcpy(bin[i].lo, w, 12);
    std::memcpy(bin[i].hi, w + 3, 12);
    std::memcpy(&bin[i].left, w + 6, 4);
    std::memcpy(&bin[i].right, w + 7, 4);
    std::memcpy(&bin[i].first, w + 8, 4);
    std::memcpy(&bin[i].count, w + 9, 4);
  }
  std::vector<uint32_t> order(bvh->prim_indices, bvh->prim_indices + bvh->prim_count);
  const int32_t grc = ensure_geo(ctx);
  if (grc != VKPTC_OK) return grc;
  std::string err;
  if (!ValidateBinaryBvh(bin, order, ctx->geo.prims.size(), err)) return fail(ctx, VKPTC_INVALID_ARGUMENT, err);
  const int32_t rc = upload_accel(ctx, bin, order, 0.0);
  if (rc == VKPTC_OK) ctx->last_error.clear();
  return rc;
}

int32_t vkptc_build_binary_bvh(const vkptc_scene_view* scene, uint32_t* nodes_out, uint32_t* node_count,
                               uint32_t* prim_out, uint32_t* prim_count) {
  if (!scene || !nodes_out || !node_count || !prim_out || !prim_count) return VKPTC_INVALID_ARGUMENT;
  SceneGeometry geo;
  std::string err;
  InstanceGeometry ig;
  const bool dyn = scene->instance_local != nullptr && scene->instance_transforms != nullptr;
  if (dyn) {
    ig.instance_local = scene->instance_local;
    ig.instance_transforms = scene->instance_transforms;
    ig.local_vertices = scene->local_vertices;
    ig.local_vertex_count = scene->local_vertex_count;
    ig.local_indices = scene->local_indices;
    ig.local_index_count = scene->local_index_count;
  }
  if (!FlattenScene(scene->vertices, scene->vertex_count, scene->indices, scene->index_count, scene->instances,
                    scene->instance_count, geo, err, dyn ? &ig : nullptr)) {
    return VKPTC_INVALID_ARGUMENT;
  }
  std::vector<BinNode> bin;
  std::vector<uint32_t> order;
  BuildBinaryBvh(geo, 4u, bin, order);
  for (size_t i = 0; i < bin.size(); ++i) {
    uint32_t* w = nodes_out + 10 * i;
    std::memcpy(w, bin[i].lo, 12);
    std::memcpy(w + 3, bin[i].hi, 12);
    std::memcpy(w + 6, &bin[i].left, 4);
    std::memcpy(w + 7, &bin[i].right, 4);
    std::memcpy(w + 8, &bin[i].first, 4);
    std::memcpy(w + 9, &bin[i].count, 4);
  }
  std::copy(order.begin(), order.end(), prim_out);
  *node_count = static_cast<uint32_t>(bin.size());
  *prim_count = static_cast<uint32_t>(order.size());
  return VKPTC_OK;
}

int32_t vkptc_get_accel_info(vkptc_ctx* ctx, vkptc_accel_info* out) {
  if (!ctx || !out) return VKPTC_INVALID_ARGUMENT;
  if (!ctx->accel_valid) return fail(ctx, VKPTC_NOT_READY, "acceleration structure not built");
  *out = ctx->accel;
  return VKPTC_OK;
}

namespace {

// The checks of a transform update; fills the refit records.
int32_t check_updates(vkptc_ctx* ctx, const vkptc_instance_update* updates, uint32_t count,
                      std::vector<RefitUpdate>& ups) {
  if (count && !updates) return fail(ctx, VKPTC_INVALID_ARGUMENT, "updates is null");
  if (!ctx->accel_valid) return fail(ctx, VKPTC_NOT_READY, "transform update before build_or_update_acceleration");
  const uint32_t ninst = static_cast<uint32_t>(ctx->raw_instances.size() / 3);
  for (uint32_t u = 0; u < count; ++u) {
    const uint32_t i = updates[u].instance_index;
    if (i >= ninst && ctx->geo_ready && ctx->raw_instances.empty())
      return fail(ctx, VKPTC_UNSUPPORTED, "transform updates need the device build");
    if (i >= ninst) return fail(ctx, VKPTC_INVALID_ARGUMENT, "transform update references an unknown instance");
    const uint32_t* loc = ctx->raw_instance_local.empty() ? nullptr : &ctx->raw_instance_local[5 * i];
    if (!loc || (loc[0] & 1u) == 0u || loc[2] == 0u || loc[4] == 0u)
      return fail(ctx, VKPTC_UNSUPPORTED, "transform update needs dynamic local geometry metadata");
    if (!ctx->refit) return fail(ctx, VKPTC_UNSUPPORTED, "transform updates need the device build");
    // refit_instance_primitives' checks (32-bit index arithmetic)
    const uint32_t tri_count = ctx->raw_instances[3 * i + 1];
    if (ctx->refit->host_inst_count[i] != tri_count)
      return fail(ctx, VKPTC_INVALID_ARGUMENT, "failed while refitting instance primitives");
    const uint32_t local_end = loc[1] + loc[2];
    for (uint32_t k = 0; k < tri_count; ++k) {
      const uint32_t base = loc[3] + k * 3u;
      if (base >= 0xFFFFFFFEu || base + 2u >= ctx->raw_local_indices_host.size())
        return fail(ctx, VKPTC_INVALID_ARGUMENT, "failed while refitting instance primitives");
      for (int j = 0; j < 3; ++j) {
        const uint32_t v = loc[1] + ctx->raw_local_indices_host[base + j];
        if (v >= local_end || v >= ctx->raw_local_vertex_count)
          return fail(ctx, VKPTC_INVALID_ARGUMENT, "failed while refitting instance primitives");
      }
    }
    RefitUpdate r{};
    r.instance = i;
    r.prim_first = ctx->refit->host_inst_first[i];
    r.prim_count = tri_count;
    r.local_first_vertex = loc[1];
    r.local_first_index = loc[3];
    r.material = ctx->raw_instances[3 * i + 2];
    const vkptc_instance_update& up = updates[u];
    const float t[10] = {up.translation[0], up.translation[1], up.translation[2], up.rotation[0], up.rotation[1],
                         up.rotation[2], up.rotation[3], up.scale[0], up.scale[1], up.scale[2]};
    std::copy(t, t + 10, r.transform);
    ups.push_back(r);
  }
  return VKPTC_OK;
}

}  // namespace

int32_t vkptc_check_instance_transforms(vkptc_ctx* ctx, const vkptc_instance_update* updates, uint32_t count) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  std::vector<RefitUpdate> ups;
  const int32_t rc = check_updates(ctx, updates, count, ups);
  if (rc == VKPTC_OK) ctx->last_error.clear();
  return rc;
}

int32_t vkptc_update_instance_transforms(vkptc_ctx* ctx, const vkptc_instance_update* updates, uint32_t count) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  std::vector<RefitUpdate> ups;
  const int32_t rc = check_updates(ctx, updates, count, ups);
  if (rc != VKPTC_OK) return rc;
  cudaSetDevice(ctx->device);
  VKPTC_CUDA(ctx, drain(ctx), "waiting for the work queued on the context's stream");
  VKPTC_CUDA(ctx, RefitOnDevice(*ctx->refit, ups, ctx->d_raw_local_vertices.ptr, ctx->d_raw_local_indices.ptr,
                                ctx->d_ref_nodes, ctx->d_ref_order, ctx->ref_count, ctx->d_nodes.ptr,
                                ctx->accel.wide_node_count, ctx->d_tris.ptr, ctx->d_tie.ptr, ctx->d_shade.ptr,
                                ctx->stream), "instance refit");
  // the scene metadata follows (ApplyInstanceTransformUpdates, metadata only)
  for (uint32_t u = 0; u < count; ++u) {
    const uint32_t i = updates[u].instance_index;
    ctx->raw_instance_local[5 * i] |= updates[u].flags;
    std::copy(ups[u].transform, ups[u].transform + 10, ctx->raw_instance_transforms.begin() + 10 * i);
  }
  ctx->geo_ready = false;   // a host flatten (external BVH) must use the new transforms
  ctx->last_error.clear();
  return VKPTC_OK;
}

int32_t vkptc_update_camera(vkptc_ctx* ctx, const vkptc_camera* camera) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  if (!ctx->configured || !ctx->has_scene)
    return fail(ctx, VKPTC_NOT_READY, "update_camera_state requires a configured tracer with a scene");
  if (!camera) return fail(ctx, VKPTC_INVALID_ARGUMENT, "camera is null");
  HostCamera& c = ctx->cam;
  std::memcpy(c.pos, camera->position, 12);
  std::memcpy(c.target, camera->target, 12);
  std::memcpy(c.up, camera->up, 12);
  c.fov = camera->fov_deg;
  c.aperture = camera->aperture_radius;
  c.focus = camera->focus_distance;
  c.iris_blades = camera->iris_blade_count;
  c.iris_rotation = camera->iris_rotation_degrees;
  c.iris_roundness = camera->iris_roundness;
  c.squeeze = camera->anamorphic_squeeze;
  ctx->adj.forward_done = false;   // a backward pass must follow a forward pass with this camera
  ctx->last_error.clear();
  return VKPTC_OK;
}

int32_t vkptc_get_camera(vkptc_ctx* ctx, vkptc_camera* out) {
  if (!ctx || !out) return VKPTC_INVALID_ARGUMENT;
  if (!ctx->has_scene) return fail(ctx, VKPTC_NOT_READY, "no scene loaded");
  const HostCamera& c = ctx->cam;
  std::memcpy(out->position, c.pos, 12);
  std::memcpy(out->target, c.target, 12);
  std::memcpy(out->up, c.up, 12);
  out->fov_deg = c.fov;
  out->aperture_radius = c.aperture;
  out->focus_distance = c.focus;
  out->iris_blade_count = c.iris_blades;
  out->iris_rotation_degrees = c.iris_rotation;
  out->iris_roundness = c.iris_roundness;
  out->anamorphic_squeeze = c.squeeze;
  return VKPTC_OK;
}

int32_t vkptc_update_scene_delta(vkptc_ctx* ctx, const vkptc_scene_delta* d) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  if (!ctx->configured || !ctx->has_scene)
    return fail(ctx, VKPTC_NOT_READY, "update_scene_delta requires a configured tracer with a scene");
  if (!d) return fail(ctx, VKPTC_INVALID_ARGUMENT, "scene delta is null");
  if ((d->material_count && (!d->material_indices || !d->materials)) ||
      (d->light_count && (!d->light_indices || !d->lights)) ||
      (d->instance_material_count && (!d->instance_indices || !d->instance_material_indices)))
    return fail(ctx, VKPTC_INVALID_ARGUMENT, "scene delta array pointer is null");
  // ApplySceneDeltaUpdate's checks, all before anything changes
  // (src/pathtracer/PathTracer.cpp:428-451).
  const uint32_t n_mat = static_cast<uint32_t>(ctx->materials.size() / 16);
  const uint32_t n_light = static_cast<uint32_t>(ctx->lights.size() / 16);
  for (uint32_t k = 0; k < d->material_count; ++k)
    if (d->material_indices[k] >= n_mat)
      return fail(ctx, VKPTC_INVALID_ARGUMENT, "scene delta did not apply: material index out of range");
  for (uint32_t k = 0; k < d->light_count; ++k)
    if (d->light_indices[k] >= n_light)
      return fail(ctx, VKPTC_INVALID_ARGUMENT, "scene delta did not apply: light index out of range");
  for (uint32_t k = 0; k < d->instance_material_count; ++k)
    if (d->instance_indices[k] >= ctx->instance_count || d->instance_material_indices[k] >= n_mat)
      return fail(ctx, VKPTC_INVALID_ARGUMENT, "scene delta did not apply: instance or material index out of range");
  // Which instances end with a new material (the last update of an instance wins).
  std::vector<uint32_t> next = ctx->instance_material;
  bool changed = d->material_count > 0u || d->light_count > 0u || d->environment_changed != 0u;
  for (uint32_t k = 0; k < d->instance_material_count; ++k) {
    const uint32_t i = d->instance_indices[k];
    if (next[i] != d->instance_material_indices[k]) changed = true;
    next[i] = d->instance_material_indices[k];
  }
  if (!changed) return fail(ctx, VKPTC_INVALID_ARGUMENT, "scene delta did not apply: nothing changed");
  cudaSetDevice(ctx->device);
  // Renders already enqueued finish with the old tables.
  VKPTC_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "synchronize");
  for (uint32_t k = 0; k < d->material_count; ++k)
    std::copy(d->materials + 16ull * k, d->materials + 16ull * (k + 1), ctx->materials.begin() + 16ull * d->material_indices[k]);
  for (uint32_t k = 0; k < d->light_count; ++k) {
    float* w = &ctx->lights[16ull * d->light_indices[k]];
    std::copy(d->lights + 16ull * k, d->lights + 16ull * (k + 1), w);
    w[7] = std::max(0.0f, w[7]);
  }
  // Pageable copies on the context's stream: staged before the call returns,
  // ordered before the next render.
  if (d->material_count) {
    scan_materials(ctx);
    VKPTC_CUDA(ctx, cudaMemcpyAsync(ctx->d_materials.ptr, ctx->materials.data(), ctx->materials.size() * sizeof(float),
                                    cudaMemcpyHostToDevice, ctx->stream), "material upload");
  }
  if (d->light_count)
    VKPTC_CUDA(ctx, cudaMemcpyAsync(ctx->d_lights.ptr, ctx->lights.data(), ctx->lights.size() * sizeof(float),
                                    cudaMemcpyHostToDevice, ctx->stream), "light upload");
  if (d->environment_changed) std::memcpy(ctx->env, d->environment, sizeof(ctx->env));
  // Instance materials: the instance table kept for later builds, the host
  // flattening when there is one, and the shading records of the built
  // accelerator.
  std::vector<uint4> ranges;
  for (uint32_t i = 0; i < ctx->instance_count; ++i) {
    if (next[i] == ctx->instance_material[i]) continue;
    ctx->instance_material[i] = next[i];
    if (3ull * i + 2 < ctx->raw_instances.size()) ctx->raw_instances[3ull * i + 2] = next[i];
    if (ctx->geo_ready && i < ctx->geo.inst_first.size())
      for (uint32_t k = 0; k < ctx->geo.inst_count[i]; ++k) ctx->geo.prims[ctx->geo.inst_first[i] + k].material = next[i];
    if (ctx->accel_valid && i + 1 < ctx->inst_prims.size() && ctx->inst_prims[i + 1] > ctx->inst_prims[i])
      ranges.push_back(make_uint4(ctx->inst_prims[i], ctx->inst_prims[i + 1] - ctx->inst_prims[i], next[i], 0u));
  }
  if (!ranges.empty()) {
    VKPTC_CUDA(ctx, ctx->d_delta_ranges.alloc(ranges.size()), "delta alloc");
    VKPTC_CUDA(ctx, cudaMemcpyAsync(ctx->d_delta_ranges.ptr, ranges.data(), ranges.size() * sizeof(uint4),
                                    cudaMemcpyHostToDevice, ctx->stream), "delta upload");
    VKPTC_CUDA(ctx, LaunchSetInstanceMaterials(ctx->d_shade.ptr, ctx->d_delta_ranges.ptr,
                                               static_cast<uint32_t>(ranges.size()), ctx->stream), "delta launch");
  }
  ctx->adj.setup = false;   // the adjoint's material tables were taken from the old scene
  ctx->adj.forward_done = false;
  ctx->last_error.clear();
  return VKPTC_OK;
}

int32_t vkptc_read_accel(vkptc_ctx* ctx, uint32_t what, void* out, uint64_t capacity, uint64_t* bytes) {
  if (!ctx || !bytes) return VKPTC_INVALID_ARGUMENT;
  if (!ctx->accel_valid) return fail(ctx, VKPTC_NOT_READY, "acceleration structure not built");
  const void* src = nullptr;
  uint64_t n = 0;
  switch (what) {
    case VKPTC_ACCEL_WIDE_NODES:
      src = ctx->d_nodes.ptr;
      n = static_cast<uint64_t>(ctx->accel.wide_node_count) * sizeof(WideNode);
      break;
    case VKPTC_ACCEL_TRIANGLES:
      src = ctx->d_tris.ptr;
      n = static_cast<uint64_t>(ctx->prim_count) * sizeof(TriRecord);
      break;
    case VKPTC_ACCEL_TIE_NODES:
      src = ctx->d_tie.ptr;
      n = ctx->prim_count ? static_cast<uint64_t>(ctx->accel.binary_node_count) * sizeof(TieNode) : 0u;
      break;
    case VKPTC_ACCEL_SHADING:
      src = ctx->d_shade.ptr;
      n = static_cast<uint64_t>(ctx->prim_count) * sizeof(float4);
      break;
    default:
      return fail(ctx, VKPTC_INVALID_ARGUMENT, "unknown accelerator array");
  }
  *bytes = n;
  if (!out || n == 0) return VKPTC_OK;
  if (capacity < n) return fail(ctx, VKPTC_INVALID_ARGUMENT, "output buffer too small");
  cudaSetDevice(ctx->device);
  VKPTC_CUDA(ctx, cudaMemcpyAsync(out, src, n, cudaMemcpyDeviceToHost, ctx->stream), "accel read");
  VKPTC_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "accel read");
  return VKPTC_OK;
}

int32_t vkptc_reset(vkptc_ctx* ctx) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  if (!ctx->configured) return fail(ctx, VKPTC_NOT_READY, "reset_accumulation called before configure");
  cudaSetDevice(ctx->device);
  VKPTC_CUDA(ctx, cudaMemsetAsync(ctx->d_film_sum.ptr, 0, ctx->d_film_sum.bytes(), ctx->stream), "film clear");
  VKPTC_CUDA(ctx, cudaMemsetAsync(ctx->d_film_count.ptr, 0, ctx->d_film_count.bytes(), ctx->stream), "film clear");
  VKPTC_CUDA(ctx, cudaMemsetAsync(ctx->d_film_invalid.ptr, 0, ctx->d_film_invalid.bytes(), ctx->stream), "film clear");
  VKPTC_CUDA(ctx, cudaMemsetAsync(ctx->d_ctr.ptr, 0, sizeof(DevCounters), ctx->stream), "counter clear");
  ctx->current_sample = 0;
  ++ctx->accumulation_gen;
  ctx->last_error.clear();
  return VKPTC_OK;
}

int32_t vkptc_shutdown(vkptc_ctx* ctx) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  ctx->configured = ctx->has_scene = ctx->accel_valid = false;
  ctx->adj.setup = false;
  ctx->geo = SceneGeometry{};
  ctx->geo_ready = false;
  ctx->d_raw_vertices.release();
  ctx->d_raw_indices.release();
  ctx->raw_instances.clear();
  ctx->d_raw_local_vertices.release();
  ctx->d_raw_local_indices.release();
  ctx->raw_instance_local.clear();
  ctx->raw_instance_transforms.clear();
  ctx->raw_local_indices_host.clear();
  release_refit(ctx);
  ctx->prim_count = 0;
  ctx->wide = WideBvh{};
  ctx->d_nodes.release();
  ctx->d_tris.release();
  ctx->d_tie.release();
  ctx->d_shade.release();
  ctx->d_materials.release();
  ctx->d_lights.release();
  ctx->d_film_sum.release();
  ctx->d_film_count.release();
  ctx->d_film_invalid.release();
  ctx->current_sample = 0;
  ctx->accumulation_gen = 0;
  ctx->last_error.clear();
  return VKPTC_OK;
}

int32_t vkptc_render(vkptc_ctx* ctx, const vkptc_tile* tiles, uint32_t tile_count, uint32_t frame,
                     const volatile int32_t* cancel_flag) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  if (!ctx->configured || !ctx->has_scene) return fail(ctx, VKPTC_NOT_READY, "render_tile requires a configured tracer with a scene");
  if (!ctx->accel_valid) return fail(ctx, VKPTC_NOT_READY, "render_tile requires a built acceleration structure");
  if (tile_count && !tiles) return fail(ctx, VKPTC_INVALID_ARGUMENT, "tiles is null");
  cudaSetDevice(ctx->device);
  const auto t0 = std::chrono::steady_clock::now();
  for (uint32_t k = 0; k < tile_count; ++k) {
    if (cancel_flag && *cancel_flag) return fail(ctx, VKPTC_CANCELLED, "render_tile cancelled");
    const vkptc_tile& t = tiles[k];
    // Clip to the film as the reference does (ScalarCpuPathTracer.Render.cpp:171-176).
    const uint32_t x0 = std::min(t.x, ctx->settings.width), y0 = std::min(t.y, ctx->settings.height);
    const uint32_t x1 = static_cast<uint32_t>(std::min<uint64_t>(ctx->settings.width, static_cast<uint64_t>(x0) + t.width));
    const uint32_t y1 = static_cast<uint32_t>(std::min<uint64_t>(ctx->settings.height, static_cast<uint64_t>(y0) + t.height));
    if (x0 >= x1 || y0 >= y1) continue;
    WaveTile wt{x0, y0, x1 - x0, y1 - y0, t.sample_index, 1u};
    const int32_t rc = run_wave(ctx, wt, frame);
    if (rc != VKPTC_OK) return rc;
    ctx->current_sample = std::max(ctx->current_sample, t.sample_index + 1u);
  }
  const int32_t rc = check_device_error(ctx);
  ctx->last_sample_us = static_cast<uint64_t>(
      std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count());
  if (rc == VKPTC_OK) ctx->last_error.clear();
  return rc;
}

int32_t vkptc_render_frame(vkptc_ctx* ctx, uint32_t first_sample, uint32_t sample_count, uint32_t frame) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  if (!ctx->configured || !ctx->has_scene) return fail(ctx, VKPTC_NOT_READY, "render requires a configured tracer with a scene");
  if (!ctx->accel_valid) return fail(ctx, VKPTC_NOT_READY, "render requires a built acceleration structure");
  cudaSetDevice(ctx->device);
  const uint32_t px = ctx->settings.width * ctx->settings.height;
  if (px == 0 || sample_count == 0) return VKPTC_OK;
  const uint32_t per_wave = std::max(1u, std::min(sample_count, wave_paths(ctx) / px));
  for (uint32_t s = 0; s < sample_count; s += per_wave) {
    const uint32_t n = std::min(per_wave, sample_count - s);
    WaveTile wt{0u, 0u, ctx->settings.width, ctx->settings.height, first_sample + s, n};
    const int32_t rc = run_wave(ctx, wt, frame);
    if (rc != VKPTC_OK) return rc;
  }
  ctx->current_sample = std::max(ctx->current_sample, first_sample + sample_count);
  return VKPTC_OK;
}

int32_t vkptc_measure_read_bandwidth(vkptc_ctx* ctx, uint64_t bytes, uint32_t reps, double* gbs) {
  if (!ctx || !gbs) return VKPTC_INVALID_ARGUMENT;
  if (bytes < 16u || (bytes & 15u) != 0u || reps == 0u) {
    return fail(ctx, VKPTC_INVALID_ARGUMENT, "bandwidth probe: bytes must be a non-zero multiple of 16, reps >= 1");
  }
  cudaSetDevice(ctx->device);
  VKPTC_CUDA(ctx, drain(ctx), "waiting for the work queued on the context's stream");
  DevBuf<float4> buf;
  DevBuf<float> sink;
  VKPTC_CUDA(ctx, buf.alloc(bytes / 16u), "bandwidth probe buffer");
  VKPTC_CUDA(ctx, sink.alloc(1), "bandwidth probe buffer");
  VKPTC_CUDA(ctx, cudaMemsetAsync(buf.ptr, 0, bytes, ctx->stream), "bandwidth probe clear");
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  VKPTC_CUDA(ctx, cudaEventCreate(&e0), "event");
  VKPTC_CUDA(ctx, cudaEventCreate(&e1), "event");
  const int grid = ctx->sm_count * 8;   // 8 blocks of 256 threads per SM
  cudaError_t e = LaunchReadProbe(buf.ptr, bytes, 1u, grid, sink.ptr, ctx->stream);   // warm-up pass
  if (e == cudaSuccess) e = cudaEventRecord(e0, ctx->stream);
  if (e == cudaSuccess) e = LaunchReadProbe(buf.ptr, bytes, reps, grid, sink.ptr, ctx->stream);
  if (e == cudaSuccess) e = cudaEventRecord(e1, ctx->stream);
  if (e == cudaSuccess) e = cudaEventSynchronize(e1);
  float ms = 0.0f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  VKPTC_CUDA(ctx, e, "bandwidth probe");
  *gbs = ms > 0.0f ? static_cast<double>(bytes) * reps / (ms / 1e3) / 1e9 : 0.0;
  return VKPTC_OK;
}

int32_t vkptc_device_name(vkptc_ctx* ctx, char* out, uint32_t capacity, uint32_t* sm_count) {
  if (!ctx || !out || capacity == 0u) return VKPTC_INVALID_ARGUMENT;
  cudaDeviceProp p{};
  VKPTC_CUDA(ctx, cudaGetDeviceProperties(&p, ctx->device), "device properties");
  std::strncpy(out, p.name, capacity - 1u);
  out[capacity - 1u] = '\0';
  if (sm_count) *sm_count = static_cast<uint32_t>(p.multiProcessorCount);
  return VKPTC_OK;
}

int32_t vkptc_set_stream(vkptc_ctx* ctx, void* stream) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
  return VKPTC_OK;
}

int32_t vkptc_read_stage_times(vkptc_ctx* ctx, double* ms_out, uint64_t* launches_out) {
  if (!ctx || !ms_out) return VKPTC_INVALID_ARGUMENT;
  if (!ctx->config.stage_timing) return fail(ctx, VKPTC_UNSUPPORTED, "stage timing not enabled in vkptc_config");
  for (int k = 0; k < StageTimer::kStages; ++k) {
    ms_out[k] = ctx->stage_ms[k];
    if (launches_out) launches_out[k] = ctx->stage_launches[k];
    ctx->stage_ms[k] = 0.0;
    ctx->stage_launches[k] = 0;
  }
  return VKPTC_OK;
}

int32_t vkptc_synchronize(vkptc_ctx* ctx) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  return check_device_error(ctx);
}

// Queues the copies of a film to host memory on `stream`: the sums packed to
// rgb on the device, then copied straight into the caller's buffer.
static int32_t enqueue_film_read(vkptc_ctx* ctx, cudaStream_t stream, float* sum_rgb, uint32_t* count) {
  const size_t px = static_cast<size_t>(ctx->settings.width) * ctx->settings.height;
  if (sum_rgb && px) {
    VKPTC_CUDA(ctx, ctx->d_pack.alloc(3 * px), "film read");
    VKPTC_CUDA(ctx, LaunchPackFilm(film_of(ctx), ctx->d_pack.ptr, stream), "film read");
    VKPTC_CUDA(ctx, cudaMemcpyAsync(sum_rgb, ctx->d_pack.ptr, 3 * px * sizeof(float), cudaMemcpyDeviceToHost, stream),
               "film read");
  }
  if (count && px)
    VKPTC_CUDA(ctx, cudaMemcpyAsync(count, ctx->d_film_count.ptr, px * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream),
               "film read");
  return VKPTC_OK;
}

int32_t vkptc_read_film(vkptc_ctx* ctx, float* sum_rgb, uint32_t* count, float* invalid) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  if (!ctx->configured) return fail(ctx, VKPTC_NOT_READY, "film not configured");
  cudaSetDevice(ctx->device);
  const int32_t rc = enqueue_film_read(ctx, ctx->stream, sum_rgb, count);
  if (rc != VKPTC_OK) return rc;
  const size_t px = static_cast<size_t>(ctx->settings.width) * ctx->settings.height;
  if (invalid) VKPTC_CUDA(ctx, cudaMemcpyAsync(invalid, ctx->d_film_invalid.ptr, px * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream), "film read");
  VKPTC_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "film read");
  return VKPTC_OK;
}

int32_t vkptc_write_film(vkptc_ctx* ctx, const float* sum_rgb, const uint32_t* count, const float* invalid) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  if (!ctx->configured) return fail(ctx, VKPTC_NOT_READY, "replace_film_history called before configure");
  if (!sum_rgb || !count) return fail(ctx, VKPTC_INVALID_ARGUMENT, "film arrays are null");
  cudaSetDevice(ctx->device);
  VKPTC_CUDA(ctx, drain(ctx), "waiting for the work queued on the context's stream");
  const size_t px = static_cast<size_t>(ctx->settings.width) * ctx->settings.height;
  std::vector<float4> tmp(px);
  for (size_t i = 0; i < px; ++i) tmp[i] = make_float4(sum_rgb[3 * i], sum_rgb[3 * i + 1], sum_rgb[3 * i + 2], 0.0f);
  VKPTC_CUDA(ctx, cudaMemcpy(ctx->d_film_sum.ptr, tmp.data(), px * sizeof(float4), cudaMemcpyHostToDevice), "film write");
  VKPTC_CUDA(ctx, cudaMemcpy(ctx->d_film_count.ptr, count, px * sizeof(uint32_t), cudaMemcpyHostToDevice), "film write");
  if (invalid) VKPTC_CUDA(ctx, cudaMemcpy(ctx->d_film_invalid.ptr, invalid, px * sizeof(float), cudaMemcpyHostToDevice), "film write");
  else VKPTC_CUDA(ctx, cudaMemset(ctx->d_film_invalid.ptr, 0, px * sizeof(float)), "film write");
  return VKPTC_OK;
}

int32_t vkptc_resolve_hdr(vkptc_ctx* ctx, float* rgb) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  if (!ctx->configured) return fail(ctx, VKPTC_NOT_READY, "film not configured");
  if (!rgb) return fail(ctx, VKPTC_INVALID_ARGUMENT, "rgb is null");
  cudaSetDevice(ctx->device);
  const size_t px = static_cast<size_t>(ctx->settings.width) * ctx->settings.height;
  float* d_rgb = nullptr;
  VKPTC_CUDA(ctx, cudaMallocAsync(reinterpret_cast<void**>(&d_rgb), std::max<size_t>(1, 3 * px) * sizeof(float), ctx->stream), "resolve alloc");
  cudaError_t e = LaunchResolveHdr(film_of(ctx), d_rgb, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(rgb, d_rgb, 3 * px * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
  cudaFreeAsync(d_rgb, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "resolve");
  return VKPTC_OK;
}

namespace {

// ColorTemperatureToRgb and WhiteBalanceScale (src/pathtracer/FilmBuffer.cpp:30-49, 216-224),
// with the same float functions, so the scale equals the reference's.
void temperature_rgb(float kelvin, float rgb[3]) {
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

LdrResolve ldr_settings(const vkptc_film_resolve& s) {
  LdrResolve r{};
  r.exposure = s.exposure;
  float d65[3], target[3];
  temperature_rgb(6500.0f, d65);
  temperature_rgb(s.white_balance_kelvin, target);
  for (int k = 0; k < 3; ++k) r.wb[k] = d65[k] / std::max(1.0e-3f, target[k]);
  r.gamma = s.gamma;
  r.tone_map = s.tone_map;
  r.output_transform = s.output_transform;
  r.clamp_output = s.clamp_output;
  return r;
}

}  // namespace

int32_t vkptc_resolve_ldr(vkptc_ctx* ctx, const vkptc_film_resolve* settings, uint8_t* rgba) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  if (!ctx->configured) return fail(ctx, VKPTC_NOT_READY, "film not configured");
  if (!settings || !rgba) return fail(ctx, VKPTC_INVALID_ARGUMENT, "resolve argument is null");
  cudaSetDevice(ctx->device);
  const size_t px = static_cast<size_t>(ctx->settings.width) * ctx->settings.height;
  VKPTC_CUDA(ctx, ctx->d_ldr.alloc(std::max<size_t>(4, 4 * px)), "resolve alloc");
  VKPTC_CUDA(ctx, LaunchResolveLdr(film_of(ctx), ldr_settings(*settings), ctx->config.math_mode == 0u, ctx->d_ldr.ptr,
                                   ctx->stream), "resolve");
  VKPTC_CUDA(ctx, cudaMemcpyAsync(rgba, ctx->d_ldr.ptr, 4 * px, cudaMemcpyDeviceToHost, ctx->stream), "resolve read");
  VKPTC_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "resolve read");
  return VKPTC_OK;
}

int32_t vkptc_request_ldr_readback(vkptc_ctx* ctx, const vkptc_film_resolve* settings, uint64_t* token) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  if (!settings || !token) return fail(ctx, VKPTC_INVALID_ARGUMENT, "readback argument is null");
  *token = 0;
  if (!ctx->configured || !ctx->has_scene || !ctx->accel_valid)
    return fail(ctx, VKPTC_NOT_READY, "film readback requested before the backend is ready");
  cudaSetDevice(ctx->device);
  const size_t px = static_cast<size_t>(ctx->settings.width) * ctx->settings.height;
  VKPTC_CUDA(ctx, ctx->d_ldr.alloc(std::max<size_t>(4, 4 * px)), "readback alloc");
  if (ctx->h_ldr_bytes < 4 * px) {
    if (ctx->h_ldr) cudaFreeHost(ctx->h_ldr);
    ctx->h_ldr = nullptr;
    ctx->h_ldr_bytes = 0;
    VKPTC_CUDA(ctx, cudaMallocHost(reinterpret_cast<void**>(&ctx->h_ldr), std::max<size_t>(4, 4 * px)), "readback alloc");
    ctx->h_ldr_bytes = std::max<size_t>(4, 4 * px);
  }
  if (!ctx->ldr_event) VKPTC_CUDA(ctx, cudaEventCreateWithFlags(&ctx->ldr_event, cudaEventDisableTiming), "readback event");
  VKPTC_CUDA(ctx, LaunchResolveLdr(film_of(ctx), ldr_settings(*settings), ctx->config.math_mode == 0u, ctx->d_ldr.ptr,
                                   ctx->stream), "readback resolve");
  VKPTC_CUDA(ctx, cudaMemcpyAsync(ctx->h_ldr, ctx->d_ldr.ptr, 4 * px, cudaMemcpyDeviceToHost, ctx->stream), "readback copy");
  VKPTC_CUDA(ctx, cudaEventRecord(ctx->ldr_event, ctx->stream), "readback event");
  ctx->ldr_token = ctx->ldr_next_token++;
  ctx->ldr_width = ctx->settings.width;
  ctx->ldr_height = ctx->settings.height;
  *token = ctx->ldr_token;
  return VKPTC_OK;
}

int32_t vkptc_poll_ldr_readback(vkptc_ctx* ctx, uint64_t token, uint8_t* rgba, uint32_t* state) {
  if (!ctx || !state) return VKPTC_INVALID_ARGUMENT;
  *state = VKPTC_READBACK_INVALID;
  if (token == 0 || token != ctx->ldr_token || ctx->ldr_width != ctx->settings.width ||
      ctx->ldr_height != ctx->settings.height)
    return fail(ctx, VKPTC_INVALID_ARGUMENT, "invalid film readback token");
  cudaSetDevice(ctx->device);
  const cudaError_t q = cudaEventQuery(ctx->ldr_event);
  if (q == cudaErrorNotReady) {
    *state = VKPTC_READBACK_PENDING;
    return VKPTC_OK;
  }
  if (q != cudaSuccess) {
    *state = VKPTC_READBACK_FAILED;
    return cuda_fail(ctx, q, "film readback");
  }
  if (!rgba) return fail(ctx, VKPTC_INVALID_ARGUMENT, "rgba is null");
  std::memcpy(rgba, ctx->h_ldr, 4ull * ctx->ldr_width * ctx->ldr_height);
  *state = VKPTC_READBACK_READY;
  return VKPTC_OK;
}

int32_t vkptc_read_counters(vkptc_ctx* ctx, vkptc_counters* out) {
  if (!ctx || !out) return VKPTC_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  DevCounters dc{};
  VKPTC_CUDA(ctx, cudaMemcpyAsync(&dc, ctx->d_ctr.ptr, sizeof(dc), cudaMemcpyDeviceToHost, ctx->stream), "counter read");
  VKPTC_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "counter read");
  std::memset(out, 0, sizeof(*out));
  out->samples = dc.samples;
  out->rays = dc.rays;
  out->shadow_tests = dc.shadow_tests;
  out->triangle_tests = dc.tris + dc.shadow_tris;
  out->bvh_node_visits = dc.nodes + dc.shadow_nodes;
  out->bvh_leaf_visits = dc.leaves + dc.shadow_leaves;
  out->sdf_tests = dc.sdf_tests;
  out->sdf_steps = dc.sdf_steps;
  out->sdf_hits = dc.sdf_hits;
  out->sdf_misses = dc.sdf_tests - dc.sdf_hits;
  return VKPTC_OK;
}

int32_t vkptc_read_traversal_stats(vkptc_ctx* ctx, uint64_t* out) {
  if (!ctx || !out) return VKPTC_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  DevCounters dc{};
  VKPTC_CUDA(ctx, cudaMemcpyAsync(&dc, ctx->d_ctr.ptr, sizeof(dc), cudaMemcpyDeviceToHost, ctx->stream), "counter read");
  VKPTC_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "counter read");
  out[0] = dc.ext_rays;
  out[1] = dc.nodes;
  out[2] = dc.leaves;
  out[3] = dc.tris;
  out[4] = dc.shadow_rays;
  out[5] = dc.shadow_nodes;
  out[6] = dc.shadow_leaves;
  out[7] = dc.shadow_tris;
  return VKPTC_OK;
}

int32_t vkptc_get_status(vkptc_ctx* ctx, vkptc_tracer_status* out) {
  if (!ctx || !out) return VKPTC_INVALID_ARGUMENT;
  vkptc_counters c{};
  const int32_t rc = vkptc_read_counters(ctx, &c);
  std::memset(out, 0, sizeof(*out));
  out->lifecycle = lifecycle(ctx);
  out->scene_loaded = ctx->has_scene;
  out->accel_valid = ctx->accel_valid;
  out->ready_to_render = ctx->configured && ctx->has_scene && ctx->accel_valid;
  out->current_sample = ctx->current_sample;
  out->last_sample_us = ctx->last_sample_us;
  out->total_samples = c.samples;
  out->accumulation_gen = ctx->accumulation_gen;
  return rc == VKPTC_OK ? VKPTC_OK : rc;
}

const char* vkptc_last_error(vkptc_ctx* ctx) {
  if (!ctx) return "null context";
  return ctx->last_error.c_str();
}

int32_t vkptc_trace_rays_device(vkptc_ctx* ctx, const float* d_rays, const float* d_tmax, uint64_t ray_count,
                                uint32_t mode, uint32_t* d_prim_out, float* d_t_out, void* stream) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  if (!ctx->accel_valid) return fail(ctx, VKPTC_NOT_READY, "acceleration structure not built");
  if (mode > VKPTC_QUERY_ANY) return fail(ctx, VKPTC_INVALID_ARGUMENT, "unknown query mode");
  if (ray_count && (!d_rays || !d_prim_out)) return fail(ctx, VKPTC_INVALID_ARGUMENT, "ray or output pointer is null");
  cudaSetDevice(ctx->device);
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  LaunchShape ls;
  int32_t rc = launch_shape(ctx, st, ls);
  if (rc != VKPTC_OK) return rc;
  if (ray_count > 0xFFFFFFF0ull) return fail(ctx, VKPTC_INVALID_ARGUMENT, "at most 2^32 - 16 rays per call");
  bool ordered = false;
  rc = order_begin(ctx, st, &ordered);
  if (rc != VKPTC_OK) return rc;
  VKPTC_CUDA(ctx, LaunchTraceRays(dev_scene(ctx), d_rays, d_tmax, ray_count, mode == VKPTC_QUERY_ANY, d_prim_out,
                                  d_t_out, ls, ctx->config.collect_stats ? ctx->d_ctr.ptr : nullptr, ctx->d_err.ptr,
                                  ctx->d_fetch.ptr),
             "trace launch");
  return order_end(ctx, st, ordered);
}

int32_t vkptc_trace_rays(vkptc_ctx* ctx, const float* rays, const float* tmax, uint64_t ray_count, uint32_t mode,
                         uint32_t* prim_out, float* t_out) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  if (!ctx->accel_valid) return fail(ctx, VKPTC_NOT_READY, "acceleration structure not built");
  if (ray_count && (!rays || !prim_out)) return fail(ctx, VKPTC_INVALID_ARGUMENT, "ray or output pointer is null");
  if (ray_count == 0) return VKPTC_OK;
  cudaSetDevice(ctx->device);
  VKPTC_CUDA(ctx, ctx->q_rays.alloc(6 * ray_count), "query alloc");
  VKPTC_CUDA(ctx, ctx->q_prim.alloc(ray_count), "query alloc");
  VKPTC_CUDA(ctx, ctx->q_t.alloc(ray_count), "query alloc");
  if (tmax) VKPTC_CUDA(ctx, ctx->q_tmax.alloc(ray_count), "query alloc");
  VKPTC_CUDA(ctx, cudaMemcpyAsync(ctx->q_rays.ptr, rays, 6 * ray_count * sizeof(float), cudaMemcpyHostToDevice, ctx->stream), "ray upload");
  if (tmax) VKPTC_CUDA(ctx, cudaMemcpyAsync(ctx->q_tmax.ptr, tmax, ray_count * sizeof(float), cudaMemcpyHostToDevice, ctx->stream), "ray upload");
  int32_t rc = vkptc_trace_rays_device(ctx, ctx->q_rays.ptr, tmax ? ctx->q_tmax.ptr : nullptr, ray_count, mode,
                                       ctx->q_prim.ptr, ctx->q_t.ptr, nullptr);
  if (rc != VKPTC_OK) return rc;
  VKPTC_CUDA(ctx, cudaMemcpyAsync(prim_out, ctx->q_prim.ptr, ray_count * sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream), "result download");
  if (t_out) VKPTC_CUDA(ctx, cudaMemcpyAsync(t_out, ctx->q_t.ptr, ray_count * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream), "result download");
  rc = check_device_error(ctx);
  if (rc == VKPTC_OK) ctx->last_error.clear();
  return rc;
}

}  // extern "C"

// ================================================================== batches
struct vkptc_batch {
  vkptc_config config{};
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::string last_error;
  std::vector<vkptc_ctx*> jobs;
  // persistent-mode device state
  DevBuf<DevJob> d_jobs;
  DevBuf<float4> staging;
  DevBuf<uint32_t> p_job, p_local, p_depth, p_q0, p_q1, p_shq, p_fin, p_free, p_ctl;
  DevBuf<uint64_t> p_rng;
  DevBuf<float4> p_o, p_d, p_thr, p_rad, p_sh_o, p_sh_d, p_sh_c;
  DevBuf<float2> p_hit;
  DevBuf<int2> spill;
  // loop-driver state: two compacted path generations, shadow queue, finished list
  DevBuf<uint32_t> l_job[2], l_local[2], l_depth[2];
  DevBuf<uint64_t> l_rng[2];
  DevBuf<float4> l_o[2], l_d[2], l_thr[2], l_rad[2];
  DevBuf<float2> l_hit;
  DevBuf<float4> l_sh_o, l_sh_d, l_sh_c, l_fin_rad;
  DevBuf<uint32_t> l_sh_dst, l_fin_job, l_fin_local, l_ctl;
  DevBuf<DevCounters> d_ctr;
  DevBuf<uint32_t> d_err;
  size_t smem_configured = 48 * 1024;
  cudaGraphExec_t graph = nullptr;
  std::string graph_key;
  cudaStream_t body_stream = nullptr;   // captures the device-driven loop's body
  cudaStream_t side_stream = nullptr;   // the body's forked shadow branch
  cudaEvent_t fork_ev[2] = {nullptr, nullptr};
  cudaEvent_t marks[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};   // stage timing
  size_t loop_smem_configured = 48 * 1024;
  vkptc_batch_stats stats{};
};

namespace {

int32_t bfail(vkptc_batch* b, int32_t code, const std::string& msg) {
  if (b) b->last_error = msg;
  return code;
}

int32_t bcuda(vkptc_batch* b, cudaError_t e, const char* what) {
  const int32_t code = (e == cudaErrorMemoryAllocation) ? VKPTC_ALLOC_FAILED : VKPTC_INTERNAL_ERROR;
  return bfail(b, code, std::string(what) + ": " + cudaGetErrorString(e));
}

#define VKPTC_BCUDA(b, call, what)                          \
  do {                                                      \
    cudaError_t e_ = (call);                                \
    if (e_ != cudaSuccess) return bcuda(b, e_, what);       \
  } while (0)

constexpr uint32_t kDefaultPoolPaths = 1u << 21;

uint32_t job_samples(const vkptc_ctx* c, uint32_t limit) {
  const uint32_t spp = std::max(1u, c->settings.spp);
  return limit ? std::min(spp, limit) : spp;
}

void release_graph(vkptc_batch* b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
  b->graph_key.clear();
}

int32_t batch_clear_films(vkptc_batch* b) {
  for (vkptc_ctx* c : b->jobs) {
    VKPTC_BCUDA(b, cudaMemsetAsync(c->d_film_sum.ptr, 0, c->d_film_sum.bytes(), b->stream), "film clear");
    VKPTC_BCUDA(b, cudaMemsetAsync(c->d_film_count.ptr, 0, c->d_film_count.bytes(), b->stream), "film clear");
  }
  return VKPTC_OK;
}

int32_t batch_run_plain(vkptc_batch* b, const vkptc_batch_tuning& t) {
  uint64_t launches = 0;
  for (vkptc_ctx* c : b->jobs) {
    VKPTC_BCUDA(b, cudaMemsetAsync(c->d_ctr.ptr, 0, sizeof(DevCounters), b->stream), "counter clear");
  }
  VKPTC_BCUDA(b, cudaEventRecord(b->ev0, b->stream), "event");
  int32_t rc = batch_clear_films(b);
  if (rc != VKPTC_OK) return rc;
  for (vkptc_ctx* c : b->jobs) {
    cudaStream_t saved = c->stream;
    const vkptc_config saved_cfg = c->config;
    c->stream = b->stream;
    if (t.block_size) c->config.block_size = t.block_size;
    if (t.stack_depth) c->config.stack_depth = t.stack_depth;
    if (t.steps) c->config.steps = t.steps;
    const uint32_t spp = job_samples(c, t.sample_limit);
    for (uint32_t sidx = 0; sidx < spp && rc == VKPTC_OK; ++sidx) {
      // One frame per launch sequence: every sample is its own wave.
      WaveTile wt{0u, 0u, c->settings.width, c->settings.height, sidx, 1u};
      rc = run_wave(c, wt, 0u);
      launches += 2u + (c->settings.enable_nee ? 3u : 2u) * c->settings.max_depth;
    }
    c->stream = saved;
    c->config = saved_cfg;
    if (rc != VKPTC_OK) return bfail(b, rc, std::string("plain batch run: ") + c->last_error);
  }
  VKPTC_BCUDA(b, cudaEventRecord(b->ev1, b->stream), "event");
  VKPTC_BCUDA(b, cudaStreamSynchronize(b->stream), "batch sync");
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, b->ev0, b->ev1);
  uint64_t segs = 0, shadow = 0;
  for (vkptc_ctx* c : b->jobs) {
    DevCounters dc{};
    VKPTC_BCUDA(b, cudaMemcpy(&dc, c->d_ctr.ptr, sizeof(dc), cudaMemcpyDeviceToHost), "counters");
    segs += dc.rays;
    shadow += dc.shadow_tests;
    uint32_t err = 0;
    VKPTC_BCUDA(b, cudaMemcpy(&err, c->d_err.ptr, sizeof(err), cudaMemcpyDeviceToHost), "error word");
    if (err) return bfail(b, VKPTC_INTERNAL_ERROR, "device traversal stack overflow");
  }
  b->stats.segments = segs;
  b->stats.shadow_rays = shadow;
  b->stats.device_ms = ms;
  b->stats.kernel_launches = launches;
  b->stats.graph_used = 0;
  return VKPTC_OK;
}

// The pool-based modes: VKPTC_BATCH_PERSISTENT (one cooperative kernel, grid
// barriers between stages) and VKPTC_BATCH_LOOP (one kernel per stage inside
// a CUDA graph while-node; host-driven iterations without a graph).
int32_t batch_run_pool(vkptc_batch* b, const vkptc_batch_tuning& t, uint32_t mode) {
  const bool parity = b->config.math_mode == 0u;
  const bool loop = mode == VKPTC_BATCH_LOOP;
  const bool watertight = b->config.triangle_test == VKPTC_TRIANGLE_WATERTIGHT;
  for (double& v : b->stats.stage_ms) v = 0.0;
  // ---- jobs table and stagings
  std::vector<DevJob> table(b->jobs.size());
  unsigned long long total = 0, staging_px = 0;
  int stack_cap = 1;
  for (size_t k = 0; k < b->jobs.size(); ++k) {
    vkptc_ctx* c = b->jobs[k];
    DevJob& J = table[k];
    J.scene = dev_scene(c);
    J.settings = dev_settings(c, 0u);
    J.path_base = total;
    J.pixels = c->settings.width * c->settings.height;
    J.spp = job_samples(c, t.sample_limit);
    J.first_sample = 0u;
    J.film = film_of(c);
    total += static_cast<unsigned long long>(J.pixels) * J.spp;
    staging_px += static_cast<unsigned long long>(J.pixels) * J.spp;
    stack_cap = std::max(stack_cap, static_cast<int>(std::max<uint32_t>(1u, c->wide.stack_required)));
  }
  VKPTC_BCUDA(b, b->staging.alloc(std::max<unsigned long long>(1, staging_px)), "staging alloc");
  unsigned long long off = 0;
  for (DevJob& J : table) {
    J.staging = b->staging.ptr + off;
    off += static_cast<unsigned long long>(J.pixels) * J.spp;
  }
  VKPTC_BCUDA(b, b->d_jobs.alloc(table.size()), "job table alloc");
  VKPTC_BCUDA(b, cudaMemcpy(b->d_jobs.ptr, table.data(), table.size() * sizeof(DevJob), cudaMemcpyHostToDevice),
              "job table upload");
  // ---- launch shape
  BatchLaunch bl{};
  bl.block = t.block_size ? static_cast<int>(std::min(256u, std::max(32u, (t.block_size + 31u) / 32u * 32u))) : 128;
  bl.stack_cap = stack_cap;
  bl.smem_entries = std::min(stack_cap, t.stack_depth ? static_cast<int>(t.stack_depth) : kDefaultSmemEntries);
  bl.steps = steps_word(t.steps, kDefaultSteps);
  bl.stream = b->stream;
  bl.parity = parity;
  bl.stats = b->config.collect_stats != 0u;
  bl.watertight = watertight;
  bl.effects = false;
  bl.sdf = false;
  bl.exotic = false;
  for (vkptc_ctx* c : b->jobs) {
    bl.effects = bl.effects || c->has_effects;
    bl.sdf = bl.sdf || c->sdf_count != 0u;
    bl.exotic = bl.exotic || c->has_exotic || c->env_w != 0u;
  }
  // Register variant of the traversal kernels: 0..3 for both drivers; the loop
  // driver's variant 4 runs its stages in 128-thread blocks.
  bl.occupancy = static_cast<int>(std::min(loop ? 4u : 3u, t.occupancy));
  if (loop && bl.occupancy == 4) bl.block = 128;
  const size_t smem = StackSmemBytes(bl.block, bl.smem_entries);
  int max_optin = 0;
  cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, b->device);
  if (smem > static_cast<size_t>(max_optin)) return bfail(b, VKPTC_UNSUPPORTED, "stack does not fit in shared memory");
  LoopGrids lg{};
  if (loop) {
    if (smem > b->loop_smem_configured) {
      VKPTC_BCUDA(b, ConfigureBatchLoopSmem(smem), "shared memory limit");
      b->loop_smem_configured = smem;
    }
    lg = BatchLoopGrids(bl.block, smem, parity, bl.stats, bl.occupancy, b->sm_count, watertight, bl.effects, bl.sdf,
                        bl.exotic);
    if (lg.regen <= 0 || lg.extend <= 0 || lg.shade <= 0 || lg.shadow <= 0 || lg.finish <= 0) {
      return bfail(b, VKPTC_UNSUPPORTED, "a batch stage kernel does not fit on an SM with this block size");
    }
    bl.grid = std::max(lg.extend, lg.shadow);   // the traversal stages own the spill area
  } else {
    if (smem > b->smem_configured) {
      VKPTC_BCUDA(b, ConfigureBatchSmem(smem), "shared memory limit");
      b->smem_configured = smem;
    }
    const int per_sm = BatchBlocksPerSm(bl.block, smem, parity, bl.stats, bl.occupancy, watertight);
    if (per_sm <= 0) return bfail(b, VKPTC_UNSUPPORTED, "persistent batch kernel does not fit on an SM with this block size");
    bl.grid = per_sm * b->sm_count;
  }
  const size_t spill_entries =
      bl.stack_cap > bl.smem_entries ? static_cast<size_t>(bl.grid) * bl.block * (bl.stack_cap - bl.smem_entries) : 0;
  // The loop driver's shadow stage may run beside EXTEND: it spills into a second half.
  if (spill_entries) VKPTC_BCUDA(b, b->spill.alloc(loop ? 2 * spill_entries : spill_entries), "spill alloc");
  bl.spill = spill_entries ? b->spill.ptr : nullptr;
  bl.spill_shadow = spill_entries && loop ? b->spill.ptr + spill_entries : bl.spill;
  // ---- pool
  const uint32_t cap = std::max<uint32_t>(1024u, t.pool_paths ? t.pool_paths : kDefaultPoolPaths);
  const size_t n = cap;
  BatchPool P{};
  LoopPool LP{};
  if (loop) {
    for (int g = 0; g < 2; ++g) {
      VKPTC_BCUDA(b, b->l_job[g].alloc(n), "pool alloc");
      VKPTC_BCUDA(b, b->l_local[g].alloc(n), "pool alloc");
      VKPTC_BCUDA(b, b->l_depth[g].alloc(n), "pool alloc");
      VKPTC_BCUDA(b, b->l_rng[g].alloc(n), "pool alloc");
      VKPTC_BCUDA(b, b->l_o[g].alloc(n), "pool alloc");
      VKPTC_BCUDA(b, b->l_d[g].alloc(n), "pool alloc");
      VKPTC_BCUDA(b, b->l_thr[g].alloc(n), "pool alloc");
      VKPTC_BCUDA(b, b->l_rad[g].alloc(n), "pool alloc");
      LP.gen[g] = PathSoA{b->l_job[g].ptr, b->l_local[g].ptr, b->l_depth[g].ptr, b->l_rng[g].ptr,
                          b->l_o[g].ptr,   b->l_d[g].ptr,     b->l_thr[g].ptr,   b->l_rad[g].ptr};
    }
    VKPTC_BCUDA(b, b->l_hit.alloc(n), "pool alloc");
    VKPTC_BCUDA(b, b->l_sh_o.alloc(n), "pool alloc");
    VKPTC_BCUDA(b, b->l_sh_d.alloc(n), "pool alloc");
    VKPTC_BCUDA(b, b->l_sh_c.alloc(n), "pool alloc");
    VKPTC_BCUDA(b, b->l_sh_dst.alloc(n), "pool alloc");
    VKPTC_BCUDA(b, b->l_fin_rad.alloc(n), "pool alloc");
    VKPTC_BCUDA(b, b->l_fin_job.alloc(n), "pool alloc");
    VKPTC_BCUDA(b, b->l_fin_local.alloc(n), "pool alloc");
    VKPTC_BCUDA(b, b->l_ctl.alloc(kLoopCtlWords), "pool alloc");
    LP.capacity = cap;
    LP.hit = b->l_hit.ptr;
    LP.sh_o = b->l_sh_o.ptr;
    LP.sh_d = b->l_sh_d.ptr;
    LP.sh_c = b->l_sh_c.ptr;
    LP.sh_dst = b->l_sh_dst.ptr;
    LP.fin_rad = b->l_fin_rad.ptr;
    LP.fin_job = b->l_fin_job.ptr;
    LP.fin_local = b->l_fin_local.ptr;
    LP.ctl = b->l_ctl.ptr;
  } else {
  VKPTC_BCUDA(b, b->p_job.alloc(n), "pool alloc");
  VKPTC_BCUDA(b, b->p_local.alloc(n), "pool alloc");
  VKPTC_BCUDA(b, b->p_depth.alloc(n), "pool alloc");
  VKPTC_BCUDA(b, b->p_q0.alloc(n), "pool alloc");
  VKPTC_BCUDA(b, b->p_q1.alloc(n), "pool alloc");
  VKPTC_BCUDA(b, b->p_shq.alloc(n), "pool alloc");
  VKPTC_BCUDA(b, b->p_fin.alloc(n), "pool alloc");
  VKPTC_BCUDA(b, b->p_free.alloc(n), "pool alloc");
  VKPTC_BCUDA(b, b->p_ctl.alloc(kBatchCtlWords), "pool alloc");
  VKPTC_BCUDA(b, b->p_rng.alloc(n), "pool alloc");
  VKPTC_BCUDA(b, b->p_o.alloc(n), "pool alloc");
  VKPTC_BCUDA(b, b->p_d.alloc(n), "pool alloc");
  VKPTC_BCUDA(b, b->p_thr.alloc(n), "pool alloc");
  VKPTC_BCUDA(b, b->p_rad.alloc(n), "pool alloc");
  VKPTC_BCUDA(b, b->p_sh_o.alloc(n), "pool alloc");
  VKPTC_BCUDA(b, b->p_sh_d.alloc(n), "pool alloc");
  VKPTC_BCUDA(b, b->p_sh_c.alloc(n), "pool alloc");
  VKPTC_BCUDA(b, b->p_hit.alloc(n), "pool alloc");
  P.capacity = cap;
  P.job = b->p_job.ptr;
  P.local = b->p_local.ptr;
  P.depth = b->p_depth.ptr;
  P.rng = b->p_rng.ptr;
  P.ray_o = b->p_o.ptr;
  P.ray_d = b->p_d.ptr;
  P.thr = b->p_thr.ptr;
  P.rad = b->p_rad.ptr;
  P.hit = b->p_hit.ptr;
  P.ext[0] = b->p_q0.ptr;
  P.ext[1] = b->p_q1.ptr;
  P.shq = b->p_shq.ptr;
  P.sh_o = b->p_sh_o.ptr;
  P.sh_d = b->p_sh_d.ptr;
  P.sh_c = b->p_sh_c.ptr;
  P.fin = b->p_fin.ptr;
  P.freel = b->p_free.ptr;
  P.ctl = b->p_ctl.ptr;
  P.barrier_spins = t.barrier_spins ? t.barrier_spins : kBatchBarrierSpins;
  }

  // ---- the run: film clear, pool reset, the pool iterations, in-order accumulation
  const uint32_t njobs = static_cast<uint32_t>(table.size());
  auto prologue = [&]() -> int32_t {
    int32_t rc = batch_clear_films(b);
    if (rc != VKPTC_OK) return rc;
    VKPTC_BCUDA(b, cudaMemsetAsync(b->d_ctr.ptr, 0, sizeof(DevCounters), b->stream), "counter clear");
    // the error word of the previous run (a barrier timeout) must not outlive it
    VKPTC_BCUDA(b, cudaMemsetAsync(b->d_err.ptr, 0, sizeof(uint32_t), b->stream), "error word clear");
    if (loop) VKPTC_BCUDA(b, LaunchBatchLoopInit(LP, b->stream), "pool init");
    else VKPTC_BCUDA(b, LaunchBatchInit(P, b->stream), "pool init");
    return VKPTC_OK;
  };
  auto epilogue = [&]() -> int32_t {
    VKPTC_BCUDA(b, LaunchStagingAccumulate(b->d_jobs.ptr, njobs, staging_px, b->stream, b->d_ctr.ptr),
                "staging accumulate");
    return VKPTC_OK;
  };
  // Everything but a host-driven loop is one stream sequence (capturable).
  auto enqueue = [&]() -> int32_t {
    int32_t rc = prologue();
    if (rc != VKPTC_OK) return rc;
    if (!loop) {
      VKPTC_BCUDA(b, LaunchBatchPersistent(b->d_jobs.ptr, njobs, total, P, bl, b->d_ctr.ptr, b->d_err.ptr),
                  "persistent launch");
    } else {
      // Inside a capture: a while-node whose body is one iteration of the stages.
      cudaStreamCaptureStatus status;
      cudaGraph_t cg = nullptr;
      const cudaGraphNode_t* deps = nullptr;
      size_t ndeps = 0;
      VKPTC_BCUDA(b, cudaStreamGetCaptureInfo(b->stream, &status, nullptr, &cg, &deps, &ndeps), "capture info");
      if (status != cudaStreamCaptureStatusActive) return bfail(b, VKPTC_INTERNAL_ERROR, "loop mode needs a capture");
      cudaGraphConditionalHandle handle;
      VKPTC_BCUDA(b, cudaGraphConditionalHandleCreate(&handle, cg, 1u, cudaGraphCondAssignDefault), "conditional handle");
      cudaGraphNodeParams cp{};
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = handle;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      cudaGraphNode_t cnode;
      VKPTC_BCUDA(b, cudaGraphAddNode(&cnode, cg, deps, ndeps, &cp), "while node");
      VKPTC_BCUDA(b, cudaStreamUpdateCaptureDependencies(b->stream, &cnode, 1, cudaStreamSetCaptureDependencies),
                  "capture dependencies");
      if (!b->body_stream) VKPTC_BCUDA(b, cudaStreamCreateWithFlags(&b->body_stream, cudaStreamNonBlocking), "stream");
      VKPTC_BCUDA(b, cudaStreamBeginCaptureToGraph(b->body_stream, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                   cudaStreamCaptureModeRelaxed),
                  "body capture");
      if (!b->side_stream) {
        VKPTC_BCUDA(b, cudaStreamCreateWithFlags(&b->side_stream, cudaStreamNonBlocking), "stream");
        VKPTC_BCUDA(b, cudaEventCreateWithFlags(&b->fork_ev[0], cudaEventDisableTiming), "fork events");
        VKPTC_BCUDA(b, cudaEventCreateWithFlags(&b->fork_ev[1], cudaEventDisableTiming), "fork events");
      }
      BatchLaunch bb = bl;
      bb.stream = b->body_stream;
      const LoopFork fork{b->side_stream, b->fork_ev[0], b->fork_ev[1]};
      const cudaError_t el = LaunchBatchLoopIteration(b->d_jobs.ptr, njobs, total, LP, bb, lg, handle, b->d_ctr.ptr,
                                                      b->d_err.ptr, nullptr, &fork);
      cudaGraph_t body = nullptr;
      const cudaError_t ee = cudaStreamEndCapture(b->body_stream, &body);
      if (el != cudaSuccess) return bcuda(b, el, "loop body");
      if (ee != cudaSuccess) return bcuda(b, ee, "body capture");
    }
    return epilogue();
  };
  VKPTC_BCUDA(b, cudaMemsetAsync(b->d_err.ptr, 0, sizeof(uint32_t), b->stream), "error clear");
  bool graph_used = false;
  if (t.use_graph) {
    const std::string key = std::string(loop ? "loop/" : "persistent/") + std::to_string(cap) + "/" +
                            std::to_string(bl.block) + "/" + std::to_string(bl.smem_entries) +
                            "/o" + std::to_string(bl.occupancy) + "/b" + std::to_string(t.barrier_spins) +
                            "/" + std::to_string(bl.steps) + "/" + std::to_string(t.sample_limit) + "/" +
                            std::to_string(b->jobs.size()) + "/" +
                            std::to_string(reinterpret_cast<uintptr_t>(b->staging.ptr)) + "/" +
                            std::to_string(reinterpret_cast<uintptr_t>(loop ? b->l_job[0].ptr : b->p_job.ptr));
    if (!b->graph || b->graph_key != key) {
      release_graph(b);
      VKPTC_BCUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "graph capture");
      const int32_t rc = enqueue();
      cudaGraph_t g = nullptr;
      const cudaError_t ec = cudaStreamEndCapture(b->stream, &g);
      if (rc != VKPTC_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
      }
      if (ec != cudaSuccess) return bcuda(b, ec, "graph capture");
      const cudaError_t ei = cudaGraphInstantiate(&b->graph, g, 0);
      cudaGraphDestroy(g);
      if (ei != cudaSuccess) {
        b->graph = nullptr;
        return bcuda(b, ei, "graph instantiate");
      }
      b->graph_key = key;
    }
    VKPTC_BCUDA(b, cudaEventRecord(b->ev0, b->stream), "event");
    VKPTC_BCUDA(b, cudaGraphLaunch(b->graph, b->stream), "graph launch");
    VKPTC_BCUDA(b, cudaEventRecord(b->ev1, b->stream), "event");
    graph_used = true;
  } else if (!loop) {
    VKPTC_BCUDA(b, cudaEventRecord(b->ev0, b->stream), "event");
    const int32_t rc = enqueue();
    if (rc != VKPTC_OK) return rc;
    VKPTC_BCUDA(b, cudaEventRecord(b->ev1, b->stream), "event");
  } else {
    // Host-driven loop (no graph): one iteration per round trip; with
    // stage_timing, CUDA events around every stage launch.
    const bool timing = b->config.stage_timing != 0u;
    if (timing && !b->marks[0]) {
      for (auto& e : b->marks) VKPTC_BCUDA(b, cudaEventCreate(&e), "stage events");
    }
    double stage_ms[5] = {0, 0, 0, 0, 0};
    VKPTC_BCUDA(b, cudaEventRecord(b->ev0, b->stream), "event");
    int32_t rc = prologue();
    if (rc != VKPTC_OK) return rc;
    for (;;) {
      VKPTC_BCUDA(b, LaunchBatchLoopIteration(b->d_jobs.ptr, njobs, total, LP, bl, lg, 0, b->d_ctr.ptr, b->d_err.ptr,
                                              timing ? b->marks : nullptr),
                  "loop iteration");
      uint32_t more = 0;
      VKPTC_BCUDA(b, cudaMemcpyAsync(&more, LP.ctl + kLoopCtlMore, sizeof(more), cudaMemcpyDeviceToHost, b->stream),
                  "loop condition");
      VKPTC_BCUDA(b, cudaStreamSynchronize(b->stream), "loop sync");
      if (timing) {
        for (int i = 0; i < 5; ++i) {
          float m = 0.0f;
          cudaEventElapsedTime(&m, b->marks[i], b->marks[i + 1]);
          stage_ms[kLoopMarkStage[i]] += m;
        }
      }
      if (!more) break;
    }
    for (int i = 0; i < 5; ++i) b->stats.stage_ms[i] = stage_ms[i];
    rc = epilogue();
    if (rc != VKPTC_OK) return rc;
    VKPTC_BCUDA(b, cudaEventRecord(b->ev1, b->stream), "event");
  }
  VKPTC_BCUDA(b, cudaStreamSynchronize(b->stream), "batch sync");
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, b->ev0, b->ev1);
  uint32_t err = 0;
  VKPTC_BCUDA(b, cudaMemcpy(&err, b->d_err.ptr, sizeof(err), cudaMemcpyDeviceToHost), "error word");
  if (err & 2u) return bfail(b, VKPTC_TIMEOUT, "persistent batch: a grid barrier wait exceeded its bound");
  if (err) return bfail(b, VKPTC_INTERNAL_ERROR, "device traversal stack overflow");
  DevCounters dc{};
  VKPTC_BCUDA(b, cudaMemcpy(&dc, b->d_ctr.ptr, sizeof(dc), cudaMemcpyDeviceToHost), "counters");
  uint32_t iterations = 0;
  VKPTC_BCUDA(b, cudaMemcpy(&iterations, loop ? LP.ctl + kLoopCtlIterations : P.ctl + kBatchCtlIterations,
                            sizeof(iterations), cudaMemcpyDeviceToHost),
              "iterations");
  b->stats.segments = dc.rays;
  b->stats.shadow_rays = dc.shadow_tests;
  b->stats.ext_rays = dc.ext_rays;
  b->stats.ext_nodes = dc.nodes;
  b->stats.ext_tris = dc.tris;
  b->stats.shadow_queries = dc.shadow_rays;
  b->stats.shadow_nodes = dc.shadow_nodes;
  b->stats.shadow_tris = dc.shadow_tris;
  b->stats.device_ms = ms;
  // init, then one persistent kernel or the loop's stage kernels per iteration (regen, extend,
  // shadow, drain, shade, decide; the two SDF stages when a job has SDF primitives), then
  // accumulate per job
  b->stats.kernel_launches = 1u + (loop ? (bl.sdf ? 8ull : 6ull) * iterations : 1ull) +
                             static_cast<uint64_t>(table.size());
  b->stats.iterations = iterations;
  b->stats.graph_used = graph_used ? 1u : 0u;
  b->stats.grid = static_cast<uint32_t>(bl.grid);
  b->stats.block = static_cast<uint32_t>(bl.block);
  b->stats.pool_paths = cap;
  b->stats.stack_depth = static_cast<uint32_t>(bl.smem_entries);
  b->stats.steps = static_cast<uint32_t>(bl.steps);
  return VKPTC_OK;
}

}  // namespace

extern "C" {

int32_t vkptc_batch_create(const vkptc_config* config, vkptc_batch** out_batch) {
  if (!out_batch) return VKPTC_INVALID_ARGUMENT;
  *out_batch = nullptr;
  auto* b = new (std::nothrow) vkptc_batch();
  if (!b) return VKPTC_ALLOC_FAILED;
  if (config) b->config = *config;
  if (b->config.triangle_test > VKPTC_TRIANGLE_WATERTIGHT) {
    delete b;
    return VKPTC_INVALID_ARGUMENT;
  }
  b->device = b->config.device;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    delete b;
    return VKPTC_UNSUPPORTED;
  }
  if (b->device < 0 || b->device >= count) {
    delete b;
    return VKPTC_INVALID_ARGUMENT;
  }
  if (cudaSetDevice(b->device) != cudaSuccess || cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess ||
      b->d_ctr.alloc(1) != cudaSuccess || b->d_err.alloc(1) != cudaSuccess) {
    delete b;
    return VKPTC_INTERNAL_ERROR;
  }
  cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, b->device);
  *out_batch = b;
  return VKPTC_OK;
}

int32_t vkptc_batch_destroy(vkptc_batch* b) {
  if (!b) return VKPTC_INVALID_ARGUMENT;
  cudaSetDevice(b->device);
  cudaStreamSynchronize(b->stream);
  release_graph(b);
  for (vkptc_ctx* c : b->jobs) vkptc_destroy(c);
  b->jobs.clear();
  cudaStream_t st = b->stream, bs = b->body_stream, ss = b->side_stream;
  cudaEvent_t marks[6];
  std::copy(std::begin(b->marks), std::end(b->marks), marks);
  cudaEvent_t e0 = b->ev0, e1 = b->ev1, f0 = b->fork_ev[0], f1 = b->fork_ev[1];
  delete b;
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (f0) cudaEventDestroy(f0);
  if (f1) cudaEventDestroy(f1);
  if (st) cudaStreamDestroy(st);
  if (bs) cudaStreamDestroy(bs);
  if (ss) cudaStreamDestroy(ss);
  for (cudaEvent_t e : marks)
    if (e) cudaEventDestroy(e);
  return VKPTC_OK;
}

int32_t vkptc_batch_add_job(vkptc_batch* b, const vkptc_scene_view* scene, const vkptc_render_settings* settings,
                            uint32_t* job_id) {
  if (!b) return VKPTC_INVALID_ARGUMENT;
  if (!scene || !settings) return bfail(b, VKPTC_INVALID_ARGUMENT, "scene or settings is null");
  cudaSetDevice(b->device);
  vkptc_ctx* c = nullptr;
  int32_t rc = vkptc_create(&b->config, &c);
  if (rc != VKPTC_OK) return bfail(b, rc, "job context creation failed");
  if ((rc = vkptc_configure(c, settings)) != VKPTC_OK || (rc = vkptc_load_scene(c, scene)) != VKPTC_OK ||
      (rc = vkptc_build_acceleration(c)) != VKPTC_OK) {
    b->last_error = std::string("job set-up failed: ") + c->last_error;
    vkptc_destroy(c);
    return rc;
  }
  if (c->has_transmissive) {
    vkptc_destroy(c);
    return bfail(b, VKPTC_UNSUPPORTED, "batched jobs with transmissive materials are not supported");
  }
  b->jobs.push_back(c);
  release_graph(b);
  if (job_id) *job_id = static_cast<uint32_t>(b->jobs.size() - 1);
  b->last_error.clear();
  return VKPTC_OK;
}

int32_t vkptc_batch_run(vkptc_batch* b, uint32_t mode, const vkptc_batch_tuning* tuning) {
  if (!b) return VKPTC_INVALID_ARGUMENT;
  if (b->jobs.empty()) return bfail(b, VKPTC_NOT_READY, "batch has no jobs");
  if (mode > VKPTC_BATCH_LOOP) return bfail(b, VKPTC_INVALID_ARGUMENT, "unknown batch mode");
  cudaSetDevice(b->device);
  vkptc_batch_tuning t{};
  if (tuning) t = *tuning;
  b->stats = vkptc_batch_stats{};
  b->stats.jobs = static_cast<uint32_t>(b->jobs.size());
  for (vkptc_ctx* c : b->jobs) {
    b->stats.paths += static_cast<uint64_t>(c->settings.width) * c->settings.height * job_samples(c, t.sample_limit);
  }
  const int32_t rc = mode == VKPTC_BATCH_PLAIN ? batch_run_plain(b, t) : batch_run_pool(b, t, mode);
  if (rc == VKPTC_OK) b->last_error.clear();
  return rc;
}

int32_t vkptc_batch_read_film(vkptc_batch* b, uint32_t job_id, float* sum_rgb, uint32_t* count) {
  if (!b) return VKPTC_INVALID_ARGUMENT;
  if (job_id >= b->jobs.size()) return bfail(b, VKPTC_INVALID_ARGUMENT, "job id out of range");
  const int32_t rc = vkptc_read_film(b->jobs[job_id], sum_rgb, count, nullptr);
  if (rc != VKPTC_OK) b->last_error = b->jobs[job_id]->last_error;
  return rc;
}

int32_t vkptc_batch_read_films(vkptc_batch* b, float* const* sums, uint32_t* const* counts) {
  if (!b) return VKPTC_INVALID_ARGUMENT;
  cudaSetDevice(b->device);
  for (size_t j = 0; j < b->jobs.size(); ++j) {
    vkptc_ctx* c = b->jobs[j];
    const int32_t rc = enqueue_film_read(c, b->stream, sums ? sums[j] : nullptr, counts ? counts[j] : nullptr);
    if (rc != VKPTC_OK) {
      b->last_error = c->last_error;
      return rc;
    }
  }
  VKPTC_BCUDA(b, cudaStreamSynchronize(b->stream), "film read");
  b->last_error.clear();
  return VKPTC_OK;
}

int32_t vkptc_batch_get_stats(vkptc_batch* b, vkptc_batch_stats* out) {
  if (!b || !out) return VKPTC_INVALID_ARGUMENT;
  *out = b->stats;
  return VKPTC_OK;
}

const char* vkptc_batch_last_error(vkptc_batch* b) {
  if (!b) return "null batch";
  return b->last_error.c_str();
}

}  // extern "C"

// ============================================================ allocation-free
namespace {

template <typename T>
T* carve(unsigned char*& cursor, size_t count) {
  T* p = reinterpret_cast<T*>(cursor);
  cursor += (count * sizeof(T) + 255) / 256 * 256;
  return p;
}

}  // namespace

extern "C" int32_t vkptc_render_tile_noalloc(vkptc_ctx* ctx, const vkptc_tile* tile, uint32_t frame,
                                             float* d_film_sum, uint32_t* d_film_count, void* stream) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  if (!ctx->configured || !ctx->has_scene || !ctx->accel_valid) {
    return fail(ctx, VKPTC_NOT_READY, "render_tile_noalloc requires a configured tracer with a scene and a built acceleration structure");
  }
  if (!tile || !d_film_sum || !d_film_count) return fail(ctx, VKPTC_INVALID_ARGUMENT, "tile or film pointer is null");
  if ((reinterpret_cast<uintptr_t>(d_film_sum) & 15u) != 0u) {
    return fail(ctx, VKPTC_INVALID_ARGUMENT, "d_film_sum must be 16-byte aligned (float4 per pixel)");
  }
  const uint32_t x0 = std::min(tile->x, ctx->settings.width), y0 = std::min(tile->y, ctx->settings.height);
  const uint32_t x1 = static_cast<uint32_t>(std::min<uint64_t>(ctx->settings.width, static_cast<uint64_t>(x0) + tile->width));
  const uint32_t y1 = static_cast<uint32_t>(std::min<uint64_t>(ctx->settings.height, static_cast<uint64_t>(y0) + tile->height));
  if (x0 >= x1 || y0 >= y1) return VKPTC_OK;
  const uint64_t paths = static_cast<uint64_t>(x1 - x0) * (y1 - y0);
  if (paths > VKPTC_NOALLOC_MAX_PATHS) {
    return fail(ctx, VKPTC_INVALID_ARGUMENT,
                "tile of " + std::to_string(paths) + " pixels exceeds the allocation-free limit of " +
                    std::to_string(VKPTC_NOALLOC_MAX_PATHS) + " paths per call; split it into smaller tiles");
  }
  if (!ctx->noalloc_scratch) {
    return fail(ctx, VKPTC_INTERNAL_ERROR, std::string("the allocation-free scratch has no device address: "
                                                       "cudaGetSymbolAddress failed when the context was created: ") +
                                               cudaGetErrorString(ctx->noalloc_lookup));
  }
  const DeviceGuard guard(ctx->device);   // the caller's current device is restored on return
  unsigned char* const base = ctx->noalloc_scratch;
  const size_t n = VKPTC_NOALLOC_MAX_PATHS;
  unsigned char* cur = base;
  WaveState w{};
  w.ray_o = carve<float4>(cur, n);
  w.ray_d = carve<float4>(cur, n);
  w.thr = carve<float4>(cur, n);
  w.rad = carve<float4>(cur, n);
  w.sh_o = carve<float4>(cur, n);
  w.sh_d = carve<float4>(cur, n);
  w.sh_c = carve<float4>(cur, n);
  w.rng = carve<uint64_t>(cur, n);
  w.hit = carve<float2>(cur, n);
  w.q[0] = carve<uint32_t>(cur, n);
  w.q[1] = carve<uint32_t>(cur, n);
  w.sh_path = carve<uint32_t>(cur, n);
  w.counts = carve<uint32_t>(cur, 8);   // set by the raygen stage of every call
  w.capacity = VKPTC_NOALLOC_MAX_PATHS;
  if (static_cast<size_t>(cur - base) > kNoAllocBytes) return fail(ctx, VKPTC_INTERNAL_ERROR, "scratch layout overflow");
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  // The whole traversal stack in shared memory (no spill buffer, which would
  // be an allocation): a BVH whose worst-case stack does not fit is refused
  // with VKPTC_UNSUPPORTED by launch_shape.
  LaunchShape ls;
  int32_t rc = launch_shape(ctx, st, ls, /*allow_spill=*/false);
  if (rc != VKPTC_OK) return rc;
  Film film{};
  film.sum = reinterpret_cast<float4*>(d_film_sum);
  film.count = d_film_count;
  film.invalid = nullptr;
  film.width = ctx->settings.width;
  film.height = ctx->settings.height;
  const WaveTile wt{x0, y0, x1 - x0, y1 - y0, tile->sample_index, 1u};
  bool ordered = false;
  rc = order_begin(ctx, st, &ordered);
  if (rc != VKPTC_OK) return rc;
  VKPTC_CUDA(ctx, LaunchWave(dev_scene(ctx), dev_settings(ctx, frame), w, wt, film, ctx->config.math_mode == 0u,
                             ctx->config.collect_stats != 0u, ls, ctx->d_ctr.ptr, ctx->d_err.ptr, nullptr),
             "allocation-free wave launch");
  rc = order_end(ctx, st, ordered);
  if (rc != VKPTC_OK) return rc;
  ctx->last_error.clear();
  return VKPTC_OK;
}

// ============================================================ adjoint
namespace {

// The supported material subset (Lambertian / Phong-lobe glossy, optionally
// emissive); returns an empty string when material m qualifies.
std::string adjoint_material_issue(const float* m, size_t i) {
  const uint32_t model = static_cast<uint32_t>(m[7] + 0.5f);
  const float rough = std::isfinite(m[6]) ? std::min(1.0f, std::max(0.0f, m[6])) : 0.0f;
  std::string why;
  if (model != 0u && model != 1u && model != 3u) why = "model " + std::to_string(model);
  else if (m[8] > 0.65f) why = "metallic";
  else if (m[10] > 0.05f) why = "transmissive";
  else if (m[11] > 0.05f) why = "clear coat";
  else if (rough <= 0.001f) why = "mirror (roughness <= 0.001)";
  else if ((static_cast<uint32_t>(m[15] + 0.5f) & 1023u) != 0u) why = "a procedural effect";
  if (why.empty()) return why;
  return "material " + std::to_string(i) + " is " + why + "; the adjoint supports Lambertian and Phong-lobe glossy "
         "materials (models 0, 1, 3) without procedural effects only";
}

// Material table with the 7 parameters of each material substituted.
void apply_params(const std::vector<float>& base, const float* params, std::vector<float>& out) {
  out = base;
  const size_t n = base.size() / 16;
  for (size_t i = 0; i < n; ++i) {
    const float* p = params + VKPTC_ADJ_PARAMS_PER_MATERIAL * i;
    float* m = &out[16 * i];
    m[0] = p[0];
    m[1] = p[1];
    m[2] = p[2];
    m[6] = p[3];
    m[3] = p[4];
    m[4] = p[5];
    m[5] = p[6];
  }
}

AdjLaunch adj_launch(vkptc_ctx* c, bool backward, int32_t& rc) {
  AdjLaunch l{};
  rc = VKPTC_OK;
  l.block = 128;
  l.stack_cap = stack_cap(c);
  l.spp = c->adj.desc.spp;
  l.first_sample = c->adj.desc.first_sample;
  l.parity = c->config.math_mode == 0u;
  l.stream = c->stream;
  const uint32_t mats = static_cast<uint32_t>(c->materials.size() / 16);
  const size_t smem = backward ? AdjBackwardSmem(l.block, l.stack_cap, mats) : AdjForwardSmem(l.block, l.stack_cap);
  int max_optin = 0;
  cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
  if (smem > static_cast<size_t>(max_optin)) {
    rc = fail(c, VKPTC_UNSUPPORTED, "adjoint: traversal stack and gradient slots do not fit in shared memory");
    return l;
  }
  if (smem > 48 * 1024) {
    const cudaError_t e = ConfigureAdjSmem(smem);
    if (e != cudaSuccess) {
      rc = cuda_fail(c, e, "adjoint shared memory limit");
      return l;
    }
  }
  l.grid = c->sm_count * AdjBlocksPerSm(backward ? AdjKernel::kReplay : AdjKernel::kForward, l.block,
                                         backward ? AdjForwardSmem(l.block, l.stack_cap) : smem, l.parity);
  l.grid_reverse = c->sm_count * AdjBlocksPerSm(AdjKernel::kReverse, l.block, AdjReverseSmem(l.block, mats), l.parity);
  return l;
}

DevScene adj_scene(vkptc_ctx* c) {
  DevScene s = dev_scene(c);
  s.materials = c->adj.mat.ptr;
  return s;
}

}  // namespace

extern "C" {

int32_t vkptc_adjoint_setup(vkptc_ctx* ctx, const vkptc_adjoint_desc* desc, const float* target_rgb,
                            uint64_t target_floats) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  if (!desc) return fail(ctx, VKPTC_INVALID_ARGUMENT, "desc is null");
  if (!ctx->configured || !ctx->has_scene || !ctx->accel_valid) {
    return fail(ctx, VKPTC_NOT_READY, "adjoint requires a configured tracer with a scene and a built acceleration structure");
  }
  if (desc->spp == 0u) return fail(ctx, VKPTC_INVALID_ARGUMENT, "spp must be positive");
  if (ctx->config.triangle_test != VKPTC_TRIANGLE_MT)
    return fail(ctx, VKPTC_UNSUPPORTED, "the adjoint uses the Moller-Trumbore triangle test");
  if (ctx->settings.max_depth > VKPTC_ADJ_MAX_DEPTH) {
    return fail(ctx, VKPTC_UNSUPPORTED, "adjoint supports max_depth <= " + std::to_string(VKPTC_ADJ_MAX_DEPTH));
  }
  const size_t mats = ctx->materials.size() / 16;
  if (mats > VKPTC_ADJ_MAX_MATERIALS) {
    return fail(ctx, VKPTC_UNSUPPORTED, "adjoint supports at most " + std::to_string(VKPTC_ADJ_MAX_MATERIALS) + " materials");
  }
  for (size_t i = 0; i < mats; ++i) {
    const std::string why = adjoint_material_issue(&ctx->materials[16 * i], i);
    if (!why.empty()) return fail(ctx, VKPTC_UNSUPPORTED, why);
  }
  if (ctx->has_transmissive) return fail(ctx, VKPTC_UNSUPPORTED, "adjoint: transmissive materials are not supported");
  if (ctx->env_w) return fail(ctx, VKPTC_UNSUPPORTED, "adjoint: environment maps are not supported");
  if (ctx->sdf_count) return fail(ctx, VKPTC_UNSUPPORTED, "adjoint: SDF primitives are not supported");
  const uint64_t npx = static_cast<uint64_t>(ctx->settings.width) * ctx->settings.height;
  if (npx == 0) return fail(ctx, VKPTC_INVALID_ARGUMENT, "empty film");
  if (target_rgb && target_floats != 3 * npx) {
    return fail(ctx, VKPTC_INVALID_ARGUMENT, "target must hold W*H*3 floats");
  }
  const uint64_t paths = npx * desc->spp;
  if (paths > (1ull << 31)) return fail(ctx, VKPTC_INVALID_ARGUMENT, "more than 2^31 paths per forward");
  cudaSetDevice(ctx->device);
  AdjointState& a = ctx->adj;
  VKPTC_CUDA(ctx, a.rad.alloc(paths), "adjoint radiance alloc");
  VKPTC_CUDA(ctx, a.adj.alloc(npx), "adjoint alloc");
  VKPTC_CUDA(ctx, a.image.alloc(3 * npx), "adjoint image alloc");
  VKPTC_CUDA(ctx, a.mat.alloc(ctx->materials.size()), "adjoint material alloc");
  VKPTC_CUDA(ctx, a.mat0.alloc(ctx->materials.size()), "adjoint material alloc");
  a.loss_grid = static_cast<int>(std::min<uint64_t>(1024, (npx + 255) / 256));
  VKPTC_CUDA(ctx, a.loss_part.alloc(a.loss_grid), "adjoint loss alloc");
  VKPTC_CUDA(ctx, a.loss.alloc(1), "adjoint loss alloc");
  if (target_rgb) {
    VKPTC_CUDA(ctx, a.target.alloc(3 * npx), "adjoint target alloc");
    VKPTC_CUDA(ctx, cudaMemcpy(a.target.ptr, target_rgb, 3 * npx * sizeof(float), cudaMemcpyHostToDevice), "target upload");
  }
  for (auto& e : a.ev)
    if (!e) VKPTC_CUDA(ctx, cudaEventCreate(&e), "adjoint events");
  a.desc = *desc;
  a.width = ctx->settings.width;
  a.height = ctx->settings.height;
  a.has_target = target_rgb != nullptr;
  a.setup = true;
  a.forward_done = false;
  a.recorded = false;
  a.stats = vkptc_adjoint_stats{};
  a.stats.paths = paths;
  ctx->last_error.clear();
  return VKPTC_OK;
}

int32_t vkptc_forward(vkptc_ctx* ctx, const float* params, uint32_t param_count, const float* rr_params, double* loss,
                      float* image_rgb) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  AdjointState& a = ctx->adj;
  if (!a.setup || a.width != ctx->settings.width || a.height != ctx->settings.height || !ctx->accel_valid) {
    return fail(ctx, VKPTC_NOT_READY, "vkptc_adjoint_setup must run (again) before vkptc_forward");
  }
  const size_t mats = ctx->materials.size() / 16;
  if (!params || param_count != VKPTC_ADJ_PARAMS_PER_MATERIAL * mats) {
    return fail(ctx, VKPTC_INVALID_ARGUMENT, "params must hold 7 floats per material (" +
                                                 std::to_string(VKPTC_ADJ_PARAMS_PER_MATERIAL * mats) + ")");
  }
  apply_params(ctx->materials, params, a.host_mat);
  apply_params(ctx->materials, rr_params ? rr_params : params, a.host_mat0);
  for (size_t i = 0; i < mats; ++i) {
    const std::string why = adjoint_material_issue(&a.host_mat[16 * i], i);
    if (!why.empty()) return fail(ctx, VKPTC_UNSUPPORTED, why);
  }
  cudaSetDevice(ctx->device);
  const size_t bytes = a.host_mat.size() * sizeof(float);
  VKPTC_CUDA(ctx, cudaMemcpyAsync(a.mat.ptr, a.host_mat.data(), bytes, cudaMemcpyHostToDevice, ctx->stream), "params upload");
  VKPTC_CUDA(ctx, cudaMemcpyAsync(a.mat0.ptr, a.host_mat0.data(), bytes, cudaMemcpyHostToDevice, ctx->stream), "params upload");
  int32_t rc = VKPTC_OK;
  const AdjLaunch l = adj_launch(ctx, false, rc);
  if (rc != VKPTC_OK) return rc;
  VKPTC_CUDA(ctx, cudaMemsetAsync(ctx->d_err.ptr, 0, sizeof(uint32_t), ctx->stream), "error clear");
  const DevSettings st = dev_settings(ctx, a.desc.frame);
  // With the backward replaying the forward's own paths and all of them one
  // chunk, the forward writes the vertex records itself and the backward
  // skips the replay (the same records, so the same gradient).
  const bool record = !(a.desc.flags & VKPTC_ADJ_DECORRELATED) && a.stats.paths <= kAdjChunkPaths;
  a.recorded = false;
  if (record) {
    VKPTC_CUDA(ctx, a.recs.alloc(std::max<size_t>(1, a.stats.paths * kAdjVertexSlots * kAdjRecordFloat4s)),
               "adjoint record alloc");
    VKPTC_CUDA(ctx, a.fwd_nrec.alloc(std::max<size_t>(1, a.stats.paths)), "adjoint record alloc");
  }
  VKPTC_CUDA(ctx, cudaEventRecord(a.ev[0], ctx->stream), "event");
  VKPTC_CUDA(ctx, LaunchAdjForward(adj_scene(ctx), st, a.mat0.ptr, l, a.rad.ptr, ctx->d_err.ptr,
                                   record ? a.recs.ptr : nullptr, record ? a.fwd_nrec.ptr : nullptr),
             "adjoint forward launch");
  VKPTC_CUDA(ctx, LaunchAdjLoss(st, a.desc.spp, a.rad.ptr, a.has_target ? a.target.ptr : nullptr, a.image.ptr, a.adj.ptr,
                                a.loss_part.ptr, a.loss.ptr, a.loss_grid, ctx->stream),
             "adjoint loss launch");
  VKPTC_CUDA(ctx, cudaEventRecord(a.ev[1], ctx->stream), "event");
  double host_loss = 0.0;
  VKPTC_CUDA(ctx, cudaMemcpyAsync(&host_loss, a.loss.ptr, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "loss readback");
  if (image_rgb) {
    VKPTC_CUDA(ctx, cudaMemcpyAsync(image_rgb, a.image.ptr, a.image.count * sizeof(float), cudaMemcpyDeviceToHost,
                                    ctx->stream), "image readback");
  }
  rc = check_device_error(ctx);
  if (rc != VKPTC_OK) return rc;
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, a.ev[0], a.ev[1]);
  a.stats.forward_ms = ms;
  a.stats.forwards++;
  a.stats.forward_grid = static_cast<uint32_t>(l.grid);
  a.stats.block = static_cast<uint32_t>(l.block);
  if (loss) *loss = host_loss;
  a.forward_done = true;
  a.recorded = record;
  ctx->last_error.clear();
  return VKPTC_OK;
}

int32_t vkptc_backward(vkptc_ctx* ctx, float* grad, uint32_t param_count) {
  return vkptc_backward_weighted(ctx, nullptr, grad, param_count);
}

int32_t vkptc_backward_weighted(vkptc_ctx* ctx, const float* path_weight, float* grad, uint32_t param_count) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  AdjointState& a = ctx->adj;
  if (!a.setup || !a.forward_done || !ctx->accel_valid) return fail(ctx, VKPTC_NOT_READY, "vkptc_backward needs a vkptc_forward first");
  const size_t mats = ctx->materials.size() / 16;
  const size_t stride = VKPTC_ADJ_PARAMS_PER_MATERIAL * mats;
  if (!grad || param_count != stride) {
    return fail(ctx, VKPTC_INVALID_ARGUMENT, "grad must hold 7 floats per material (" + std::to_string(stride) + ")");
  }
  cudaSetDevice(ctx->device);
  int32_t rc = VKPTC_OK;
  const AdjLaunch l = adj_launch(ctx, true, rc);
  if (rc != VKPTC_OK) return rc;
  VKPTC_CUDA(ctx, a.grad_part.alloc(static_cast<size_t>(l.grid_reverse) * stride), "gradient partials alloc");
  const size_t chunk = static_cast<size_t>(std::min<uint64_t>(kAdjChunkPaths, a.stats.paths));
  VKPTC_CUDA(ctx, a.recs.alloc(std::max<size_t>(1, chunk * kAdjVertexSlots * kAdjRecordFloat4s)),
             "adjoint record alloc");
  VKPTC_CUDA(ctx, a.gout.alloc(std::max<size_t>(1, chunk)), "adjoint record alloc");
  VKPTC_CUDA(ctx, a.grad.alloc(stride), "gradient alloc");
  if (path_weight) {
    VKPTC_CUDA(ctx, a.path_weight.alloc(a.stats.paths), "path weight alloc");
    VKPTC_CUDA(ctx, cudaMemcpyAsync(a.path_weight.ptr, path_weight, a.stats.paths * sizeof(float), cudaMemcpyHostToDevice,
                                    ctx->stream), "path weight upload");
  }
  VKPTC_CUDA(ctx, cudaMemsetAsync(ctx->d_err.ptr, 0, sizeof(uint32_t), ctx->stream), "error clear");
  VKPTC_CUDA(ctx, cudaEventRecord(a.ev[2], ctx->stream), "event");
  const uint32_t replay_frame = (a.desc.flags & VKPTC_ADJ_DECORRELATED) ? a.desc.backward_frame : a.desc.frame;
  const bool use_records = a.recorded && !(a.desc.flags & VKPTC_ADJ_DECORRELATED);
  VKPTC_CUDA(ctx, LaunchAdjBackward(adj_scene(ctx), dev_settings(ctx, replay_frame), a.mat0.ptr, l, a.adj.ptr,
                                    path_weight ? a.path_weight.ptr : nullptr, a.recs.ptr, a.gout.ptr,
                                    a.grad_part.ptr, a.grad.ptr, ctx->d_err.ptr, use_records ? a.rad.ptr : nullptr,
                                    use_records ? a.fwd_nrec.ptr : nullptr),
             "adjoint backward launch");
  VKPTC_CUDA(ctx, cudaEventRecord(a.ev[3], ctx->stream), "event");
  VKPTC_CUDA(ctx, cudaMemcpyAsync(grad, a.grad.ptr, stride * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream),
             "gradient readback");
  rc = check_device_error(ctx);
  if (rc != VKPTC_OK) return rc;
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, a.ev[2], a.ev[3]);
  a.stats.backward_ms = ms;
  a.stats.backwards++;
  a.stats.backward_grid = static_cast<uint32_t>(l.grid);
  ctx->last_error.clear();
  return VKPTC_OK;
}

int32_t vkptc_adjoint_set_frames(vkptc_ctx* ctx, uint32_t frame, uint32_t backward_frame) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  if (!ctx->adj.setup) return fail(ctx, VKPTC_NOT_READY, "vkptc_adjoint_setup must run first");
  ctx->adj.desc.frame = frame;
  ctx->adj.desc.backward_frame = backward_frame;
  ctx->adj.forward_done = false;
  return VKPTC_OK;
}

int32_t vkptc_adjoint_read_samples(vkptc_ctx* ctx, float* rgb, uint32_t* signature) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  AdjointState& a = ctx->adj;
  if (!a.setup || !a.forward_done) return fail(ctx, VKPTC_NOT_READY, "no forward to read");
  if (!rgb && !signature) return VKPTC_OK;
  cudaSetDevice(ctx->device);
  std::vector<float4> host(a.stats.paths);
  VKPTC_CUDA(ctx, cudaMemcpy(host.data(), a.rad.ptr, host.size() * sizeof(float4), cudaMemcpyDeviceToHost),
             "sample readback");
  for (size_t j = 0; j < host.size(); ++j) {
    if (rgb) {
      rgb[3 * j + 0] = host[j].x;
      rgb[3 * j + 1] = host[j].y;
      rgb[3 * j + 2] = host[j].z;
    }
    if (signature) std::memcpy(&signature[j], &host[j].w, sizeof(uint32_t));
  }
  return VKPTC_OK;
}

int32_t vkptc_adjoint_get_stats(vkptc_ctx* ctx, vkptc_adjoint_stats* out) {
  if (!ctx) return VKPTC_INVALID_ARGUMENT;
  if (!out) return fail(ctx, VKPTC_INVALID_ARGUMENT, "out is null");
  *out = ctx->adj.stats;
  return VKPTC_OK;
}

}  // extern "C"
