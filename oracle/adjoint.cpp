// adjoint.cpp -- FP64 forward-mode adjoint of the render path.
//
// TEST INFRASTRUCTURE ONLY (see vkpt_adjoint.h): the checker of the GPU
// forward/backward pair, never part of the product.
//
// A double-precision restatement of the reference's trace loop with every
// continuous quantity carried as a dual number whose tangents are the
// requested material parameters.  Cited reference lines:
//   camera_rays / shade_pixel   src/pathtracer/ScalarCpuPathTracer.Render.cpp:55-119, 228-284
//   trace                       src/pathtracer/ScalarCpuPathTracer.cpp:1148-1289
//   sample_direct_light         src/pathtracer/ScalarCpuPathTracer.cpp:1022-1118
//   light_pdf / MisWeight       src/pathtracer/ScalarCpuPathTracer.cpp:1120-1146
//   hemisphere / Phong lobe     src/pathtracer/ScalarCpuPathTracer.cpp:978-1020
//   Rng / splitmix64            src/pathtracer/ScalarCpuPathTracer.cpp:36-41, 383-393
//   Moller-Trumbore             src/cpu/BvhTriangleIntersector.cpp:35-74
//   film add / resolve          src/pathtracer/FilmBuffer.cpp:80-91, 160-214
#include "vkpt_adjoint.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace {

constexpr int kMaxT = static_cast<int>(VKO_ADJ_MAX_TANGENTS);
constexpr double kEps = 1e-4;
constexpr double kPi = 3.14159265358979323846;
thread_local int NT = 0;   // tangents in use
std::string g_error;

// ------------------------------------------------------------ dual numbers
struct D {
  double v;
  double g[kMaxT];
  D() : v(0.0) { std::fill(g, g + NT, 0.0); }
  D(double x) : v(x) { std::fill(g, g + NT, 0.0); }  // NOLINT: implicit constants
};
D operator+(const D& a, const D& b) {
  D r(a.v + b.v);
  for (int i = 0; i < NT; ++i) r.g[i] = a.g[i] + b.g[i];
  return r;
}
D operator-(const D& a, const D& b) {
  D r(a.v - b.v);
  for (int i = 0; i < NT; ++i) r.g[i] = a.g[i] - b.g[i];
  return r;
}
D operator-(const D& a) {
  D r(-a.v);
  for (int i = 0; i < NT; ++i) r.g[i] = -a.g[i];
  return r;
}
D operator*(const D& a, const D& b) {
  D r(a.v * b.v);
  for (int i = 0; i < NT; ++i) r.g[i] = a.g[i] * b.v + a.v * b.g[i];
  return r;
}
D operator/(const D& a, const D& b) {
  D r(a.v / b.v);
  for (int i = 0; i < NT; ++i) r.g[i] = (a.g[i] - r.v * b.g[i]) / b.v;
  return r;
}
D dsqrt(const D& a) {
  D r(std::sqrt(a.v));
  const double s = r.v > 0.0 ? 0.5 / r.v : 0.0;
  for (int i = 0; i < NT; ++i) r.g[i] = a.g[i] * s;
  return r;
}
D dpow(const D& x, const D& y) {
  D r(std::pow(x.v, y.v));
  if (!(x.v > 0.0)) {
    for (int i = 0; i < NT; ++i) r.g[i] = 0.0;
    return r;
  }
  const double a = r.v * y.v / x.v, b = r.v * std::log(x.v);
  for (int i = 0; i < NT; ++i) r.g[i] = a * x.g[i] + b * y.g[i];
  return r;
}
// std::max / std::min / std::clamp semantics on the primal values.
D dmax(const D& a, const D& b) { return (a.v < b.v) ? b : a; }
D dmin(const D& a, const D& b) { return (b.v < a.v) ? b : a; }
D dclamp(const D& v, double lo, double hi) { return (v.v < lo) ? D(lo) : ((hi < v.v) ? D(hi) : v); }
D dclamp01(const D& v) {
  if (!std::isfinite(v.v)) return D(0.0);
  return dmin(D(1.0), dmax(D(0.0), v));
}

struct V {
  D x, y, z;
};
V vk(double x, double y, double z) { return V{D(x), D(y), D(z)}; }
V operator+(const V& a, const V& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V operator-(const V& a, const V& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V operator*(const V& a, const D& s) { return {a.x * s, a.y * s, a.z * s}; }
V operator/(const V& a, const D& s) { return {a.x / s, a.y / s, a.z / s}; }
V vneg(const V& a) { return {-a.x, -a.y, -a.z}; }
V vmul(const V& a, const V& b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
D dot(const V& a, const V& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V cross(const V& a, const V& b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
V unit(const V& v) {
  const D l = dsqrt(dot(v, v));
  if (l.v <= kEps) return vk(0.0, 1.0, 0.0);
  return v / l;
}

// plain double vectors for geometry queries
struct P3 {
  double x, y, z;
};
P3 pv(const V& v) { return {v.x.v, v.y.v, v.z.v}; }
P3 psub(P3 a, P3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
double pdot(P3 a, P3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
P3 pcross(P3 a, P3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
P3 punit(P3 v) {
  const double l = std::sqrt(pdot(v, v));
  if (l <= kEps) return {0.0, 1.0, 0.0};
  return {v.x / l, v.y / l, v.z / l};
}
V vc(P3 p) { return vk(p.x, p.y, p.z); }

// ------------------------------------------------------------------ RNG
uint64_t mix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ULL;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}
struct Rng {
  uint64_t s;
  Rng(uint64_t seed, uint64_t frame, uint64_t sample, uint64_t path, uint64_t dim, uint64_t depth, uint64_t pixel) {
    const uint64_t m = mix64(seed ^ mix64(frame) ^ mix64(sample) ^ mix64(path) ^ mix64(dim) ^ mix64(depth));
    s = mix64(m + mix64(pixel));
  }
  float u() {
    s = mix64(s);
    return static_cast<float>(static_cast<uint32_t>((s >> 8) & 0x00ffffffu)) * (1.0f / 16777215.0f);
  }
};

// ------------------------------------------------------------------ scene
struct Tri {
  P3 v0, e1, e2, n;
  uint32_t mat;
};
struct Mat {
  V alb, le;
  P3 alb0;   // albedo that drives the roulette throughput
  D rough;
  uint32_t model;
  double metallic, clearcoat;
};
struct Light {
  P3 pos, color, dir;
  double intensity, radius, inner, outer;
};

struct World {
  std::vector<Tri> tris;
  std::vector<Mat> mats;      // dual parameters (tangents set per request)
  std::vector<Light> lights;
  P3 env{}, cam_pos{}, cam_fwd{}, cam_right{}, cam_up{};
  double tan_half = 0.0;
  float fov = 60.0f;
  double aperture = 0.0, focus = 0.0;
  uint32_t iris_blades = 0u;                 // lens shape (camera_rays' polygonal aperture)
  double iris_rotation = 0.0, iris_roundness = 1.0, squeeze = 1.0;

  bool hit(P3 o, P3 d, double tmax, double& t_out, int& idx) const {
    double best = tmax;
    idx = -1;
    for (size_t i = 0; i < tris.size(); ++i) {
      const Tri& tr = tris[i];
      const P3 h = pcross(d, tr.e2);
      const double det = pdot(tr.e1, h);
      if (std::fabs(det) < kEps) continue;
      const double inv = 1.0 / det;
      const P3 s = psub(o, tr.v0);
      const double u = pdot(s, h) * inv;
      if (u < 0.0 || u > 1.0) continue;
      const P3 q = pcross(s, tr.e1);
      const double v = pdot(d, q) * inv;
      if (v < 0.0 || u + v > 1.0) continue;
      const double t = pdot(tr.e2, q) * inv;
      if (t > kEps && t < best) {
        best = t;
        idx = static_cast<int>(i);
      }
    }
    t_out = best;
    return idx >= 0;
  }
};

struct Cfg {
  uint32_t width, height, max_depth, nee, mis, rr_start;
  double rr_min, rr_max;
  uint64_t seed;
  double clamp;
  uint32_t frame;
};

D mis(const D& a, const D& b) {
  const D a2 = a * a, b2 = b * b, den = a2 + b2;
  if (den.v <= 0.0) return D(1.0);
  return a2 / den;
}

D light_pdf(const World& w, const V& p, const V& dir) {
  D total(0.0);
  if (w.lights.empty()) return total;
  const double inv_n = 1.0 / static_cast<double>(w.lights.size());
  for (const Light& L : w.lights) {
    const V tl = vc(L.pos) - p;
    const D dist = dsqrt(dot(tl, tl));
    if (dist.v < kEps) continue;
    if (dot(tl / dist, dir).v > 0.9999) total = total + D(inv_n) / (dist * dist + D(kEps));
  }
  return total;
}

D spot(const Light& L, const V& from_light) {
  if (L.inner <= -0.999) return D(1.0);
  const D cone = dot(unit(from_light), vc(punit(L.dir)));
  if (cone.v <= L.outer) return D(0.0);
  if (cone.v >= L.inner || L.inner <= L.outer) return D(1.0);
  const D t = dclamp((cone - D(L.outer)) / D(L.inner - L.outer), 0.0, 1.0);
  return t * t * (D(3.0) - D(2.0) * t);
}

V hemisphere(Rng& r, P3 n) {
  const double u1 = r.u(), u2 = r.u();
  const double rr = std::sqrt(std::max(0.0, 1.0 - u1));
  const double phi = 2.0 * kPi * u2;
  const P3 loc{rr * std::cos(phi), rr * std::sin(phi), std::sqrt(std::max(0.0, u1))};
  const P3 ref = (std::fabs(n.z) < 0.999) ? P3{0.0, 0.0, 1.0} : P3{0.0, 1.0, 0.0};
  const P3 t = punit(pcross(ref, n));
  const P3 b = pcross(n, t);
  return vc(punit({t.x * loc.x + b.x * loc.y + n.x * loc.z, t.y * loc.x + b.y * loc.y + n.y * loc.z,
                   t.z * loc.x + b.z * loc.y + n.z * loc.z}));
}

V phong(Rng& r, const V& refl, const D& ex, P3 n, uint32_t& fl) {
  const double u1 = r.u(), u2 = r.u();
  const D ct = dpow(D(std::max(0.0, u1)), D(1.0) / (ex + D(1.0)));
  const D sn = dsqrt(dmax(D(0.0), D(1.0) - ct * ct));
  const double phi = 2.0 * kPi * u2;
  const bool alt = !(std::fabs(refl.z.v) < 0.999);
  if (alt) fl |= 8u;
  const V ref = alt ? vk(0.0, 1.0, 0.0) : vk(0.0, 0.0, 1.0);
  const V t = unit(cross(ref, refl));
  const V b = cross(refl, t);
  V out = unit(t * (sn * D(std::cos(phi))) + b * (sn * D(std::sin(phi))) + refl * ct);
  const V nn = vc(n);
  if (dot(out, nn).v <= 0.0) {
    fl |= 16u;
    out = out - nn * (D(2.0) * dot(out, nn));
    if (dot(out, nn).v <= 0.0) {
      fl |= 32u;
      return hemisphere(r, n);
    }
  }
  return out;
}

// One path; returns its radiance (dual).  sig receives a hash of the path's
// discrete decisions (hit triangles, visibility, lobe fallbacks, termination).
V trace_path(const World& w, const Cfg& c, uint32_t x, uint32_t y, uint32_t sample, uint64_t& sig) {
  const uint32_t W = c.width, H = c.height;
  const uint64_t sample_seed = (static_cast<uint64_t>(y) << 32) | x;
  const uint64_t path_id = sample_seed + sample + c.frame;
  Rng crng(c.seed, c.frame, sample, static_cast<uint32_t>(path_id), 0u, 0u, static_cast<uint64_t>(y) * W + x);
  const double fx = (static_cast<double>(x) + crng.u()) / static_cast<double>(std::max(1u, W));
  const double fy = (static_cast<double>(y) + crng.u()) / static_cast<double>(std::max(1u, H));
  const uint64_t cam_seed = static_cast<uint64_t>(crng.u() * static_cast<float>(0xffffu));
  const double aspect = static_cast<double>(W) / std::max(1.0, static_cast<double>(H));
  const double nx = (2.0 * fx - 1.0) * aspect * w.tan_half;
  const double ny = (1.0 - 2.0 * fy) * w.tan_half;
  P3 dir = punit({w.cam_fwd.x + w.cam_right.x * nx + w.cam_up.x * ny, w.cam_fwd.y + w.cam_right.y * nx + w.cam_up.y * ny,
                  w.cam_fwd.z + w.cam_right.z * nx + w.cam_up.z * ny});
  P3 org = w.cam_pos;
  if (w.aperture > 0.0 && w.focus > kEps) {
    const double lr = std::sqrt(static_cast<double>(crng.u()));
    const double lphi = 2.0 * kPi * crng.u();
    double boundary = 1.0;
    if (w.iris_blades >= 3u && w.iris_roundness < 0.999) {
      const double sector = 2.0 * kPi / static_cast<double>(w.iris_blades);
      const double local_phi = lphi - w.iris_rotation;
      const double wrapped = local_phi - sector * std::floor(local_phi / sector);
      const double centered = wrapped > sector * 0.5 ? wrapped - sector : wrapped;
      const double polygon = std::cos(sector * 0.5) / std::max(0.1, std::cos(centered));
      boundary = polygon * (1.0 - w.iris_roundness) + w.iris_roundness;
    }
    const double rr = w.aperture * lr * boundary;
    const double rs = rr * w.squeeze;
    const P3 off{w.cam_right.x * rs * std::cos(lphi) + w.cam_up.x * rr * std::sin(lphi),
                 w.cam_right.y * rs * std::cos(lphi) + w.cam_up.y * rr * std::sin(lphi),
                 w.cam_right.z * rs * std::cos(lphi) + w.cam_up.z * rr * std::sin(lphi)};
    const P3 fp{w.cam_pos.x + dir.x * w.focus, w.cam_pos.y + dir.y * w.focus, w.cam_pos.z + dir.z * w.focus};
    org = {w.cam_pos.x + off.x, w.cam_pos.y + off.y, w.cam_pos.z + off.z};
    dir = punit(psub(fp, org));
  }
  Rng rng(c.seed + sample_seed + cam_seed, c.frame, sample, path_id, 0u, 0u, sample_seed);
  V o = vc(org), d = vc(dir);
  V thr = vk(1.0, 1.0, 1.0), rad = vk(0.0, 0.0, 0.0);
  P3 thr0{1.0, 1.0, 1.0};
  const double nl = static_cast<double>(w.lights.size());
  for (uint32_t depth = 0; depth < c.max_depth; ++depth) {
    double th;
    int ti;
    if (!w.hit(pv(o), pv(d), INFINITY, th, ti)) {
      rad = rad + vmul(thr, vc(w.env));
      sig = mix64(sig ^ 0xFFFFFFFFull);
      break;
    }
    const Tri& tr = w.tris[ti];
    // distance along d to the hit triangle's plane, as a function of (o, d)
    const V gn = vc(tr.n);
    const D t = dot(vc(tr.v0) - o, gn) / dot(d, gn);
    const V hp = o + d * t;
    const bool entering = dot(d, gn).v < 0.0;
    uint32_t fl = entering ? 1u : 0u;
    const P3 nvec = entering ? tr.n : P3{-tr.n.x, -tr.n.y, -tr.n.z};
    const V nrm = vc(nvec);
    const Mat& m = w.mats[std::min<size_t>(tr.mat, w.mats.size() - 1)];
    const V alb{dclamp(m.alb.x, 0.0, 1.5), dclamp(m.alb.y, 0.0, 1.5), dclamp(m.alb.z, 0.0, 1.5)};
    const D rough = dclamp01(m.rough);
    const bool emissive_model = m.model == 1u || m.le.x.v > 0.0 || m.le.y.v > 0.0 || m.le.z.v > 0.0;
    const bool diffuse = rough.v >= 0.999;

    if (!c.nee || depth == 0u) {
      rad = rad + vmul(thr, m.le);
    } else if (c.mis && emissive_model) {
      const D bp = dmax(D(0.0), dot(nrm, vneg(d))) * D(1.0 / kPi);
      const D lp = light_pdf(w, o, d);
      rad = rad + vmul(thr, m.le) * mis(bp, lp);
    }

    if (c.nee && depth + 1u < c.max_depth && !w.lights.empty()) {
      const uint32_t nli = static_cast<uint32_t>(w.lights.size());
      uint32_t pick = static_cast<uint32_t>(rng.u() * static_cast<float>(nli));
      if (pick > nli - 1u) pick = nli - 1u;
      const Light& L = w.lights[pick];
      P3 lpos = L.pos;
      if (L.radius > 1e-5) {
        const double uz = 1.0 - 2.0 * rng.u();
        const double r = std::sqrt(std::max(0.0, 1.0 - uz * uz));
        const double phi = 2.0 * kPi * rng.u();
        lpos = {lpos.x + r * std::cos(phi) * L.radius, lpos.y + uz * L.radius, lpos.z + r * std::sin(phi) * L.radius};
      }
      const V tl = vc(lpos) - hp;
      const D d2 = dot(tl, tl);
      const D dist = dsqrt(d2);
      bool valid = dist.v >= kEps;
      V ldir{}, acc = vk(0.0, 0.0, 0.0);
      D cth(0.0);
      if (valid) {
        ldir = tl / dist;
        cth = dot(nrm, ldir);
        valid = cth.v > 0.0;
      }
      D sf(0.0);
      if (valid) {
        sf = spot(L, vneg(ldir));
        valid = sf.v > 0.0;
      }
      if (valid) {
        const V irr = vc(L.color) * (D(L.intensity) * sf / (d2 + D(kEps)));
        acc = vmul(alb * D(1.0 / kPi), irr) * (cth * D(nl));
        if (rough.v < 0.65) {
          const V hv = unit(ldir + unit(vneg(d)));
          const D er = dmax(D(0.025), rough);
          const D a2 = er * er;
          const D pw = dclamp(D(2.0) / dmax(D(0.0005), a2 * a2) - D(2.0), 4.0, 96.0);
          const D spec = dpow(dmax(D(0.0), dot(nrm, hv)), pw);
          const D ss = dclamp01((D(1.0) - rough) * D(0.8) + D(m.metallic * 0.45) + D(m.clearcoat * 0.35));
          const V tint = vk(0.88, 0.88, 0.88) + alb * D(0.12);
          acc = acc + vmul(tint, irr) * (spec * cth * D(nl) * dmax(D(0.15), ss));
        }
        V contrib;
        if (c.mis) {
          const V ld = unit(vc(w.lights[0].pos) - hp);
          const D bp = dmax(D(0.0), dot(nrm, ld)) * D(1.0 / kPi);
          contrib = vmul(thr, acc) * mis(D(1.0 / nl), bp);
        } else {
          contrib = vmul(thr, acc);
        }
        const double remain = dist.v - 0.004;
        bool visible = true;
        if (remain > 0.004) {
          const P3 so{hp.x.v + nvec.x * 0.002, hp.y.v + nvec.y * 0.002, hp.z.v + nvec.z * 0.002};
          double ts;
          int tj;
          visible = !w.hit(so, pv(ldir), remain, ts, tj);
        }
        if (visible) rad = rad + contrib;
        fl |= visible ? 6u : 2u;
      }
    }

    const V refl = d - nrm * (D(2.0) * dot(nrm, d));
    V out;
    if (diffuse) {
      out = hemisphere(rng, nvec);
    } else {
      const D er = dmax(D(0.025), rough);
      const D a2 = er * er;
      const D ex = dmax(D(0.0), D(2.0) / (a2 * a2) - D(2.0));
      out = phong(rng, refl, ex, nvec, fl);
    }
    sig = mix64(sig ^ (static_cast<uint64_t>(ti + 1) | (static_cast<uint64_t>(fl) << 32)));
    if (dot(out, nrm).v <= 0.0) break;
    thr = vmul(thr, alb);
    auto c15 = [](double a) { return std::min(1.5, std::max(0.0, a)); };
    thr0 = {thr0.x * c15(m.alb0.x), thr0.y * c15(m.alb0.y), thr0.z * c15(m.alb0.z)};
    const double tmx = std::max(thr0.x, std::max(thr0.y, thr0.z));
    if (tmx < 0.001) break;
    const double rr = std::min(c.rr_max, std::max(c.rr_min, tmx));
    if (depth >= c.rr_start && rng.u() > rr) {
      sig = mix64(sig ^ 0x5252ull);   // roulette kill
      break;
    }
    thr = thr * D(1.0 / rr);   // the survival probability is held constant
    thr0 = {thr0.x / rr, thr0.y / rr, thr0.z / rr};
    if (depth + 1u >= c.max_depth) break;
    o = hp + out * D(0.002);
    d = out;
  }
  return rad;
}

bool load_world(const vko_scene& s, const float* params, const float* rr_params, uint32_t param_count,
                const uint32_t* grad_index, uint32_t grad_count, World& w) {
  for (uint32_t i = 0; i < s.instance_count; ++i) {
    const uint32_t first = s.instances[3 * i], count = s.instances[3 * i + 1], mat = s.instances[3 * i + 2];
    for (uint32_t k = 0; k < count; ++k) {
      const uint32_t base = (first + k) * 3u;
      if (base + 2u >= s.index_count) continue;
      const uint32_t a = s.indices[base], b = s.indices[base + 1], c = s.indices[base + 2];
      if (a >= s.vertex_count || b >= s.vertex_count || c >= s.vertex_count) continue;
      auto ld = [&](uint32_t vi) {
        return P3{s.vertices[3 * vi], s.vertices[3 * vi + 1], s.vertices[3 * vi + 2]};
      };
      Tri t;
      t.v0 = ld(a);
      t.e1 = psub(ld(b), t.v0);
      t.e2 = psub(ld(c), t.v0);
      t.n = punit(pcross(t.e1, t.e2));
      t.mat = mat;
      w.tris.push_back(t);
    }
  }
  const uint32_t nm = std::max(1u, s.material_count);
  if (param_count != VKO_ADJ_PARAMS_PER_MATERIAL * nm) {
    g_error = "params must hold 7 floats per material";
    return false;
  }
  for (uint32_t i = 0; i < nm; ++i) {
    const float* mm = s.material_count ? s.materials + 16 * i : nullptr;
    const float* p = params + VKO_ADJ_PARAMS_PER_MATERIAL * i;
    Mat m;
    m.alb = vk(p[0], p[1], p[2]);
    const float* q = (rr_params ? rr_params : params) + VKO_ADJ_PARAMS_PER_MATERIAL * i;
    m.alb0 = {q[0], q[1], q[2]};
    m.rough = D(p[3]);
    m.le = vk(p[4], p[5], p[6]);
    m.model = mm ? static_cast<uint32_t>(mm[7] + 0.5f) : 0u;
    m.metallic = mm ? mm[8] : 0.0;
    m.clearcoat = mm ? mm[11] : 0.0;
    const double transmission = mm ? mm[10] : 0.0;
    const double rough = std::min(1.0, std::max(0.0, static_cast<double>(p[3])));
    if ((m.model != 0u && m.model != 1u && m.model != 3u) || m.metallic > 0.65 || transmission > 0.05 ||
        m.clearcoat > 0.05 || rough <= 0.001) {
      g_error = "material " + std::to_string(i) + " is outside the supported set (Lambertian / Phong-lobe glossy)";
      return false;
    }
    w.mats.push_back(m);
  }
  // tangent slots
  for (uint32_t k = 0; k < grad_count; ++k) {
    const uint32_t gi = grad_index[k];
    const uint32_t mi = gi / VKO_ADJ_PARAMS_PER_MATERIAL, pi = gi % VKO_ADJ_PARAMS_PER_MATERIAL;
    if (mi >= w.mats.size()) {
      g_error = "grad_index out of range";
      return false;
    }
    Mat& m = w.mats[mi];
    D* slot = pi < 3 ? (pi == 0 ? &m.alb.x : pi == 1 ? &m.alb.y : &m.alb.z)
                     : pi == 3 ? &m.rough : (pi == 4 ? &m.le.x : pi == 5 ? &m.le.y : &m.le.z);
    slot->g[k] = 1.0;
  }
  for (uint32_t i = 0; i < s.light_count; ++i) {
    const float* l = s.lights + 16 * i;
    w.lights.push_back(Light{{l[0], l[1], l[2]}, {l[3], l[4], l[5]}, {l[8], l[9], l[10]}, l[6], l[7], l[11], l[12]});
  }
  w.env = {s.environment[0], s.environment[1], s.environment[2]};
  w.cam_pos = {s.camera_position[0], s.camera_position[1], s.camera_position[2]};
  const P3 tgt{s.camera_target[0], s.camera_target[1], s.camera_target[2]};
  const P3 up{s.camera_up[0], s.camera_up[1], s.camera_up[2]};
  w.cam_fwd = punit(psub(tgt, w.cam_pos));
  w.cam_right = punit(pcross(w.cam_fwd, up));
  if (pdot(w.cam_right, w.cam_right) <= kEps * kEps) w.cam_right = {1.0, 0.0, 0.0};
  w.cam_up = punit(pcross(w.cam_right, w.cam_fwd));
  if (pdot(w.cam_up, w.cam_up) <= kEps * kEps) w.cam_up = {0.0, 1.0, 0.0};
  w.tan_half = std::tan(0.5 * (static_cast<double>(s.camera_fov_deg) * (kPi / 180.0)));
  w.aperture = s.camera_aperture_radius;
  w.focus = s.camera_focus_distance;
  if (s.camera_lens_set) {
    w.iris_blades = std::min(s.camera_iris_blade_count, 64u);
    w.iris_rotation = static_cast<double>(s.camera_iris_rotation_degrees) * (kPi / 180.0);
    const float rd = s.camera_iris_roundness;
    w.iris_roundness = std::isfinite(rd) ? std::min(1.0f, std::max(0.0f, rd)) : 0.0;
    w.squeeze = std::isfinite(s.camera_anamorphic_squeeze) ? std::max(0.01f, s.camera_anamorphic_squeeze) : 1.0;
  }
  return true;
}

}  // namespace

extern "C" {

int vko_adjoint(const vko_scene* scene, const vko_settings* settings, const vko_adjoint_request* req, double* loss,
                double* grad, double* image) {
  if (!scene || !settings || !req || !req->params) {
    g_error = "null argument";
    return 1;
  }
  if (req->grad_count > VKO_ADJ_MAX_TANGENTS || (req->grad_count && (!req->grad_index || !grad))) {
    g_error = "grad_count above the tangent limit, or grad arrays missing";
    return 1;
  }
  NT = static_cast<int>(req->grad_count);
  World w;
  if (!load_world(*scene, req->params, req->rr_params, req->param_count, req->grad_index, req->grad_count, w)) return 1;
  Cfg c{settings->width, settings->height, settings->max_depth, settings->enable_nee, settings->enable_mis,
        settings->rr_start, settings->rr_min, settings->rr_max, settings->seed, settings->firefly_clamp, req->frame};
  const uint32_t W = c.width, H = c.height;
  const uint64_t npx = static_cast<uint64_t>(W) * H;
  const uint32_t threads = std::max(1u, req->threads);
  const int nt = NT;
  std::vector<double> t_loss(threads, 0.0), t_grad(static_cast<size_t>(threads) * std::max(1, nt), 0.0);
  std::vector<double> img(3 * npx, 0.0);
  auto work = [&](uint32_t tid) {
    NT = nt;
    std::vector<double> sg(3 * std::max(1, nt));
    for (uint32_t y = tid; y < H; y += threads) {
      for (uint32_t x = 0; x < W; ++x) {
        double sum[3] = {0.0, 0.0, 0.0};
        std::fill(sg.begin(), sg.end(), 0.0);
        uint32_t count = 0;
        for (uint32_t sm = 0; sm < req->spp; ++sm) {
          uint64_t sig = 0;
          const V r = trace_path(w, c, x, y, req->first_sample + sm, sig);
          const D* ch[3] = {&r.x, &r.y, &r.z};
          if (!(std::isfinite(r.x.v) && std::isfinite(r.y.v) && std::isfinite(r.z.v))) continue;
          ++count;
          for (int k = 0; k < 3; ++k) {
            const bool clamped = c.clamp > 0.0 && ch[k]->v > c.clamp;
            sum[k] += clamped ? c.clamp : ch[k]->v;
            if (!clamped)
              for (int i = 0; i < nt; ++i) sg[3 * i + k] += ch[k]->g[i];
          }
        }
        const double inv = 1.0 / static_cast<double>(std::max(1u, count));
        const size_t p = static_cast<size_t>(y) * W + x;
        for (int k = 0; k < 3; ++k) {
          const double iv = sum[k] * inv;
          img[3 * p + k] = iv;
          if (req->target) {
            const double diff = iv - static_cast<double>(req->target[3 * p + k]);
            t_loss[tid] += diff * diff;
            for (int i = 0; i < nt; ++i) t_grad[static_cast<size_t>(tid) * nt + i] += diff * inv * sg[3 * i + k];
          }
        }
      }
    }
  };
  if (threads == 1) {
    work(0);
  } else {
    std::vector<std::thread> pool;
    for (uint32_t t = 0; t < threads; ++t) pool.emplace_back(work, t);
    for (auto& th : pool) th.join();
  }
  double l = 0.0;
  for (uint32_t t = 0; t < threads; ++t) l += t_loss[t];
  const double scale = 1.0 / (3.0 * static_cast<double>(npx));
  if (loss) *loss = l * scale;
  for (int i = 0; i < nt; ++i) {
    double g = 0.0;
    for (uint32_t t = 0; t < threads; ++t) g += t_grad[static_cast<size_t>(t) * nt + i];
    grad[i] = 2.0 * scale * g;
  }
  if (image) std::memcpy(image, img.data(), img.size() * sizeof(double));
  return 0;
}

int vko_adjoint_fd(const vko_scene* scene, const vko_settings* settings, const vko_adjoint_request* req, double h,
                   double* fd_out, uint64_t* flips_out) {
  if (!scene || !settings || !req || !req->params || !req->target || !fd_out || h <= 0.0 ||
      (req->grad_count && !req->grad_index)) {
    g_error = "null argument or non-positive step";
    return 1;
  }
  NT = 0;
  World w;
  if (!load_world(*scene, req->params, nullptr, req->param_count, nullptr, 0, w)) return 1;
  Cfg c{settings->width, settings->height, settings->max_depth, settings->enable_nee, settings->enable_mis,
        settings->rr_start, settings->rr_min, settings->rr_max, settings->seed, settings->firefly_clamp, req->frame};
  const uint32_t W = c.width, H = c.height, spp = req->spp;
  const uint64_t npx = static_cast<uint64_t>(W) * H;
  const uint32_t threads = std::max(1u, req->threads);
  // Base pass: per-path radiance and signature, per-pixel loss weights.
  std::vector<double> L0(3 * npx * spp);
  std::vector<uint64_t> S0(npx * spp);
  std::vector<uint8_t> ok(npx * spp);
  std::vector<double> wgt(3 * npx);
  auto run = [&](const World& ww, std::vector<double>& L, std::vector<uint64_t>& S) {
    auto body = [&](uint32_t tid) {
      NT = 0;
      for (uint32_t y = tid; y < H; y += threads)
        for (uint32_t x = 0; x < W; ++x)
          for (uint32_t sm = 0; sm < spp; ++sm) {
            const size_t j = (static_cast<size_t>(y) * W + x) * spp + sm;
            uint64_t sig = 0;
            const V r = trace_path(ww, c, x, y, req->first_sample + sm, sig);
            L[3 * j] = r.x.v;
            L[3 * j + 1] = r.y.v;
            L[3 * j + 2] = r.z.v;
            S[j] = sig;
          }
    };
    std::vector<std::thread> pool;
    for (uint32_t t = 0; t < threads; ++t) pool.emplace_back(body, t);
    for (auto& th : pool) th.join();
  };
  run(w, L0, S0);
  for (uint64_t p = 0; p < npx; ++p) {
    double sum[3] = {0, 0, 0};
    uint32_t cnt = 0;
    for (uint32_t sm = 0; sm < spp; ++sm) {
      const size_t j = p * spp + sm;
      ok[j] = std::isfinite(L0[3 * j]) && std::isfinite(L0[3 * j + 1]) && std::isfinite(L0[3 * j + 2]);
      if (!ok[j]) continue;
      ++cnt;
      for (int k = 0; k < 3; ++k) sum[k] += (c.clamp > 0.0 && L0[3 * j + k] > c.clamp) ? c.clamp : L0[3 * j + k];
    }
    const double inv = 1.0 / std::max(1u, cnt);
    for (int k = 0; k < 3; ++k)
      wgt[3 * p + k] = 2.0 * (sum[k] * inv - req->target[3 * p + k]) / (3.0 * npx) * inv;
  }
  std::vector<double> Lp(L0.size()), Lm(L0.size());
  std::vector<uint64_t> Sp(S0.size()), Sm(S0.size());
  for (uint32_t gi = 0; gi < req->grad_count; ++gi) {
    const uint32_t idx = req->grad_index[gi];
    const uint32_t mi = idx / VKO_ADJ_PARAMS_PER_MATERIAL, pi = idx % VKO_ADJ_PARAMS_PER_MATERIAL;
    if (mi >= w.mats.size()) {
      g_error = "grad_index out of range";
      return 1;
    }
    auto slot = [&](World& ww) -> double& {
      Mat& m = ww.mats[mi];
      D* d = pi < 3 ? (pi == 0 ? &m.alb.x : pi == 1 ? &m.alb.y : &m.alb.z)
                    : pi == 3 ? &m.rough : (pi == 4 ? &m.le.x : pi == 5 ? &m.le.y : &m.le.z);
      return d->v;
    };
    World wp = w, wm = w;
    slot(wp) += h;
    slot(wm) -= h;
    run(wp, Lp, Sp);
    run(wm, Lm, Sm);
    double acc = 0.0;
    uint64_t flips = 0;
    for (size_t j = 0; j < S0.size(); ++j) {
      if (!ok[j]) continue;
      if (Sp[j] != S0[j] || Sm[j] != S0[j]) {
        ++flips;
        continue;
      }
      const size_t p = j / spp;
      for (int k = 0; k < 3; ++k) {
        if (c.clamp > 0.0 && L0[3 * j + k] > c.clamp) continue;
        acc += wgt[3 * p + k] * (Lp[3 * j + k] - Lm[3 * j + k]) / (2.0 * h);
      }
    }
    fd_out[gi] = acc;
    if (flips_out) flips_out[gi] = flips;
  }
  return 0;
}

const char* vko_adjoint_last_error(void) { return g_error.c_str(); }

}  // extern "C"
