// Test infrastructure (oracle): scalar CPU restatement of the reference's
// differentiable k-closest-hit trace path. Only tests, the smoke check and the
// CPU baseline leg of the benchmark use it; the product never links it.
//
// Real = float reproduces the reference's FP32 arithmetic, expression by
// expression, so that it can be compared bit for bit with the host build of
// the reference's own sources (refshim/). Real = double is the FP64 oracle:
// the same algorithm with every shading quantity in double and, with
// `exact_geometry`, the hit point taken from an FP64 plane intersection
// instead of the FP32 hit distance.
//
// Sources restated (paths relative to the reference project):
//   k-closest chunk query ........ tritracer/closestk.h:17-149
//   forward chunk loop ........... tritracer/forward.cu:76-155, raygen :161-215
//   computeScaling/angleBetween .. tritracer/forward.cu:25-74
//   window function .............. tritracer/common.h:57-114
//   SH -> RGB .................... tritracer/common.h:16-55, auxiliary.h:13-30
//   adjoint chunk loop ........... tritracer/backward.cu:191-350
//   window/SH adjoints ........... tritracer/backward.cu:25-189
//   3x3 Jacobian helpers ......... tritracer/vecmath.h:2626-2859
//   sphere variants .............. tritracer/reflect.cu, refract.cu, envlight.cu,
//                                  common.h:116-148
//   constants .................... tritracer/config.h:10-20, auxiliary.h:9-10
//
// Parity status: the FP32 instantiation is pinned bit for bit against the
// reference's own device code compiled for the host (refshim/), with one
// stand-in: OptiX's closed BVH traversal and triangle intersector are
// replaced by accel.hpp in both. Intersection t values and the tmin
// inclusivity of optixTrace are therefore unpinned against OptiX itself.
#pragma once
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>

#include "accel.hpp"
#include "hostmath.h"

namespace tto {

// ---------------------------------------------------------------- constants
// config.h:10-11, auxiliary.h:9-10, forward.cu:129-134
constexpr int kChunk = 16;
constexpr double kStepEps = 1e-9;  // a double literal in the reference
constexpr float kNear = 0.2f;
constexpr float kFar = 1000.0f;
constexpr float kAlphaMax = 0.99f;
constexpr float kAlphaMin = 1.0f / 255.0f;
constexpr float kTMin = 0.0001f;
constexpr uint32_t kInvalid = 0xFFFFFFFFu;
constexpr float kInfDist = 1e6f;
// config.h:16-20: channel offsets of the 7-channel side output
constexpr int kDepth = 0, kAlphaOff = 1, kNormal = 2, kMidDepth = 5, kDistortion = 6;

// auxiliary.h:13-30 (real SH basis constants, degree <= 3)
constexpr float kSH0 = 0.28209479177387814f;
constexpr float kSH1 = 0.4886025119029199f;
constexpr float kSH2[5] = {1.0925484305920792f, -1.0925484305920792f, 0.31539156525252005f, -1.0925484305920792f,
                           0.5462742152960396f};
constexpr float kSH3[7] = {-0.5900435899266435f, 2.890611442640554f, -0.4570457994644658f, 0.3731763325901154f,
                           -0.4570457994644658f, 1.445305721320277f, -0.5900435899266435f};

// ---------------------------------------------------------------- vectors
template <class R>
struct V3 {
  R x, y, z;
};
template <class R>
inline V3<R> mk(R x, R y, R z) {
  return V3<R>{x, y, z};
}
template <class R>
inline V3<R> from_f(const float* p) {
  return V3<R>{(R)p[0], (R)p[1], (R)p[2]};
}
template <class R>
inline V3<R> operator+(V3<R> a, V3<R> b) {
  return {a.x + b.x, a.y + b.y, a.z + b.z};
}
template <class R>
inline V3<R> operator-(V3<R> a, V3<R> b) {
  return {a.x - b.x, a.y - b.y, a.z - b.z};
}
template <class R>
inline V3<R> operator-(V3<R> a) {
  return {-a.x, -a.y, -a.z};
}
template <class R>
inline V3<R> operator*(V3<R> a, R s) {
  return {a.x * s, a.y * s, a.z * s};
}
template <class R>
inline V3<R> operator*(R s, V3<R> a) {
  return {a.x * s, a.y * s, a.z * s};
}
template <class R>
inline V3<R> vmul(V3<R> a, V3<R> b) {
  return {a.x * b.x, a.y * b.y, a.z * b.z};
}
// scalar division is a reciprocal followed by a multiply (vecmath.h:491-503)
template <class R>
inline V3<R> operator/(V3<R> a, R s) {
  R inv = R(1) / s;
  return a * inv;
}
template <class R>
inline R dot(V3<R> a, V3<R> b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <class R>
inline V3<R> cross(V3<R> a, V3<R> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class R>
inline R length(V3<R> v) {
  return std::sqrt(dot(v, v));
}
template <class R>
inline V3<R> normalize(V3<R> v) {
  R inv = R(1) / std::sqrt(dot(v, v));
  return v * inv;
}
template <class R>
inline V3<R> reflect(V3<R> i, V3<R> n) {
  return i - (R(2) * n) * dot(n, i);
}
template <class R>
inline R sum3(V3<R> a) {
  return a.x + a.y + a.z;
}

// ---------------------------------------------------------------- 3x3 helpers
// Row-major 3x3 matrices (vecmath.h:2626-2859, restated).
template <class R>
struct M3 {
  R m[9];
};
template <class R>
inline V3<R> vecmat(V3<R> v, const M3<R>& A) {  // v^T A
  return {A.m[0] * v.x + A.m[3] * v.y + A.m[6] * v.z, A.m[1] * v.x + A.m[4] * v.y + A.m[7] * v.z,
          A.m[2] * v.x + A.m[5] * v.y + A.m[8] * v.z};
}
template <class R>
inline M3<R> identity_scaled(R s) {
  M3<R> I;
  for (int i = 0; i < 9; ++i) I.m[i] = (i % 4 == 0 ? R(1) : R(0)) * s;
  return I;
}
template <class R>
inline M3<R> outer(V3<R> u, V3<R> v) {
  return M3<R>{{u.x * v.x, u.x * v.y, u.x * v.z, u.y * v.x, u.y * v.y, u.y * v.z, u.z * v.x, u.z * v.y, u.z * v.z}};
}
template <class R>
inline M3<R> skew(V3<R> v) {
  return M3<R>{{R(0), -v.z, v.y, v.z, R(0), -v.x, -v.y, v.x, R(0)}};
}
template <class R>
inline M3<R> madd(const M3<R>& a, const M3<R>& b) {
  M3<R> c;
  for (int i = 0; i < 9; ++i) c.m[i] = a.m[i] + b.m[i];
  return c;
}
template <class R>
inline M3<R> msub(const M3<R>& a, const M3<R>& b) {
  M3<R> c;
  for (int i = 0; i < 9; ++i) c.m[i] = a.m[i] - b.m[i];
  return c;
}
// Jacobian of v/|v| w.r.t. v: (I - n n^T) / |v|. The reference scales by the
// double quotient 1./|v| rounded to the working type (vecmath.h:2796-2806).
template <class R>
inline M3<R> dnormvdv(V3<R> n, V3<R> v) {
  M3<R> out = msub(identity_scaled(R(1)), outer(n, n));
  const R s = (R)(1.0 / (double)length(v));
  for (int i = 0; i < 9; ++i) out.m[i] *= s;
  return out;
}
// Jacobians of the unnormalised edge normal ne = ((p1-p3) x (p2-p3)) x (p1-p2)
// w.r.t. p1, p2, p3, in the form the reference uses (vecmath.h:2808-2859).
template <class R>
inline M3<R> dne_dp1(V3<R> p1, V3<R> p2, V3<R> p3) {
  V3<R> b = p2 - p3, c = p1 - p2;
  V3<R> axb = cross(p1 - p3, b);
  M3<R> t = msub(outer(b, c), identity_scaled(dot(b, c)));
  return madd(t, skew(axb));
}
template <class R>
inline M3<R> dne_dp2(V3<R> p1, V3<R> p2, V3<R> p3) {
  V3<R> a = p1 - p3, b = p2 - p3, c = p1 - p2;
  V3<R> axb = cross(p1 - p3, b);
  M3<R> t = msub(identity_scaled(dot(a, c)), outer(a, c));
  return msub(t, skew(axb));
}
template <class R>
inline M3<R> dne_dp3(V3<R> p1, V3<R> p2, V3<R> p3) {
  V3<R> c = p1 - p2;
  return msub(outer(c, c), identity_scaled(dot(c, c)));
}

// ---------------------------------------------------------------- scalar ops
template <class R>
inline R fast_pow(R x, R y);
template <>
inline float fast_pow<float>(float x, float y) {
  return tt_host_powf(x, y);
}
template <>
inline double fast_pow<double>(double x, double y) {
  if (!(x >= 0.0)) return std::numeric_limits<double>::quiet_NaN();
  return std::pow(x, y);
}
template <class R>
inline R fast_log(R x);
template <>
inline float fast_log<float>(float x) {
  return tt_host_logf(x);
}
template <>
inline double fast_log<double>(double x) {
  return std::log(x);
}

template <class R>
inline void atomic_add(R* p, R v, bool mt) {
  if (!mt) {
    *p += v;
    return;
  }
  R cur;
  __atomic_load(p, &cur, __ATOMIC_RELAXED);
  R nxt;
  do {
    nxt = cur + v;
  } while (!__atomic_compare_exchange(p, &cur, &nxt, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED));
}
template <class R>
inline void atomic_max(R* p, R v, bool mt) {
  if (!mt) {
    if (v > *p) *p = v;
    return;
  }
  R cur;
  __atomic_load(p, &cur, __ATOMIC_RELAXED);
  while (v > cur) {
    if (__atomic_compare_exchange(p, &cur, &v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) break;
  }
}

// ---------------------------------------------------------------- options
struct Opts {
  bool exact_adjoint = false;   // full chain rule + depth accumulation (no reference counterpart)
  bool tmin_inclusive = true;   // optixTrace's closed [tmin, tmax]
  bool canonical_ties = false;  // order equal-t hits by primitive id
  bool exact_geometry = false;  // hit point from an FP64 plane intersection
  bool mt = false;              // several threads share the output arrays
};

struct Hit {
  uint32_t id;
  float t;
};

// ------------------------------------------------------------ k-closest query
// closestk.h:17-149: 16 (id, t) pairs start as (invalid, 1e6); every candidate
// that beats slot 15 is bubbled in by compare-and-swap; the candidate is
// ignored unless it ends up in slot 15, so tmax only shrinks to the 16th hit.
inline bool hit_less(const Hit& a, const Hit& b, bool canonical) {
  if (a.t < b.t) return true;
  return canonical && a.t == b.t && a.id < b.id;
}

inline void trace_chunk(const Scene& sc, const RayPre& r, float tmin, float tmax, const Opts& o, Hit pl[kChunk]) {
  for (int k = 0; k < kChunk; ++k) pl[k] = Hit{kInvalid, kInfDist};
  sc.for_each_hit(r, tmin, tmax, o.tmin_inclusive, [&](int prim, float t, float tcur) -> float {
    Hit h{(uint32_t)prim, t};
    if (hit_less(h, pl[kChunk - 1], o.canonical_ties)) {
      for (int k = 0; k < kChunk; ++k) {
        if (hit_less(h, pl[k], o.canonical_ties)) std::swap(h, pl[k]);
      }
      const bool landed_last = o.canonical_ties ? (pl[kChunk - 1].id == (uint32_t)prim && pl[kChunk - 1].t == t)
                                                : !(pl[kChunk - 1].t > t);
      if (!landed_last) return tcur;  // optixIgnoreIntersection
    }
    return t;  // accepted: the interval's upper end shrinks to t
  });
}

// Drives the chunked march of forward.cu:97-154: trace 16 hits from
// last_hit_t, visit them in order, re-trace from the last one. `visit`
// receives (prim, t) for every entry at or beyond the near plane and returns
// true to end the ray; `record` sees every entry, including near ones.
//
// A proposed interval [t_near, t_far] (the GPU's clipped traversal, no
// reference counterpart) starts the march at t_near, closed, when the
// interval holds a hit; otherwise, or when t_near is not in (0, far), the
// march is the plain one. t_far only bounds the GPU's work: a ray that
// reaches it unterminated goes on, so the visited hits do not depend on it.
template <class Visit, class Record>
inline void march(const Scene& sc, const RayPre& r, const Opts& o, Visit&& visit, Record&& record,
                  float t_near = 0.f, float t_far = kFar) {
  float last_hit_t = 0.f;
  Hit pl[kChunk];
  bool clipped = false;
  if (t_near > 0.f && t_near < kFar) {
    Opts closed = o;
    closed.tmin_inclusive = true;
    const float hi = (t_far >= 0.f && t_far < kFar) ? t_far : kFar;
    trace_chunk(sc, r, t_near, hi, closed, pl);
    if (pl[0].id != kInvalid) {
      trace_chunk(sc, r, t_near, kFar, closed, pl);
      clipped = true;
    }
  }
  for (int guard = 0; guard < (1 << 22); ++guard) {
    if (!clipped) trace_chunk(sc, r, last_hit_t, kFar, o, pl);
    clipped = false;
    for (int i = 0; i < kChunk; ++i) {
      const Hit h = pl[i];
      if (h.id == kInvalid) return;
      record(h);
      // fmaxf(last + STEP_EPSILON, t): the sum is formed in double and rounded
      // back to float by fmaxf's parameter (forward.cu:111)
      last_hit_t = std::fmax((float)((double)last_hit_t + kStepEps), h.t);
      if (h.t < kNear) continue;
      if (visit(h.id, h.t)) return;
    }
  }
}

// ---------------------------------------------------------------- inputs
struct Inputs {
  int H = 0, W = 0;
  const float* ray_o = nullptr;
  const float* ray_d = nullptr;
  const float* verts = nullptr;
  const int* num_points = nullptr;
  const int* cumsum = nullptr;
  int P = 0;
  const float* shs = nullptr;
  int sh_degree = 0;
  int M = 0;
  const float* opacities = nullptr;
  const float* sigma = nullptr;
  const float* bg = nullptr;
  const float* extra = nullptr;
  int extra_len = 0;
  const float* interval = nullptr;  // optional [2][H][W] proposed [t_near, t_far] per ray
  const float* colors = nullptr;    // optional [P][3] precomputed colours in place of SH
};

inline void ray_interval(const Inputs& in, int pix, float& t_near, float& t_far) {
  t_near = 0.f;
  t_far = kFar;
  if (!in.interval) return;
  const int HW = in.H * in.W;
  t_near = in.interval[pix];
  t_far = in.interval[HW + pix];
}

template <class R>
inline V3<R> vert(const Inputs& in, int off) {
  return from_f<R>(in.verts + 3 * (size_t)off);
}

// Hit point on the triangle. Reference: o + t d from the FP32 distance
// (forward.cu:118). Exact-geometry: the same point from an FP64 plane solve.
template <class R>
inline V3<R> hit_point(const Inputs& in, int prim, V3<R> o, V3<R> d, float t, const Opts& opt) {
  if (!opt.exact_geometry) return o + R(t) * d;
  const int off = in.cumsum[prim];
  const V3<double> A = from_f<double>(in.verts + 3 * (size_t)off);
  const V3<double> B = from_f<double>(in.verts + 3 * (size_t)(off + 1));
  const V3<double> C = from_f<double>(in.verts + 3 * (size_t)(off + 2));
  const V3<double> od{(double)o.x, (double)o.y, (double)o.z}, dd{(double)d.x, (double)d.y, (double)d.z};
  const V3<double> n = cross(B - A, C - A);
  const double te = dot(A - od, n) / dot(dd, n);
  const V3<double> p = od + te * dd;
  return V3<R>{(R)p.x, (R)p.y, (R)p.z};
}

template <class R>
inline R hit_dist(const Inputs& in, int prim, V3<R> o, V3<R> d, float t, const Opts& opt) {
  if (!opt.exact_geometry) return R(t);
  const int off = in.cumsum[prim];
  const V3<double> A = from_f<double>(in.verts + 3 * (size_t)off);
  const V3<double> B = from_f<double>(in.verts + 3 * (size_t)(off + 1));
  const V3<double> C = from_f<double>(in.verts + 3 * (size_t)(off + 2));
  const V3<double> od{(double)o.x, (double)o.y, (double)o.z}, dd{(double)d.x, (double)d.y, (double)d.z};
  const V3<double> n = cross(B - A, C - A);
  return (R)(dot(A - od, n) / dot(dd, n));
}

// ---------------------------------------------------------------- shading
// common.h:57-114. Edge normals are normalize(edge_cross x (p_i - p_{i+1}));
// the incenter's signed distance to edge 0 is `dist` (negative inside);
// phi = max edge distance of the hit point; phi_final = phi / dist;
// Cx = max(0, phi_final^sigma) with a NaN (negative base) clamped to 0.
template <class R>
struct Window {
  R Cx;
  V3<R> n;
  R phi_final, phi_max;
  R d[3];
  R dist;         // signed distance of the incenter to edge 0
  V3<R> incenter;
  V3<R> en[3];    // edge normals as used (edge 0 oriented by the incenter)
};

template <class R>
inline Window<R> window_fn(const Inputs& in, int prim, V3<R> hit_p) {
  Window<R> w;
  const int off = in.cumsum[prim];
  const V3<R> A = vert<R>(in, off), B = vert<R>(in, off + 1), C = vert<R>(in, off + 2);
  const V3<R> P3[3] = {A, B, C};
  const R a = length(B - C), b = length(A - C), c = length(A - B);
  const V3<R> incenter = (a * A + b * B + c * C) / (a + b + c);
  const V3<R> edge_cross = cross(B - A, C - A);
  w.n = normalize(edge_cross);
  R dist = std::numeric_limits<R>::infinity();
  R phi = -std::numeric_limits<R>::infinity();
  for (int i = 0; i < 3; ++i) {
    const V3<R> p1 = P3[i], p2 = P3[(i + 1) % 3];
    V3<R> en = normalize(cross(edge_cross, p1 - p2));
    R offset = -dot(en, p1);
    if (dist == std::numeric_limits<R>::infinity()) {
      dist = dot(en, incenter) + offset;
      if (dist > R(0)) {
        en = -en;
        offset = -offset;
        dist = -dist;
      }
    }
    const R ed = dot(en, hit_p) + offset;
    phi = std::fmax(phi, ed);
    w.d[i] = ed;
    w.en[i] = en;
  }
  w.dist = dist;
  w.incenter = incenter;
  w.phi_max = phi;
  w.phi_final = phi / dist;
  w.Cx = std::fmax(R(0), fast_pow<R>(w.phi_final, (R)in.sigma[prim]));
  return w;
}

// common.h:16-55: real SH basis on the normalised direction, +0.5, clamp >= 0.
template <class R>
inline V3<R> sh_color(const Inputs& in, int idx, V3<R> dir, bool clamped[3]) {
  if (in.colors) {  // precomputed colours (no reference counterpart: it never reads them)
    if (clamped) clamped[0] = clamped[1] = clamped[2] = false;
    return from_f<R>(in.colors + 3 * (size_t)idx);
  }
  dir = dir / length(dir);
  const float* base = in.shs + 3 * (size_t)idx * in.M;
  auto sh = [&](int k) { return from_f<R>(base + 3 * k); };
  V3<R> result = R(kSH0) * sh(0);
  const int deg = in.sh_degree;
  if (deg > 0) {
    const R x = dir.x, y = dir.y, z = dir.z;
    result = result - R(kSH1) * y * sh(1) + R(kSH1) * z * sh(2) - R(kSH1) * x * sh(3);
    if (deg > 1) {
      const R xx = x * x, yy = y * y, zz = z * z;
      const R xy = x * y, yz = y * z, xz = x * z;
      result = result + R(kSH2[0]) * xy * sh(4) + R(kSH2[1]) * yz * sh(5) +
               R(kSH2[2]) * (R(2) * zz - xx - yy) * sh(6) + R(kSH2[3]) * xz * sh(7) +
               R(kSH2[4]) * (xx - yy) * sh(8);
      if (deg > 2) {
        result = result + R(kSH3[0]) * y * (R(3) * xx - yy) * sh(9) + R(kSH3[1]) * xy * z * sh(10) +
                 R(kSH3[2]) * y * (R(4) * zz - xx - yy) * sh(11) +
                 R(kSH3[3]) * z * (R(2) * zz - R(3) * xx - R(3) * yy) * sh(12) +
                 R(kSH3[4]) * x * (R(4) * zz - xx - yy) * sh(13) + R(kSH3[5]) * z * (xx - yy) * sh(14) +
                 R(kSH3[6]) * x * (xx - R(3) * yy) * sh(15);
      }
    }
  }
  result = result + mk<R>(R(0.5f), R(0.5f), R(0.5f));
  if (clamped) {
    clamped[0] = result.x < R(0);
    clamped[1] = result.y < R(0);
    clamped[2] = result.z < R(0);
  }
  return mk<R>(std::fmax(result.x, R(0)), std::fmax(result.y, R(0)), std::fmax(result.z, R(0)));
}

// forward.cu:25-74: the first ray to blend a triangle records the largest
// angle its vertices subtend around the centroid direction.
template <class R>
inline R angle_between(V3<R> a, V3<R> b) {
  const R len_ab = length(a) * length(b);
  if (len_ab < R(1e-12f)) return R(0);
  const R cos_t = std::fmax(R(-1), std::fmin(R(1), dot(a, b) / len_ab));
  return std::acos(cos_t);
}

template <class R>
inline void compute_scaling(const Inputs& in, int idx, V3<R> ray_o, R* scaling, bool mt) {
  R cur = scaling[idx];
  if (mt) __atomic_load(&scaling[idx], &cur, __ATOMIC_RELAXED);
  if (cur > R(0)) return;
  const int off = in.cumsum[idx];
  const int np = in.num_points[idx];
  V3<R> center = mk<R>(R(0), R(0), R(0));
  for (int i = 0; i < np; ++i) center = center + vert<R>(in, off + i);
  {
    const R inv = R(1) / (R)np;
    center = center * inv;
  }
  const V3<R> tri2org = center - ray_o;
  R max_angle = R(0);
  for (int i = 0; i < np; ++i) {
    const R ang = angle_between(vert<R>(in, off + i) - ray_o, tri2org);
    max_angle = std::fmax(ang, max_angle);
  }
  if (mt)
    __atomic_store(&scaling[idx], &max_angle, __ATOMIC_RELAXED);
  else
    scaling[idx] = max_angle;
}

// ---------------------------------------------------------------- recording
struct RayRecord {
  int max_rec = 0;
  int* ids = nullptr;  // [max_rec] processed entries in order
  int count = 0;
  double margin = INFINITY;  // smallest relative distance of a decision to its threshold
  void add(const Hit& h) {
    if (count < max_rec) ids[count] = (int)h.id;
    ++count;
  }
  void near(double v, double thr) {
    const double m = std::fabs(v - thr) / std::fabs(thr);
    if (m < margin) margin = m;
  }
};

// ---------------------------------------------------------------- forward
template <class R>
struct FwdOut {
  R* scaling;
  R* density;
  R* color;   // [3, H, W]
  R* others;  // [7, H, W]
  R* max_blending;
};

// forward.cu:76-155 + raygen :161-215 (plain variant).
template <class R>
inline void forward_ray(const Scene& sc, const Inputs& in, int pix, const Opts& opt, FwdOut<R>& out, RayRecord* rec) {
  const int HW = in.H * in.W;
  const float* of = in.ray_o + 3 * (size_t)pix;
  const float* df = in.ray_d + 3 * (size_t)pix;
  const V3<R> o = from_f<R>(of), d = from_f<R>(df);
  const RayPre rp = ray_pre(of, df);
  float t_near, t_far;
  ray_interval(in, pix, t_near, t_far);
  R C[3] = {0, 0, 0}, N[3] = {0, 0, 0};
  R T = 1;
  R D = 0;  // the reference never accumulates depth; the exact adjoint's forward does
  // exact adjoint's forward only: middepth (t of the hit after which T <= 0.5)
  // and distortion sum_{i<j} w_i w_j (t_i - t_j)^2 with running sums of w, w t^2
  R Wsum = 0, C2 = 0, mid = 0, dist2 = 0;
  bool mid_set = false;
  march(
      sc, rp, opt,
      [&](uint32_t prim, float t) -> bool {
        const V3<R> hp = hit_point(in, (int)prim, o, d, t, opt);
        const Window<R> w = window_fn(in, (int)prim, hp);
        const R alpha = std::fmin(R(kAlphaMax), (R)in.opacities[prim] * w.Cx);
        if (rec) rec->near((double)alpha, (double)kAlphaMin);
        if (alpha < R(kAlphaMin)) return false;
        const R test_T = T * (R(1) - alpha);
        if (rec) rec->near((double)test_T, (double)kTMin);
        if (test_T < R(kTMin)) return true;
        out.density[prim] = R(1);
        compute_scaling(in, (int)prim, o, out.scaling, opt.mt);
        const R bw = alpha * T;
        atomic_max(&out.max_blending[prim], bw, opt.mt);
        N[0] += w.n.x * bw;
        N[1] += w.n.y * bw;
        N[2] += w.n.z * bw;
        if (opt.exact_adjoint) {
          const R ht = hit_dist(in, (int)prim, o, d, t, opt);
          dist2 += bw * (ht * ht * Wsum - R(2) * ht * D + C2);
          Wsum += bw;
          D += bw * ht;
          C2 += bw * ht * ht;
          if (!mid_set && test_T <= R(0.5)) {
            mid = ht;
            mid_set = true;
          }
        }
        const V3<R> col = sh_color(in, (int)prim, d, nullptr);
        C[0] += col.x * bw;
        C[1] += col.y * bw;
        C[2] += col.z * bw;
        T = test_T;
        return false;
      },
      [&](const Hit& h) {
        if (rec) rec->add(h);
      },
      t_near, t_far);
  for (int ch = 0; ch < 3; ++ch) out.color[ch * HW + pix] = C[ch] + T * (R)in.bg[ch];
  out.others[pix + kDepth * HW] = D;
  out.others[pix + kAlphaOff * HW] = R(1) - T;
  for (int ch = 0; ch < 3; ++ch) out.others[pix + (kNormal + ch) * HW] = N[ch];
  out.others[pix + kMidDepth * HW] = mid;
  out.others[pix + kDistortion * HW] = dist2;
}

// ---------------------------------------------------------------- variants
// The chunk loop of reflect.cu/refract.cu/envlight.cu: like the plain one but
// without side outputs (reflect.cu:25-96).
template <class R>
inline void march_color(const Scene& sc, const Inputs& in, V3<float> of, V3<float> df, const Opts& opt, R C[3], R& T,
                        RayRecord* rec) {
  const float ofa[3] = {of.x, of.y, of.z}, dfa[3] = {df.x, df.y, df.z};
  const V3<R> o = from_f<R>(ofa), d = from_f<R>(dfa);
  const RayPre rp = ray_pre(ofa, dfa);
  march(
      sc, rp, opt,
      [&](uint32_t prim, float t) -> bool {
        const V3<R> hp = hit_point(in, (int)prim, o, d, t, opt);
        const Window<R> w = window_fn(in, (int)prim, hp);
        const R alpha = std::fmin(R(kAlphaMax), (R)in.opacities[prim] * w.Cx);
        if (rec) rec->near((double)alpha, (double)kAlphaMin);
        if (alpha < R(kAlphaMin)) return false;
        const R test_T = T * (R(1) - alpha);
        if (rec) rec->near((double)test_T, (double)kTMin);
        if (test_T < R(kTMin)) return true;
        const R bw = alpha * T;
        const V3<R> col = sh_color(in, (int)prim, d, nullptr);
        C[0] += col.x * bw;
        C[1] += col.y * bw;
        C[2] += col.z * bw;
        T = test_T;
        return false;
      },
      [&](const Hit& h) {
        if (rec) rec->add(h);
      });
}

// common.h:116-141 (ray/sphere, nearest root beyond STEP_EPSILON). The sphere
// geometry is always FP32: it decides the secondary ray, which then feeds the
// FP32 intersector exactly as in the reference.
inline bool hit_sphere(float r, V3<float> cnt, V3<float> o, V3<float> d, float& t) {
  const V3<float> op = o - cnt;
  const float a = dot(d, d);
  if (a <= 0.0f) return false;
  const float b = dot(op, d);
  const float c = dot(op, op) - r * r;
  float det = b * b - c * a;
  if (det < 0.0f) return false;
  det = std::sqrt(det);
  t = (-b - det) / a;
  if ((double)t < kStepEps) {
    t = (-b + det) / a;
    if ((double)t < kStepEps) return false;
  }
  return true;
}

// refract.cu:24-45, kept with its arithmetic as written (square roots where
// Snell's law has squares; the double/float mix of the original).
inline bool refract_dir(V3<float>& out_dir, V3<float> in_dir, V3<float> normal, float eta_org) {
  const float cos_i = dot(in_dir, normal);
  float eta = eta_org;
  if ((double)cos_i > 0.0) {
    eta = (float)(1.0 / (double)eta_org);
    normal = -normal;
  }
  const float sin2_i = (float)std::fmax(0.0, 1.0 - (double)std::sqrt(cos_i));
  const float sin2_t = sin2_i / std::sqrt(eta);
  if (sin2_t >= 1.0f) return false;
  const float cos_t = (float)std::sqrt(std::fmax(0.0, 1.0 - (double)sin2_t));
  out_dir = in_dir / eta + (-cos_i / eta - cos_t) * normal;
  return true;
}

// envlight.cu:25-51: LCG and cosine-weighted hemisphere sample.
inline float lcg(uint32_t& u) {
  u = u * 1664525u + 1013904223u;
  return (float)(u & 0x00FFFFFFu) * (1.0f / 16777216.0f);
}
inline V3<float> cosine_hemisphere(uint32_t& seed, V3<float> normal) {
  const float u = lcg(seed);
  const float v = lcg(seed);
  const float PI2 = 6.2831853071795864769f;
  const float z = std::sqrt(u);
  const float r = std::sqrt(std::fmax(0.0f, (float)(1.0 - (double)(z * z))));
  const float phi = v * PI2;
  const V3<float> dir{r * std::cos(phi), r * std::sin(phi), z};
  const V3<float> up = std::fabs(normal.z) < 0.999f ? V3<float>{0.f, 0.f, 1.f} : V3<float>{0.f, 1.f, 0.f};
  const V3<float> t = normalize(cross(up, normal));
  const V3<float> b = normalize(cross(normal, t));
  const V3<float> world = dir.x * t + dir.y * b + dir.z * normal;
  return normalize(world);
}

enum Variant { kPlain = 0, kReflect = 1, kRefract = 2, kEnvlight = 3 };

template <class R>
inline void variant_ray(const Scene& sc, const Inputs& in, int pix, int variant, const Opts& opt, FwdOut<R>& out,
                        RayRecord* rec) {
  const int HW = in.H * in.W;
  V3<float> o{in.ray_o[3 * pix], in.ray_o[3 * pix + 1], in.ray_o[3 * pix + 2]};
  V3<float> d{in.ray_d[3 * pix], in.ray_d[3 * pix + 1], in.ray_d[3 * pix + 2]};
  // extract_sphere: extra = [r, cx, cy, cz, samples] (common.h:143-148)
  const float rad = in.extra[0];
  const V3<float> cnt{in.extra[1], in.extra[2], in.extra[3]};
  const float eps = (float)kStepEps;
  R C[3] = {0, 0, 0};
  R T = 1;
  if (variant == kReflect) {  // reflect.cu:42-48
    float st;
    if (hit_sphere(rad, cnt, o, d, st)) {
      o = o + d * st;
      const V3<float> n = normalize(o - cnt);
      o = o + n * eps;
      d = reflect(normalize(d), n);
    }
    march_color(sc, in, o, d, opt, C, T, rec);
  } else if (variant == kRefract) {  // refract.cu:47-71
    float st;
    if (hit_sphere(rad, cnt, o, d, st)) {
      const V3<float> hp = o + d * st;
      const V3<float> n = normalize(hp - cnt);
      const V3<float> in_dir = normalize(d);
      const float n1 = 1.0003f, n2 = 1.5f;
      const float ior = n2 / n1;
      V3<float> nd = in_dir;
      if (!refract_dir(nd, in_dir, n, ior)) {
        const V3<float> rn = dot(in_dir, n) < 0.0f ? n : -n;
        nd = reflect(in_dir, rn);
      }
      o = hp + n * eps;
      d = nd;
    }
    march_color(sc, in, o, d, opt, C, T, rec);
  } else {  // envlight.cu:116-184
    const int samples = (int)in.extra[4];
    float st;
    if (hit_sphere(rad, cnt, o, d, st)) {
      o = o + d * st;
      const V3<float> n0 = normalize(o - cnt);
      o = o + n0 * eps;
      R acc[3] = {0, 0, 0};
      for (int i = 0; i < samples; ++i) {
        const V3<float> n = normalize(o - cnt);
        uint32_t seed = ((uint32_t)(pix + 1u) * 9781u) ^ ((uint32_t)(i + 1u) * 6271u);
        const V3<float> dn = cosine_hemisphere(seed, n);
        const V3<float> on = o + dn * eps;
        R Cn[3] = {0, 0, 0};
        R Tn = 1;
        march_color(sc, in, on, dn, opt, Cn, Tn, rec);
        for (int ch = 0; ch < 3; ++ch) acc[ch] += Cn[ch] + Tn * (R)in.bg[ch];
      }
      const R inv = R(1.0f / (float)samples);
      for (int ch = 0; ch < 3; ++ch) C[ch] += acc[ch] * inv;
      T = 0;
    } else {
      march_color(sc, in, o, d, opt, C, T, rec);
    }
  }
  for (int ch = 0; ch < 3; ++ch) out.color[ch * HW + pix] = C[ch] + T * (R)in.bg[ch];
}

// ---------------------------------------------------------------- backward
template <class R>
struct BwdIn {
  const R* colors;  // forward outputs [3, H, W]
  const R* others;  // [7, H, W]
  const float* dL_dpixels;
  const float* dL_dothers;
};
template <class R>
struct BwdOut {
  R* dtri;    // [sum points, 3]
  R* dsigma;  // [P]
  R* dopac;   // [P]
  R* dsh;     // [P, M, 3]
  R* dcolors = nullptr;  // [P, 3] with precomputed colours
  R* denv = nullptr;     // secondary rays: [env_h, env_w, 3] environment map
  R* dior = nullptr;     // secondary rays: [P] IOR (through the Fresnel share)
};

template <class R>
inline void add3(R* g, int idx, V3<R> v, bool mt) {
  atomic_add(&g[3 * (size_t)idx + 0], v.x, mt);
  atomic_add(&g[3 * (size_t)idx + 1], v.y, mt);
  atomic_add(&g[3 * (size_t)idx + 2], v.z, mt);
}

// backward.cu:33-102
template <class R>
inline void sh_color_bwd(const Inputs& in, int idx, V3<R> dir_orig, const bool clamped[3], const R dL_dcolor[3],
                         R* dsh, bool mt) {
  const V3<R> dir = dir_orig / length(dir_orig);
  V3<R> g = mk<R>(dL_dcolor[0], dL_dcolor[1], dL_dcolor[2]);
  g.x *= clamped[0] ? R(0) : R(1);
  g.y *= clamped[1] ? R(0) : R(1);
  g.z *= clamped[2] ? R(0) : R(1);
  const R x = dir.x, y = dir.y, z = dir.z;
  const int base = idx * in.M;
  const int deg = in.sh_degree;
  add3(dsh, base + 0, R(kSH0) * g, mt);
  if (deg > 0) {
    add3(dsh, base + 1, (R(-kSH1) * y) * g, mt);
    add3(dsh, base + 2, (R(kSH1) * z) * g, mt);
    add3(dsh, base + 3, (R(-kSH1) * x) * g, mt);
    if (deg > 1) {
      const R xx = x * x, yy = y * y, zz = z * z;
      const R xy = x * y, yz = y * z, xz = x * z;
      add3(dsh, base + 4, (R(kSH2[0]) * xy) * g, mt);
      add3(dsh, base + 5, (R(kSH2[1]) * yz) * g, mt);
      add3(dsh, base + 6, (R(kSH2[2]) * (R(2) * zz - xx - yy)) * g, mt);
      add3(dsh, base + 7, (R(kSH2[3]) * xz) * g, mt);
      add3(dsh, base + 8, (R(kSH2[4]) * (xx - yy)) * g, mt);
      if (deg > 2) {
        add3(dsh, base + 9, (R(kSH3[0]) * y * (R(3) * xx - yy)) * g, mt);
        add3(dsh, base + 10, (R(kSH3[1]) * xy * z) * g, mt);
        add3(dsh, base + 11, (R(kSH3[2]) * y * (R(4) * zz - xx - yy)) * g, mt);
        add3(dsh, base + 12, (R(kSH3[3]) * z * (R(2) * zz - R(3) * xx - R(3) * yy)) * g, mt);
        add3(dsh, base + 13, (R(kSH3[4]) * x * (R(4) * zz - xx - yy)) * g, mt);
        add3(dsh, base + 14, (R(kSH3[5]) * z * (xx - yy)) * g, mt);
        add3(dsh, base + 15, (R(kSH3[6]) * x * (xx - R(3) * yy)) * g, mt);
      }
    }
  }
}

// backward.cu:104-189: gradient of phi_max through the unit normal of each
// edge whose distance equals phi_max (within 1e-6), plus the face-normal
// gradient through the cross product of two edges.
template <class R>
inline void window_bwd(const Inputs& in, int prim, V3<R> hit_p, R dL_dphi_x, R phi_x, const R dist[3],
                       V3<R> dL_dnormal3D, R* dtri, bool mt) {
  const int off = in.cumsum[prim];
  const V3<R> v[3] = {vert<R>(in, off), vert<R>(in, off + 1), vert<R>(in, off + 2)};
  for (int k = 0; k < 3; ++k) {
    if (std::fabs(dist[k] - phi_x) > R(1e-6f)) continue;
    const V3<R> p1 = v[k], p2 = v[(k + 1) % 3], p3 = v[(k + 2) % 3];
    const V3<R> n = cross(p1 - p3, p2 - p3);
    const V3<R> ne = cross(n, p1 - p2);
    const V3<R> Ne = normalize(ne);
    const M3<R> dNe_dne = dnormvdv(Ne, ne);
    const V3<R> dL_dNe = dL_dphi_x * (hit_p - p1);
    const V3<R> dL_dne = vecmat(dL_dNe, dNe_dne);
    const M3<R> j1 = dne_dp1(p1, p2, p3);
    const M3<R> j2 = dne_dp2(p1, p2, p3);
    const M3<R> j3 = dne_dp3(p1, p2, p3);
    const V3<R> g1 = vecmat(dL_dne, j1) - dL_dphi_x * Ne;
    const V3<R> g2 = vecmat(dL_dne, j2);
    const V3<R> g3 = vecmat(dL_dne, j3);
    add3(dtri, off + k, g1, mt);
    add3(dtri, off + (k + 1) % 3, g2, mt);
    add3(dtri, off + (k + 2) % 3, g3, mt);
  }
  {
    const V3<R> p1 = v[0], p2 = v[1], p3 = v[2];
    const V3<R> n = cross(p1 - p3, p2 - p3);
    const V3<R> Nn = normalize(n);
    const M3<R> dN_dn = dnormvdv(Nn, n);
    const V3<R> dL_dn = vecmat(dL_dnormal3D, dN_dn);
    const V3<R> g1 = vecmat(dL_dn, skew(p3 - p2));
    const V3<R> g2 = vecmat(dL_dn, skew(p1 - p3));
    const V3<R> g3 = vecmat(dL_dn, skew(p2 - p1));
    add3(dtri, off + 0, g1, mt);
    add3(dtri, off + 1, g2, mt);
    add3(dtri, off + 2, g3, mt);
  }
}

// Exact adjoint (no reference counterpart): the complete chain rule of the
// window function, written from its definition (not from backward.cu's
// partial Jacobians). nc = (B - A) x (C - A); edge k's unit normal
// en_k = s_k normalize(nc x (P_k - P_k+1)) (s_0 orients edge 0 by the
// incenter); d_k = en_k . (p - P_k); phi = max d_k; dist = en_0 . (I - A),
// I = (a A + b B + c C) / (a + b + c); phi_final = phi / dist; the face
// normal n = normalize(nc); the hit point p = o + t d with t solving
// (p - A) . nc = 0, so dt/dX = -(df/dX) / (d . nc). Inputs: dL/dphi,
// dL/ddist, dL/dn and the depth term dL/dt = dL/dD w.
template <class R>
inline void window_bwd_exact(const Inputs& in, int prim, V3<R> dir, V3<R> hit_p, const Window<R>& w, R dL_dphi,
                             R dL_ddist, V3<R> dL_dn, R dL_dt_depth, R* dtri, bool mt) {
  const int off = in.cumsum[prim];
  const V3<R> P[3] = {vert<R>(in, off), vert<R>(in, off + 1), vert<R>(in, off + 2)};
  const V3<R> e1 = P[1] - P[0], e2 = P[2] - P[0];
  const V3<R> nc = cross(e1, e2);
  V3<R> gP[3] = {mk<R>(0, 0, 0), mk<R>(0, 0, 0), mk<R>(0, 0, 0)};
  V3<R> g_nc = mk<R>(0, 0, 0);
  // unit normal of edge k, given dL/d(en_k)
  auto edge_bwd = [&](int k, V3<R> g_en) {
    const V3<R> e = P[k] - P[(k + 1) % 3];
    const V3<R> ne = cross(nc, e);
    const R len = length(ne);
    const V3<R> raw = ne * (R(1) / len);
    const R sgn = dot(raw, w.en[k]) < R(0) ? R(-1) : R(1);
    const V3<R> gr = sgn * g_en;
    const V3<R> v = (gr - raw * dot(raw, gr)) * (R(1) / len);  // dL/d(ne)
    g_nc = g_nc + cross(e, v);
    const V3<R> ge = cross(v, nc);
    gP[k] = gP[k] + ge;
    gP[(k + 1) % 3] = gP[(k + 1) % 3] - ge;
  };
  // phi = d_m at every edge at the maximum
  V3<R> g_p = mk<R>(0, 0, 0);
  for (int k = 0; k < 3; ++k) {
    if (std::fabs(w.d[k] - w.phi_max) > R(1e-6f)) continue;
    edge_bwd(k, dL_dphi * (hit_p - P[k]));
    g_p = g_p + dL_dphi * w.en[k];
    gP[k] = gP[k] - dL_dphi * w.en[k];
  }
  // dist = en_0 . (I - A)
  {
    edge_bwd(0, dL_ddist * (w.incenter - P[0]));
    const V3<R> gI = dL_ddist * w.en[0];
    gP[0] = gP[0] - gI;
    const R a = length(P[1] - P[2]), b = length(P[2] - P[0]), c = length(P[0] - P[1]), sum = a + b + c;
    const V3<R> I = w.incenter;
    gP[0] = gP[0] + (a / sum) * gI;
    gP[1] = gP[1] + (b / sum) * gI;
    gP[2] = gP[2] + (c / sum) * gI;
    const R ga = dot(gI, P[0] - I) / sum, gb = dot(gI, P[1] - I) / sum, gc = dot(gI, P[2] - I) / sum;
    gP[1] = gP[1] + (ga / a) * (P[1] - P[2]);
    gP[2] = gP[2] - (ga / a) * (P[1] - P[2]);
    gP[2] = gP[2] + (gb / b) * (P[2] - P[0]);
    gP[0] = gP[0] - (gb / b) * (P[2] - P[0]);
    gP[0] = gP[0] + (gc / c) * (P[0] - P[1]);
    gP[1] = gP[1] - (gc / c) * (P[0] - P[1]);
  }
  // face normal n = nc / |nc|
  {
    const R len = length(nc);
    const V3<R> n = nc * (R(1) / len);
    g_nc = g_nc + (dL_dn - n * dot(n, dL_dn)) * (R(1) / len);
  }
  // t from the plane, with dL/dt from the hit point and the depth
  {
    const R dL_dt = dot(g_p, dir) + dL_dt_depth;
    const V3<R> u = hit_p - P[0];
    const R s = -dL_dt / dot(dir, nc);
    const V3<R> fB = cross(e2, u), fC = cross(u, e1);
    gP[0] = gP[0] + s * (-nc - fB - fC);
    gP[1] = gP[1] + s * fB;
    gP[2] = gP[2] + s * fC;
  }
  // nc = e1 x e2
  {
    const V3<R> g1 = cross(e2, g_nc), g2 = cross(g_nc, e1);
    gP[1] = gP[1] + g1;
    gP[2] = gP[2] + g2;
    gP[0] = gP[0] - g1 - g2;
  }
  for (int k = 0; k < 3; ++k) add3(dtri, off + k, gP[k], mt);
}

// backward.cu:191-350: re-march with the forward's decisions, keeping running
// C/N/D that include the current hit, and take each hit's alpha gradient from
// the difference to the final values.
template <class R>
inline void backward_ray(const Scene& sc, const Inputs& in, int pix, const Opts& opt, const BwdIn<R>& bi,
                         BwdOut<R>& bo) {
  const int HW = in.H * in.W;
  const float* of = in.ray_o + 3 * (size_t)pix;
  const float* df = in.ray_d + 3 * (size_t)pix;
  const V3<R> o = from_f<R>(of), d = from_f<R>(df);
  const RayPre rp = ray_pre(of, df);
  const R final_depth = bi.others[pix + kDepth * HW];
  const V3<R> final_normal = mk<R>(bi.others[pix + (kNormal + 0) * HW], bi.others[pix + (kNormal + 1) * HW],
                                   bi.others[pix + (kNormal + 2) * HW]);
  R final_color[3], dL_dpixel[3];
  for (int ch = 0; ch < 3; ++ch) final_color[ch] = bi.colors[ch * HW + pix];
  for (int ch = 0; ch < 3; ++ch) dL_dpixel[ch] = (R)bi.dL_dpixels[ch * HW + pix];
  const R dL_ddepth = (R)bi.dL_dothers[kDepth * HW + pix];
  const V3<R> dL_dnormal2D = mk<R>((R)bi.dL_dothers[(kNormal + 0) * HW + pix], (R)bi.dL_dothers[(kNormal + 1) * HW + pix],
                                   (R)bi.dL_dothers[(kNormal + 2) * HW + pix]);
  float t_near, t_far;
  ray_interval(in, pix, t_near, t_far);
  // exact adjoint: middepth / distortion from their final values; the
  // distortion's alpha gradient is T_k E_k - (2 dist_f - S_k) / (1 - alpha_k)
  // with E_k = t_k^2 W_f - 2 t_k B_f + C_f (C_f = (dist_f + B_f^2) / W_f) and
  // S_k = sum_{i<=k} w_i E_i; its t gradient is 2 w_k (t_k W_f - B_f)
  const R g_mid = (R)bi.dL_dothers[kMidDepth * HW + pix], g_dist = (R)bi.dL_dothers[kDistortion * HW + pix];
  const R W_f = bi.others[pix + kAlphaOff * HW], dist_f = bi.others[pix + kDistortion * HW];
  const R C_f = W_f > R(0) ? (dist_f + final_depth * final_depth) / W_f : R(0);
  R S = 0;
  bool mid_seen = false;
  R C[3] = {0, 0, 0}, N[3] = {0, 0, 0};
  R D = 0, T = 1;
  march(
      sc, rp, opt,
      [&](uint32_t prim, float t) -> bool {
        const V3<R> hp = hit_point(in, (int)prim, o, d, t, opt);
        const R hit_t = hit_dist(in, (int)prim, o, d, t, opt);
        const Window<R> w = window_fn(in, (int)prim, hp);
        const R opacity = (R)in.opacities[prim];
        const R alpha = std::fmin(R(kAlphaMax), opacity * w.Cx);
        if (alpha < R(kAlphaMin)) return false;
        const R test_T = T * (R(1) - alpha);
        if (test_T < R(kTMin)) return true;
        const R bw = alpha * T;
        bool clamped[3];
        const V3<R> col = sh_color(in, (int)prim, d, clamped);
        C[0] += col.x * bw;
        C[1] += col.y * bw;
        C[2] += col.z * bw;
        N[0] += w.n.x * bw;
        N[1] += w.n.y * bw;
        N[2] += w.n.z * bw;
        D += bw * hit_t;
        R dL_dcolor[3];
        const R c[3] = {col.x, col.y, col.z};
        R dL_dalpha = R(0);
        const R inv_1_alpha = R(1) / (R(1) - alpha);
        for (int ch = 0; ch < 3; ++ch) {
          const R g = dL_dpixel[ch];
          dL_dcolor[ch] = g * bw;
          dL_dalpha += g * (T * c[ch] - (final_color[ch] - C[ch]) * inv_1_alpha);
        }
        dL_dalpha += dL_ddepth * (T * hit_t - (final_depth - D) * inv_1_alpha);
        const V3<R> Nf = mk<R>(N[0], N[1], N[2]);
        dL_dalpha += sum3(vmul(dL_dnormal2D, T * w.n - (final_normal - Nf) * inv_1_alpha));
        R dL_dt_extra = dL_ddepth * bw;
        if (opt.exact_adjoint) {
          const R E = hit_t * hit_t * W_f - R(2) * hit_t * final_depth + C_f;
          S += bw * E;
          dL_dalpha += g_dist * (T * E - (R(2) * dist_f - S) * inv_1_alpha);
          dL_dt_extra += g_dist * R(2) * bw * (hit_t * W_f - final_depth);
          if (!mid_seen && test_T <= R(0.5)) {
            mid_seen = true;
            dL_dt_extra += g_mid;
          }
        }
        // the exact adjoint honours the alpha clamp (no gradient through a
        // clamped alpha); the reference differentiates through it
        const bool live = !opt.exact_adjoint || opacity * w.Cx < R(kAlphaMax);
        const R dL_dC = live ? opacity * dL_dalpha : R(0);
        if (live) atomic_add(&bo.dopac[prim], dL_dalpha * w.Cx, opt.mt);
        if (w.phi_final > R(0)) {
          atomic_add(&bo.dsigma[prim], dL_dC * w.Cx * fast_log<R>(w.phi_final), opt.mt);
        }
        const R dL_dphi_x = (R)in.sigma[prim] / w.phi_max * dL_dC * w.Cx;
        const V3<R> dL_dnormal = dL_dnormal2D * bw;
        if (opt.exact_adjoint) {
          const R dL_ddist = -dL_dC * (R)in.sigma[prim] * w.Cx / w.dist;
          window_bwd_exact(in, (int)prim, d, hp, w, dL_dphi_x, dL_ddist, dL_dnormal, dL_dt_extra, bo.dtri, opt.mt);
        } else {
          window_bwd(in, (int)prim, hp, dL_dphi_x, w.phi_max, w.d, dL_dnormal, bo.dtri, opt.mt);
        }
        if (in.colors)
          add3(bo.dcolors, (int)prim, mk<R>(dL_dcolor[0], dL_dcolor[1], dL_dcolor[2]), opt.mt);
        else
          sh_color_bwd(in, (int)prim, d, clamped, dL_dcolor, bo.dsh, opt.mt);
        T = test_T;
        return false;
      },
      [](const Hit&) {}, t_near, t_far);
}

// ---------------------------------------------------------------- secondary rays
// Secondary-ray passes with per-triangle dielectric interfaces and an
// environment map. No reference counterpart (the reference bends rays only
// at one analytic sphere, reflect.cu / refract.cu / envlight.cu); these are
// the semantics the GPU's ray-queue passes implement:
//  * every ray marches as forward.cu does (window function, alpha, the
//    1/255 floor, the 1e-4 transmittance cut-off, SH colour, front-to-back
//    compositing); its radiance is L = sum_i w_i c_i + T_final env(d), with
//    a lat-long environment map in place of bg;
//  * the first blended hit of a ray of depth < max_depth on a triangle of
//    material 1 spawns a reflected and (unless totally reflected) a
//    refracted ray from the exact hit point (FP64 plane solve), and that
//    hit's colour is F L(reflected) + (1 - F) L(refracted) instead of its SH
//    colour (Schlick's Fresnel term with the triangle's IOR; set-up in FP64
//    without contraction, so GPU and CPU spawn the same FP32 rays);
//  * pixel colour = L(primary); alpha, normal, density, scaling and
//    max_blending come from the primary ray only;
//  * adjoint: the same march for every ray of the tree with upstream
//    gradient tau dL/dpixel, tau the product of the spawn weights (w F or
//    w (1 - F)) along the path; the spawn geometry (directions, F) is held
//    constant, as the reference's vertex gradient ignores how hit points
//    move.
struct SecInputs {
  const int* material = nullptr;  // [P], 1 = dielectric interface
  const float* ior = nullptr;     // [P]
  const float* env = nullptr;     // [env_h][env_w][3]
  int env_h = 0, env_w = 0;
  int max_depth = 2;
  // test hook: per-triangle IOR used for the Fresnel share F only (the bent
  // directions keep `ior`), so that finite differences over it measure the
  // adjoint's IOR gradient, which holds the directions constant
  const float* ior_fresnel = nullptr;
};

// Lat-long lookup: longitude atan2(d.z, d.x) over the columns (wrapping),
// colatitude acos(d.y) over the rows (clamped), bilinear between texel
// centres.
template <class R>
inline V3<R> env_lookup(const SecInputs& s, V3<R> d) {
  const double kPi = 3.14159265358979323846;
  const double dx = d.x, dy = d.y, dz = d.z;
  const double len = std::sqrt(dx * dx + dy * dy + dz * dz);
  const double u = std::atan2(dz, dx) / (2.0 * kPi) + 0.5;
  const double v = std::acos(std::fmax(-1.0, std::fmin(1.0, dy / len))) / kPi;
  const double fx = u * s.env_w - 0.5, fy = v * s.env_h - 0.5;
  const double x0f = std::floor(fx), y0f = std::floor(fy);
  const double ax = fx - x0f, ay = fy - y0f;
  const int W = s.env_w, H = s.env_h;
  const int x0 = (((int)x0f % W) + W) % W, x1 = (x0 + 1) % W;
  const int y0 = std::max(0, std::min(H - 1, (int)y0f)), y1 = std::max(0, std::min(H - 1, (int)y0f + 1));
  double out[3];
  for (int c = 0; c < 3; ++c) {
    auto tx = [&](int x, int y) { return (double)s.env[((size_t)y * W + x) * 3 + c]; };
    out[c] = (1 - ay) * ((1 - ax) * tx(x0, y0) + ax * tx(x1, y0)) + ay * ((1 - ax) * tx(x0, y1) + ax * tx(x1, y1));
  }
  return V3<R>{(R)out[0], (R)out[1], (R)out[2]};
}

// Adjoint of T env(d): each of the four texels of the lookup gets
// gL T (bilinear weight).
template <class R>
inline void env_lookup_bwd(const SecInputs& s, V3<R> d, R T, const R gL[3], R* denv, bool mt) {
  const double kPi = 3.14159265358979323846;
  const double dx = d.x, dy = d.y, dz = d.z;
  const double len = std::sqrt(dx * dx + dy * dy + dz * dz);
  const double u = std::atan2(dz, dx) / (2.0 * kPi) + 0.5;
  const double v = std::acos(std::fmax(-1.0, std::fmin(1.0, dy / len))) / kPi;
  const double fx = u * s.env_w - 0.5, fy = v * s.env_h - 0.5;
  const double x0f = std::floor(fx), y0f = std::floor(fy);
  const double ax = fx - x0f, ay = fy - y0f;
  const int W = s.env_w, H = s.env_h;
  const int x0 = (((int)x0f % W) + W) % W, x1 = (x0 + 1) % W;
  const int y0 = std::max(0, std::min(H - 1, (int)y0f)), y1 = std::max(0, std::min(H - 1, (int)y0f + 1));
  const int xs[4] = {x0, x1, x0, x1}, ys[4] = {y0, y0, y1, y1};
  const double wt[4] = {(1 - ay) * (1 - ax), (1 - ay) * ax, ay * (1 - ax), ay * ax};
  for (int k = 0; k < 4; ++k)
    for (int c = 0; c < 3; ++c)
      atomic_add(&denv[((size_t)ys[k] * W + xs[k]) * 3 + c], gL[c] * T * R(wt[k]), mt);
}

inline double fresnel_ior(const SecInputs& s, int prim) {
  return (double)(s.ior_fresnel ? s.ior_fresnel[prim] : s.ior[prim]);
}

struct Spawn {
  float o[3];   // exact hit point
  float r[3];   // reflected direction
  float t[3];   // refracted direction (if refracts)
  bool refracts;
  double F;     // reflected share
  double dF_dior;  // its derivative in the IOR, directions held constant
};

// Reflected / refracted rays at the hit of ray (of, df) on triangle prim.
inline Spawn spawn_rays(const Inputs& in, int prim, const float* of, const float* df, double ior, double ior_F) {
  const int off = in.cumsum[prim];
  const V3<double> A = from_f<double>(in.verts + 3 * (size_t)off);
  const V3<double> B = from_f<double>(in.verts + 3 * (size_t)(off + 1));
  const V3<double> C = from_f<double>(in.verts + 3 * (size_t)(off + 2));
  const V3<double> o = from_f<double>(of), d = from_f<double>(df);
  const V3<double> nc = cross(B - A, C - A);
  const double te = dot(A - o, nc) / dot(d, nc);
  const V3<double> x = o + te * d;
  const V3<double> n = nc / std::sqrt(dot(nc, nc));
  const V3<double> du = d / std::sqrt(dot(d, d));
  const double cosi = dot(du, n);
  const bool entering = cosi < 0.0;
  const V3<double> nf = entering ? n : -n;
  const double c = entering ? -cosi : cosi;
  const double ei = entering ? 1.0 : ior, et = entering ? ior : 1.0;
  const double eta = ei / et;
  // Schlick's r0 is the same on both sides of the interface
  const double qF = (ior_F - 1.0) / (ior_F + 1.0);
  const double r0 = qF * qF;
  const double k = 1.0 - eta * eta * (1.0 - c * c);
  Spawn sp;
  const V3<double> r = du + (2.0 * c) * nf;
  sp.refracts = k >= 0.0;
  V3<double> t = du;
  if (sp.refracts) {
    const double m = 1.0 - c;
    const double m2 = m * m;
    sp.F = r0 + (1.0 - r0) * (m2 * m2 * m);
    // dr0/dior = 4 (ior - 1) / (ior + 1)^3; F moves by (1 - m^5) of it
    sp.dF_dior = 4.0 * (ior_F - 1.0) / ((ior_F + 1.0) * (ior_F + 1.0) * (ior_F + 1.0)) * (1.0 - m2 * m2 * m);
    t = eta * du + (eta * c - std::sqrt(k)) * nf;
  } else {
    sp.F = 1.0;
    sp.dF_dior = 0.0;
  }
  const double xs[3] = {x.x, x.y, x.z}, rs[3] = {r.x, r.y, r.z}, ts[3] = {t.x, t.y, t.z};
  for (int i = 0; i < 3; ++i) {
    sp.o[i] = (float)xs[i];
    sp.r[i] = (float)rs[i];
    sp.t[i] = (float)ts[i];
  }
  return sp;
}

// Radiance of one ray of the tree (recursive over its spawned rays). For the
// primary ray (out != nullptr) also the side outputs of pixel pix.
template <class R>
inline V3<R> sec_radiance(const Scene& sc, const Inputs& in, const SecInputs& s, const float* of, const float* df,
                          int depth, const Opts& opt, FwdOut<R>* out, int pix, RayRecord* rec) {
  const V3<R> o = from_f<R>(of), d = from_f<R>(df);
  const RayPre rp = ray_pre(of, df);
  V3<R> C = mk<R>(0, 0, 0), N = mk<R>(0, 0, 0);
  R T = 1;
  bool spawned = false;
  march(
      sc, rp, opt,
      [&](uint32_t prim, float t) -> bool {
        const V3<R> hp = hit_point(in, (int)prim, o, d, t, opt);
        const Window<R> w = window_fn(in, (int)prim, hp);
        const R alpha = std::fmin(R(kAlphaMax), (R)in.opacities[prim] * w.Cx);
        if (rec) rec->near((double)alpha, (double)kAlphaMin);
        if (alpha < R(kAlphaMin)) return false;
        const R test_T = T * (R(1) - alpha);
        if (rec) rec->near((double)test_T, (double)kTMin);
        if (test_T < R(kTMin)) return true;
        const R bw = alpha * T;
        if (out) {
          out->density[prim] = R(1);
          compute_scaling(in, (int)prim, o, out->scaling, opt.mt);
          atomic_max(&out->max_blending[prim], bw, opt.mt);
          N = N + w.n * bw;
        }
        V3<R> col;
        if (!spawned && depth < s.max_depth && s.material[prim] == 1) {
          spawned = true;
          const Spawn sp = spawn_rays(in, (int)prim, of, df, (double)s.ior[prim], fresnel_ior(s, (int)prim));
          const V3<R> Lr = sec_radiance<R>(sc, in, s, sp.o, sp.r, depth + 1, opt, nullptr, pix, rec);
          const V3<R> Lt = sp.refracts ? sec_radiance<R>(sc, in, s, sp.o, sp.t, depth + 1, opt, nullptr, pix, rec)
                                       : mk<R>(0, 0, 0);
          col = R(sp.F) * Lr + R(1.0 - sp.F) * Lt;
        } else {
          col = sh_color(in, (int)prim, d, nullptr);
        }
        C = C + col * bw;
        T = test_T;
        return false;
      },
      [&](const Hit& h) {
        if (rec && out) rec->add(h);
      });
  const V3<R> L = C + T * env_lookup<R>(s, d);
  if (out) {
    const int HW = in.H * in.W;
    out->color[pix] = L.x;
    out->color[HW + pix] = L.y;
    out->color[2 * HW + pix] = L.z;
    out->others[pix + kDepth * HW] = R(0);
    out->others[pix + kAlphaOff * HW] = R(1) - T;
    out->others[pix + (kNormal + 0) * HW] = N.x;
    out->others[pix + (kNormal + 1) * HW] = N.y;
    out->others[pix + (kNormal + 2) * HW] = N.z;
    out->others[pix + kMidDepth * HW] = R(0);
    out->others[pix + kDistortion * HW] = R(0);
  }
  return L;
}

// Adjoint of one ray of the tree with upstream dL/dL = gL (and, for the
// primary ray, dL/d(depth, normal) and its final side outputs).
template <class R>
inline void sec_backward(const Scene& sc, const Inputs& in, const SecInputs& s, const float* of, const float* df,
                         int depth, const Opts& opt, const R gL[3], const R* g_others, const R* f_others,
                         BwdOut<R>& bo) {
  const V3<R> o = from_f<R>(of), d = from_f<R>(df);
  const RayPre rp = ray_pre(of, df);
  const V3<R> Lf = sec_radiance<R>(sc, in, s, of, df, depth, opt, nullptr, 0, nullptr);
  const R final_color[3] = {Lf.x, Lf.y, Lf.z};
  const R gD = g_others ? g_others[0] : R(0);
  const V3<R> gN = g_others ? mk<R>(g_others[1], g_others[2], g_others[3]) : mk<R>(0, 0, 0);
  const R final_depth = f_others ? f_others[0] : R(0);
  const V3<R> final_normal = f_others ? mk<R>(f_others[1], f_others[2], f_others[3]) : mk<R>(0, 0, 0);
  R C[3] = {0, 0, 0};
  V3<R> N = mk<R>(0, 0, 0);
  R D = 0, T = 1;
  bool spawned = false;
  march(
      sc, rp, opt,
      [&](uint32_t prim, float t) -> bool {
        const V3<R> hp = hit_point(in, (int)prim, o, d, t, opt);
        const R hit_t = hit_dist(in, (int)prim, o, d, t, opt);
        const Window<R> w = window_fn(in, (int)prim, hp);
        const R opacity = (R)in.opacities[prim];
        const R alpha = std::fmin(R(kAlphaMax), opacity * w.Cx);
        if (alpha < R(kAlphaMin)) return false;
        const R test_T = T * (R(1) - alpha);
        if (test_T < R(kTMin)) return true;
        const R bw = alpha * T;
        bool clamped[3] = {false, false, false};
        V3<R> col;
        bool spawn = false;
        if (!spawned && depth < s.max_depth && s.material[prim] == 1) {
          spawned = spawn = true;
          const Spawn sp = spawn_rays(in, (int)prim, of, df, (double)s.ior[prim], fresnel_ior(s, (int)prim));
          const V3<R> Lr = sec_radiance<R>(sc, in, s, sp.o, sp.r, depth + 1, opt, nullptr, 0, nullptr);
          V3<R> Lt = mk<R>(0, 0, 0);
          const R gr[3] = {gL[0] * bw * R(sp.F), gL[1] * bw * R(sp.F), gL[2] * bw * R(sp.F)};
          sec_backward<R>(sc, in, s, sp.o, sp.r, depth + 1, opt, gr, nullptr, nullptr, bo);
          if (sp.refracts) {
            Lt = sec_radiance<R>(sc, in, s, sp.o, sp.t, depth + 1, opt, nullptr, 0, nullptr);
            const R ft = R(1.0 - sp.F);
            const R gt[3] = {gL[0] * bw * ft, gL[1] * bw * ft, gL[2] * bw * ft};
            sec_backward<R>(sc, in, s, sp.o, sp.t, depth + 1, opt, gt, nullptr, nullptr, bo);
          }
          col = R(sp.F) * Lr + R(1.0 - sp.F) * Lt;
          if (bo.dior && sp.refracts) {
            const R dL_dF = bw * (gL[0] * (Lr.x - Lt.x) + gL[1] * (Lr.y - Lt.y) + gL[2] * (Lr.z - Lt.z));
            atomic_add(&bo.dior[prim], dL_dF * R(sp.dF_dior), opt.mt);
          }
        } else {
          col = sh_color(in, (int)prim, d, clamped);
        }
        const R c[3] = {col.x, col.y, col.z};
        for (int ch = 0; ch < 3; ++ch) C[ch] += c[ch] * bw;
        N = N + w.n * bw;
        D += bw * hit_t;
        const R inv_1_alpha = R(1) / (R(1) - alpha);
        R dL_dalpha = R(0);
        R dL_dcolor[3];
        for (int ch = 0; ch < 3; ++ch) {
          dL_dcolor[ch] = gL[ch] * bw;
          dL_dalpha += gL[ch] * (T * c[ch] - (final_color[ch] - C[ch]) * inv_1_alpha);
        }
        if (g_others) {
          // the exact adjoint differentiates the outputs the passes compute:
          // depth is 0 there, so it has no gradient (the reference-style
          // adjoint keeps backward.cu's depth term)
          if (!opt.exact_adjoint) dL_dalpha += gD * (T * hit_t - (final_depth - D) * inv_1_alpha);
          dL_dalpha += sum3(vmul(gN, T * w.n - (final_normal - N) * inv_1_alpha));
        }
        const bool live = !opt.exact_adjoint || opacity * w.Cx < R(kAlphaMax);
        const R dL_dC = live ? opacity * dL_dalpha : R(0);
        if (live) atomic_add(&bo.dopac[prim], dL_dalpha * w.Cx, opt.mt);
        if (w.phi_final > R(0)) atomic_add(&bo.dsigma[prim], dL_dC * w.Cx * fast_log<R>(w.phi_final), opt.mt);
        const R dL_dphi_x = (R)in.sigma[prim] / w.phi_max * dL_dC * w.Cx;
        if (opt.exact_adjoint) {  // full chain rule; the spawn geometry stays constant
          const R dL_ddist = -dL_dC * (R)in.sigma[prim] * w.Cx / w.dist;
          window_bwd_exact(in, (int)prim, d, hp, w, dL_dphi_x, dL_ddist, gN * bw, R(0), bo.dtri, opt.mt);
        } else {
          window_bwd(in, (int)prim, hp, dL_dphi_x, w.phi_max, w.d, gN * bw, bo.dtri, opt.mt);
        }
        if (!spawn) sh_color_bwd(in, (int)prim, d, clamped, dL_dcolor, bo.dsh, opt.mt);
        T = test_T;
        return false;
      },
      [](const Hit&) {});
  if (bo.denv) env_lookup_bwd<R>(s, d, T, gL, bo.denv, opt.mt);
}

}  // namespace tto