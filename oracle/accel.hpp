// Test infrastructure (oracle): ray/triangle intersection and a CPU bounding
// volume hierarchy that enumerates every triangle hit inside a ray interval.
//
// The reference delegates both to OptiX 7.7 (optixAccelBuild in
// tritracer/pipeline.cpp:206-265 and the built-in triangle intersector reached
// through optixTrace in tritracer/closestk.h:17-106). Those are closed driver
// code, so this file restates them from published methods:
//  * intersection: the watertight, non-culling test of Woop, Benthin and Wald,
//    "Watertight Ray/Triangle Intersection", JCGT 2(1), 2013, evaluated in FP32
//    (as OptiX does) with the paper's FP64 fall-back when a scaled barycentric
//    is exactly zero. Every operation is written out so that the CUDA kernels,
//    which evaluate the same expression tree with round-to-nearest intrinsics
//    and no contraction, produce bit-identical t values;
//  * acceleration: a median-split binary BVH with FP64 slab tests padded by a
//    relative margin, so it never culls a box a reported hit lies in.
// Interval semantics follow optixTrace's [tmin, tmax] (closed at both ends) by
// default; `tmin_inclusive = false` gives the open lower bound instead.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace tto {

struct RayPre {
  float o[3];
  float d[3];
  int kx, ky, kz;
  float Sx, Sy, Sz;
};

// Per-ray set-up of the watertight test: kz is the axis of largest |d|, and
// kx/ky are swapped when d[kz] < 0 to keep the winding (Woop et al. 2013, Fig. 1).
inline RayPre ray_pre(const float o[3], const float d[3]) {
  RayPre r;
  for (int i = 0; i < 3; ++i) {
    r.o[i] = o[i];
    r.d[i] = d[i];
  }
  const float ax = std::fabs(d[0]), ay = std::fabs(d[1]), az = std::fabs(d[2]);
  int kz = (ax > ay) ? ((ax > az) ? 0 : 2) : ((ay > az) ? 1 : 2);
  int kx = kz + 1;
  if (kx == 3) kx = 0;
  int ky = kx + 1;
  if (ky == 3) ky = 0;
  if (d[kz] < 0.0f) std::swap(kx, ky);
  r.kx = kx;
  r.ky = ky;
  r.kz = kz;
  r.Sx = d[kx] / d[kz];
  r.Sy = d[ky] / d[kz];
  r.Sz = 1.0f / d[kz];
  return r;
}

// Returns true and the hit distance t when the ray's line crosses the triangle
// (either winding). Range checks on t are left to the caller.
inline bool isect_tri(const RayPre& r, const float* v0, const float* v1, const float* v2, float* t_out) {
  const float A[3] = {v0[0] - r.o[0], v0[1] - r.o[1], v0[2] - r.o[2]};
  const float B[3] = {v1[0] - r.o[0], v1[1] - r.o[1], v1[2] - r.o[2]};
  const float C[3] = {v2[0] - r.o[0], v2[1] - r.o[1], v2[2] - r.o[2]};
  const float Ax = A[r.kx] - r.Sx * A[r.kz];
  const float Ay = A[r.ky] - r.Sy * A[r.kz];
  const float Bx = B[r.kx] - r.Sx * B[r.kz];
  const float By = B[r.ky] - r.Sy * B[r.kz];
  const float Cx = C[r.kx] - r.Sx * C[r.kz];
  const float Cy = C[r.ky] - r.Sy * C[r.kz];
  float U = Cx * By - Cy * Bx;
  float V = Ax * Cy - Ay * Cx;
  float W = Bx * Ay - By * Ax;
  if (U == 0.0f || V == 0.0f || W == 0.0f) {
    // Products of two floats are exact in FP64, so the sign of each edge
    // function is exact here (the paper's fall-back).
    U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
    V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
    W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
  }
  if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
  const float det = (U + V) + W;
  if (det == 0.0f) return false;
  const float Az = r.Sz * A[r.kz];
  const float Bz = r.Sz * B[r.kz];
  const float Cz = r.Sz * C[r.kz];
  const float T = (U * Az + V * Bz) + W * Cz;
  *t_out = T / det + 0.0f;  // a -0 distance (ray starting on the plane) counts as +0, like the GPU's keys
  return true;
}

// Closed/open interval test on a candidate hit distance.
inline bool t_in_range(float t, float tmin, float tmax, bool tmin_inclusive) {
  const bool lo_ok = tmin_inclusive ? (t >= tmin) : (t > tmin);
  return lo_ok && (t <= tmax);
}

struct Scene {
  // vertex positions, 3 floats per vertex; triangle i uses vertices
  // cumsum[i], cumsum[i]+1, cumsum[i]+2 (tritracer/tracer.cpp:58-64)
  const float* verts = nullptr;
  const int* cumsum = nullptr;
  int P = 0;

  struct Node {
    float lo[3], hi[3];
    int left = -1, right = -1;  // children (internal) or -1
    int first = 0, count = 0;   // leaf range in `order`
  };
  std::vector<Node> nodes;
  std::vector<int> order;

  const float* vtx(int prim, int k) const { return verts + 3 * (size_t)(cumsum[prim] + k); }

  void build(const float* v, const int* cs, int p) {
    verts = v;
    cumsum = cs;
    P = p;
    nodes.clear();
    order.resize(P);
    for (int i = 0; i < P; ++i) order[i] = i;
    std::vector<float> cen((size_t)3 * P), blo((size_t)3 * P), bhi((size_t)3 * P);
    for (int i = 0; i < P; ++i) {
      for (int a = 0; a < 3; ++a) {
        float x0 = vtx(i, 0)[a], x1 = vtx(i, 1)[a], x2 = vtx(i, 2)[a];
        blo[3 * i + a] = std::min(x0, std::min(x1, x2));
        bhi[3 * i + a] = std::max(x0, std::max(x1, x2));
        cen[3 * i + a] = 0.5f * (blo[3 * i + a] + bhi[3 * i + a]);
      }
    }
    if (P == 0) return;
    nodes.reserve((size_t)2 * P);
    struct Item {
      int node, first, count;
    };
    std::vector<Item> work;
    nodes.push_back(Node());
    work.push_back({0, 0, P});
    while (!work.empty()) {
      Item it = work.back();
      work.pop_back();
      Node nd;
      for (int a = 0; a < 3; ++a) {
        nd.lo[a] = INFINITY;
        nd.hi[a] = -INFINITY;
      }
      float clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
      for (int j = it.first; j < it.first + it.count; ++j) {
        int p = order[j];
        for (int a = 0; a < 3; ++a) {
          nd.lo[a] = std::min(nd.lo[a], blo[3 * p + a]);
          nd.hi[a] = std::max(nd.hi[a], bhi[3 * p + a]);
          clo[a] = std::min(clo[a], cen[3 * p + a]);
          chi[a] = std::max(chi[a], cen[3 * p + a]);
        }
      }
      if (it.count <= 4) {
        nd.first = it.first;
        nd.count = it.count;
        nodes[it.node] = nd;
        continue;
      }
      int axis = 0;
      float ext = chi[0] - clo[0];
      for (int a = 1; a < 3; ++a)
        if (chi[a] - clo[a] > ext) {
          ext = chi[a] - clo[a];
          axis = a;
        }
      int mid = it.first + it.count / 2;
      std::nth_element(order.begin() + it.first, order.begin() + mid, order.begin() + it.first + it.count,
                       [&](int a, int b) { return cen[3 * a + axis] < cen[3 * b + axis]; });
      nd.left = (int)nodes.size();
      nodes.push_back(Node());
      nd.right = (int)nodes.size();
      nodes.push_back(Node());
      nodes[it.node] = nd;
      work.push_back({nd.right, mid, it.first + it.count - mid});
      work.push_back({nd.left, it.first, mid - it.first});
    }
  }

  // FP64 slab test of `nd` against [tlo, thi], padded by a relative margin.
  static bool box_overlaps(const Node& nd, const RayPre& r, double tlo, double thi) {
    double t0 = -INFINITY, t1 = INFINITY;
    for (int a = 0; a < 3; ++a) {
      const double o = r.o[a], d = r.d[a];
      if (d == 0.0) {
        if (o < nd.lo[a] || o > nd.hi[a]) return false;
        continue;
      }
      double ta = (nd.lo[a] - o) / d, tb = (nd.hi[a] - o) / d;
      if (ta > tb) std::swap(ta, tb);
      t0 = std::max(t0, ta);
      t1 = std::min(t1, tb);
    }
    const double pad = 1e-5 * (std::fabs(t0) + std::fabs(t1)) + 1e-9;
    t0 -= pad;
    t1 += pad;
    return t0 <= t1 && t1 >= tlo && t0 <= thi;
  }

  // Calls fn(prim, t) for every triangle hit with t in the interval; fn returns
  // the (possibly shrunk) upper bound, mirroring an any-hit program that
  // accepts or ignores each candidate.
  template <class Fn>
  void for_each_hit(const RayPre& r, float tmin, float tmax, bool tmin_inclusive, Fn&& fn) const {
    if (nodes.empty()) return;
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    float tcur = tmax;
    while (sp > 0) {
      const Node& nd = nodes[stack[--sp]];
      if (!box_overlaps(nd, r, tmin, tcur)) continue;
      if (nd.left < 0) {
        for (int j = nd.first; j < nd.first + nd.count; ++j) {
          const int p = order[j];
          float t;
          if (!isect_tri(r, vtx(p, 0), vtx(p, 1), vtx(p, 2), &t)) continue;
          if (!t_in_range(t, tmin, tcur, tmin_inclusive)) continue;
          tcur = fn(p, t, tcur);
        }
      } else {
        stack[sp++] = nd.right;
        stack[sp++] = nd.left;
      }
    }
  }
};

}  // namespace tto
