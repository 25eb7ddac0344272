// Trace kernels: the k-closest-hit forward pass and its adjoint.
//
// Replaces the reference's OptiX programs tritracer/forward.cu (raygen
// :161-215, chunk loop :76-155), tritracer/closestk.h (k-closest query) and
// tritracer/backward.cu (adjoint :191-391).
//
// Shape of the kernels:
//  * persistent: every warp pulls 8x4-pixel tiles from an atomic counter until
//    the image is done, so rays of very different depth complexity balance;
//  * one ray per thread; the traversal stack (node reference + entry distance)
//    lives in shared memory, strided by the block size (no bank conflicts);
//  * k-buffer: 16 (t, primitive) pairs packed as 64-bit keys in registers,
//    inserted by a branch-free compare-exchange chain;
//  * the chunked march of the reference is reproduced exactly on top of the
//    key stream: after every 16th visited hit the next query starts AT the
//    last hit's t (closed interval, optixTrace) or strictly after it;
//  * per hit, the window function runs in FP64 from the plane intersection
//    (the FP32 hit point loses ~4 digits on small triangles far from the
//    camera); SH, compositing and the side outputs are FP32 like the
//    reference; the adjoint re-traverses instead of storing hit lists.
#include <cfloat>

#include "trace.cuh"

namespace tt {
namespace {

constexpr int kMaxChunks = 1 << 20;   // bound on re-traces per ray
constexpr int kMaxSteps = 1 << 24;    // bound on stack pops per query

struct Stack {
  uint32_t* ref;
  float* tn;
  int stride;
  __device__ __forceinline__ void put(int i, uint32_t r, float t) {
    ref[i * stride] = r;
    tn[i * stride] = t;
  }
};

__device__ __forceinline__ void kb_insert(unsigned long long (&kb)[kChunk], unsigned long long key) {
#pragma unroll
  for (int i = 0; i < kChunk; ++i) {
    const unsigned long long cur = kb[i];
    const bool lt = key < cur;
    kb[i] = lt ? key : cur;
    key = lt ? cur : key;
  }
}

// The kChunk smallest hit keys >= key_min (t <= far) along the ray, in
// ascending order, EMPTY-padded. If the stack overflowed, subtrees were
// dropped and t_drop is the smallest entry distance among them: only keys with
// t < t_drop are then guaranteed.
__device__ __forceinline__ void query(const BvhView& bvh, const RayW& r, unsigned long long key_min,
                                      unsigned long long (&kb)[kChunk], Stack st, float& t_drop, int* status) {
#pragma unroll
  for (int i = 0; i < kChunk; ++i) kb[i] = kEmptyKey;
  t_drop = INFINITY;
  if (!bvh.has_root) return;
  const float t_lo = key_t(key_min);
  int sp = 0;
  st.put(sp++, 0u, t_lo);
  int steps = 0;
  while (sp > 0) {
    if (++steps > kMaxSteps) {
      atomicOr(status, kStatusTimeout);
      break;
    }
    --sp;
    const uint32_t ref = st.ref[sp * st.stride];
    const float tn = st.tn[sp * st.stride];
    const float tmax = (kb[kChunk - 1] != kEmptyKey) ? key_t(kb[kChunk - 1]) : kFar;
    if (tn > tmax) continue;
    if (ref_is_leaf(ref)) {
      const uint32_t first = leaf_first(ref), cnt = leaf_count(ref);
      for (uint32_t j = 0; j < cnt; ++j) {
        const float4* tr = bvh.tris + 3 * (size_t)(first + j);
        const float4 a = __ldg(tr), b = __ldg(tr + 1), c = __ldg(tr + 2);
        float t;
        if (!isect_tri(r, a, b, c, t)) continue;
        const float tm = (kb[kChunk - 1] != kEmptyKey) ? key_t(kb[kChunk - 1]) : kFar;
        if (!(t >= t_lo) || !(t <= tm)) continue;
        const unsigned long long key = hit_key(t, (uint32_t)__float_as_int(a.w));
        if (key >= key_min && key < kb[kChunk - 1]) kb_insert(kb, key);
      }
      continue;
    }
    const float4* nd = bvh.nodes + (size_t)ref * kNodeF4;
    float lox[8], hix[8], loy[8], hiy[8], loz[8], hiz[8];
    uint32_t cref[8];
    {
      float4 v;
#define TT_LD8(arr, word)                                                           \
  v = __ldg(nd + (word));                                                           \
  arr[0] = v.x; arr[1] = v.y; arr[2] = v.z; arr[3] = v.w;                           \
  v = __ldg(nd + (word) + 1);                                                       \
  arr[4] = v.x; arr[5] = v.y; arr[6] = v.z; arr[7] = v.w;
      TT_LD8(lox, 0) TT_LD8(hix, 2) TT_LD8(loy, 4) TT_LD8(hiy, 6) TT_LD8(loz, 8) TT_LD8(hiz, 10)
#undef TT_LD8
      v = __ldg(nd + 12);
      cref[0] = __float_as_uint(v.x); cref[1] = __float_as_uint(v.y);
      cref[2] = __float_as_uint(v.z); cref[3] = __float_as_uint(v.w);
      v = __ldg(nd + 13);
      cref[4] = __float_as_uint(v.x); cref[5] = __float_as_uint(v.y);
      cref[6] = __float_as_uint(v.z); cref[7] = __float_as_uint(v.w);
    }
    float tnear[8];
    bool hit[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const float x0 = fmaf(lox[c], r.ix, -r.oix), x1 = fmaf(hix[c], r.ix, -r.oix);
      const float y0 = fmaf(loy[c], r.iy, -r.oiy), y1 = fmaf(hiy[c], r.iy, -r.oiy);
      const float z0 = fmaf(loz[c], r.iz, -r.oiz), z1 = fmaf(hiz[c], r.iz, -r.oiz);
      const float tn0 = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fmaxf(fminf(z0, z1), t_lo));
      const float tf0 = fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fminf(fmaxf(z0, z1), tmax));
      // padded by a few ulps so a rounded slab test never culls a reported hit
      tnear[c] = tn0 * 0.9999990f;
      hit[c] = (cref[c] != kEmptyRef) && (tnear[c] <= tf0 * 1.0000010f);
    }
    int nhit = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) nhit += hit[c] ? 1 : 0;
    const int avail = kStackDepth - sp;
    const int npush = nhit < avail ? nhit : avail;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      if (!hit[c]) continue;
      int rank = 0;
#pragma unroll
      for (int c2 = 0; c2 < 8; ++c2) {
        if (c2 == c) continue;
        const bool before = hit[c2] && (tnear[c2] < tnear[c] || (tnear[c2] == tnear[c] && c2 < c));
        rank += before ? 1 : 0;
      }
      if (rank < npush)
        st.put(sp + npush - 1 - rank, cref[c], tnear[c]);  // nearest on top
      else
        t_drop = fminf(t_drop, tnear[c]);
    }
    sp += npush;
  }
}

// ---------------------------------------------------------------- shading
struct Geom {
  float Cx;
  float3 n;
  double phi_final, phi_max;
  double d[3];
  d3 hp;
  double t;
};

// Window function of tritracer/common.h:57-114 in FP64, evaluated at the
// exact ray/plane intersection.
__device__ __forceinline__ Geom window_fp64(float4 a, float4 b, float4 c, const RayW& r, float sigma) {
  Geom g;
  const d3 A = tod(a), B = tod(b), C = tod(c);
  const d3 o = mkd(r.ox, r.oy, r.oz), d = mkd(r.dx, r.dy, r.dz);
  const d3 ec = cross(B - A, C - A);
  g.t = dot(A - o, ec) / dot(d, ec);
  g.hp = o + g.t * d;
  const double la = len(B - C), lb = len(A - C), lc = len(A - B);
  const d3 inc = (la * A + lb * B + lc * C) * (1.0 / (la + lb + lc));
  const d3 fn = normalize(ec);
  g.n = make_float3((float)fn.x, (float)fn.y, (float)fn.z);
  const d3 P3[3] = {A, B, C};
  double dist = 0.0, phi = -INFINITY;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const d3 p1 = P3[i], p2 = P3[(i + 1) % 3];
    d3 en = normalize(cross(ec, p1 - p2));
    double off = -dot(en, p1);
    if (i == 0) {
      dist = dot(en, inc) + off;
      if (dist > 0.0) {
        en = -en;
        off = -off;
        dist = -dist;
      }
    }
    const double ed = dot(en, g.hp) + off;
    phi = fmax(phi, ed);
    g.d[i] = ed;
  }
  g.phi_max = phi;
  g.phi_final = phi / dist;
  // __powf of the reference is NaN for a negative base and then clamped to 0
  g.Cx = (g.phi_final >= 0.0) ? (float)pow(g.phi_final, (double)sigma) : 0.0f;
  return g;
}

__device__ __constant__ float c_sh2[5] = {1.0925484305920792f, -1.0925484305920792f, 0.31539156525252005f,
                                          -1.0925484305920792f, 0.5462742152960396f};
__device__ __constant__ float c_sh3[7] = {-0.5900435899266435f, 2.890611442640554f, -0.4570457994644658f,
                                          0.3731763325901154f, -0.4570457994644658f, 1.445305721320277f,
                                          -0.5900435899266435f};
constexpr float kSH0 = 0.28209479177387814f;
constexpr float kSH1 = 0.4886025119029199f;

// Degree-<=3 SH basis (tritracer/common.h:16-55, auxiliary.h:13-30).
__device__ __forceinline__ void sh_basis(float x, float y, float z, int deg, float (&B)[16]) {
  B[0] = kSH0;
  if (deg > 0) {
    B[1] = -kSH1 * y;
    B[2] = kSH1 * z;
    B[3] = -kSH1 * x;
  }
  if (deg > 1) {
    const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
    B[4] = c_sh2[0] * xy;
    B[5] = c_sh2[1] * yz;
    B[6] = c_sh2[2] * (2.0f * zz - xx - yy);
    B[7] = c_sh2[3] * xz;
    B[8] = c_sh2[4] * (xx - yy);
    if (deg > 2) {
      B[9] = c_sh3[0] * y * (3.0f * xx - yy);
      B[10] = c_sh3[1] * xy * z;
      B[11] = c_sh3[2] * y * (4.0f * zz - xx - yy);
      B[12] = c_sh3[3] * z * (2.0f * zz - 3.0f * xx - 3.0f * yy);
      B[13] = c_sh3[4] * x * (4.0f * zz - xx - yy);
      B[14] = c_sh3[5] * z * (xx - yy);
      B[15] = c_sh3[6] * x * (xx - 3.0f * yy);
    }
  }
}

__device__ __forceinline__ int sh_count(int deg) { return (deg + 1) * (deg + 1); }

// RGB = sum_k B_k * sh_k + 0.5 (before the clamp at 0).
__device__ __forceinline__ float3 sh_raw(const float* __restrict__ shs, int M, int prim, int deg, const float (&B)[16]) {
  const float* base = shs + (size_t)prim * M * 3;
  float r = 0.f, g = 0.f, b = 0.f;
  if (M == 16 && deg == 3) {
    const float4* q = reinterpret_cast<const float4*>(base);  // 192-byte aligned rows
    float v[48];
#pragma unroll
    for (int i = 0; i < 12; ++i) {
      const float4 w = __ldg(q + i);
      v[4 * i] = w.x; v[4 * i + 1] = w.y; v[4 * i + 2] = w.z; v[4 * i + 3] = w.w;
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      r = fmaf(B[k], v[3 * k], r);
      g = fmaf(B[k], v[3 * k + 1], g);
      b = fmaf(B[k], v[3 * k + 2], b);
    }
  } else {
    const int n = sh_count(deg);
#pragma unroll 4
    for (int k = 0; k < n; ++k) {
      r = fmaf(B[k], __ldg(base + 3 * k), r);
      g = fmaf(B[k], __ldg(base + 3 * k + 1), g);
      b = fmaf(B[k], __ldg(base + 3 * k + 2), b);
    }
  }
  return make_float3(r + 0.5f, g + 0.5f, b + 0.5f);
}

__device__ __forceinline__ float3 unit_dir(const RayW& r) {
  const float inv = 1.0f / sqrtf(r.dx * r.dx + r.dy * r.dy + r.dz * r.dz);
  return make_float3(r.dx * inv, r.dy * inv, r.dz * inv);
}

// computeScaling of tritracer/forward.cu:25-74 (first blending ray records the
// largest angle the vertices subtend around the centroid direction), in FP64.
__device__ __forceinline__ void compute_scaling(const TraceParams& p, int prim, const RayW& r) {
  if (p.scaling[prim] > 0.0f) return;
  const int off = p.cumsum[prim], np = p.num_points[prim];
  const d3 o = mkd(r.ox, r.oy, r.oz);
  d3 cen = mkd(0, 0, 0);
  for (int i = 0; i < np; ++i) {
    const float* v = p.verts + 3 * (size_t)(off + i);
    cen = cen + mkd(v[0], v[1], v[2]);
  }
  cen = cen * (1.0 / (double)np);
  const d3 t2o = cen - o;
  double best = 0.0;
  for (int i = 0; i < np; ++i) {
    const float* v = p.verts + 3 * (size_t)(off + i);
    const d3 a = mkd(v[0], v[1], v[2]) - o;
    const double lab = len(a) * len(t2o);
    double ang = 0.0;
    if (!(lab < 1e-12)) ang = acos(fmax(-1.0, fmin(1.0, dot(a, t2o) / lab)));
    best = fmax(ang, best);
  }
  p.scaling[prim] = (float)best;
}

// ---------------------------------------------------------------- the march
// Visits the hit stream of one ray in the reference's chunk order and calls
// visit(prim, t) for each hit at or beyond the near plane; visit returns true
// to end the ray (transmittance cut-off).
template <class Visit>
__device__ __forceinline__ void march(const BvhView& bvh, const RayW& r, int tmin_inclusive, Stack st, int* status,
                                      Visit&& visit) {
  unsigned long long key_min = tmin_inclusive ? 0ull : (1ull << 32);
  float last_hit_t = 0.f;
  int ref_pos = 0;
  unsigned long long kb[kChunk];
  for (int chunk = 0; chunk < kMaxChunks; ++chunk) {
    float t_drop;
    query(bvh, r, key_min, kb, st, t_drop, status);
    const bool truncated = t_drop < INFINITY;
    int consumed = 0;
    unsigned long long last_key = 0;
    bool boundary = false, done = false;
    for (int i = 0; i < kChunk; ++i) {
      const unsigned long long key = kb[0];
#pragma unroll
      for (int j = 0; j < kChunk - 1; ++j) kb[j] = kb[j + 1];
      kb[kChunk - 1] = kEmptyKey;
      if (key == kEmptyKey || (truncated && key_t(key) >= t_drop)) break;
      ++consumed;
      last_key = key;
      const float t = key_t(key);
      // fmaxf(last + STEP_EPSILON, t) with the sum in double (forward.cu:111)
      last_hit_t = fmaxf(__double2float_rn(__dadd_rn((double)last_hit_t, kStepEps)), t);
      ++ref_pos;
      if (t >= kNear && visit(key_prim(key), t)) {
        done = true;
        break;
      }
      if (ref_pos == kChunk) {
        boundary = true;
        break;
      }
    }
    if (done) return;
    if (boundary) {
      // the reference's next optixTrace starts at last_hit_t
      ref_pos = 0;
      const unsigned long long tb = __float_as_uint(last_hit_t);
      key_min = tmin_inclusive ? (tb << 32) : ((tb + 1ull) << 32);
      continue;
    }
    if (truncated) {
      if (consumed == 0) {
        atomicOr(status, kStatusStack);
        return;
      }
      key_min = last_key + 1ull;  // continue the same stream exactly
      continue;
    }
    return;  // fewer than 16 hits left: the stream is exhausted
  }
  atomicOr(status, kStatusTimeout);
}

__device__ __forceinline__ bool next_tile(const TraceParams& p, int& px, int& py) {
  const int lane = threadIdx.x & 31;
  int tile = 0;
  if (lane == 0) tile = atomicAdd(p.work, 1);
  tile = __shfl_sync(0xFFFFFFFFu, tile, 0);
  if (tile >= p.ntiles) return false;
  const int tx = tile % p.ntx, ty = tile / p.ntx;
  px = tx * 8 + (lane & 7);
  py = ty * 4 + (lane >> 3);
  return true;
}

__device__ __forceinline__ Stack thread_stack() {
  extern __shared__ uint32_t smem[];
  Stack st;
  st.stride = blockDim.x;
  st.ref = smem + threadIdx.x;
  st.tn = reinterpret_cast<float*>(smem + kStackDepth * blockDim.x) + threadIdx.x;
  return st;
}

__device__ __forceinline__ RayW load_ray(const float* ro, const float* rd, int pix) {
  const float3 o = make_float3(ro[3 * pix], ro[3 * pix + 1], ro[3 * pix + 2]);
  const float3 d = make_float3(rd[3 * pix], rd[3 * pix + 1], rd[3 * pix + 2]);
  return make_ray(o, d);
}

// ---------------------------------------------------------------- forward
__device__ __forceinline__ void add_stats(unsigned long long* stats, unsigned rays, unsigned evals, unsigned blends) {
  rays = __reduce_add_sync(0xFFFFFFFFu, rays);
  evals = __reduce_add_sync(0xFFFFFFFFu, evals);
  blends = __reduce_add_sync(0xFFFFFFFFu, blends);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(stats, (unsigned long long)rays);
    atomicAdd(stats + 1, (unsigned long long)evals);
    atomicAdd(stats + 2, (unsigned long long)blends);
  }
}

__global__ void __launch_bounds__(kTraceThreads) k_forward(TraceParams p) {
  const Stack st = thread_stack();
  const int HW = p.H * p.W;
  unsigned n_rays = 0, n_eval = 0, n_blend = 0;
  int px, py;
  while (next_tile(p, px, py)) {
    if (px >= p.W || py >= p.H) continue;
    ++n_rays;
    const int pix = py * p.W + px;
    const RayW r = load_ray(p.ray_o, p.ray_d, pix);
    const float3 u = unit_dir(r);
    float B[16];
    sh_basis(u.x, u.y, u.z, p.sh_degree, B);
    float C0 = 0.f, C1 = 0.f, C2 = 0.f, N0 = 0.f, N1 = 0.f, N2 = 0.f, T = 1.0f;
    march(p.bvh, r, p.tmin_inclusive, st, p.status, [&](uint32_t prim, float) -> bool {
      const float4* tr = p.bvh.tri_prim + 3 * (size_t)prim;
      const Geom g = window_fp64(__ldg(tr), __ldg(tr + 1), __ldg(tr + 2), r, __ldg(p.sigma + prim));
      ++n_eval;
      const float alpha = fminf(kAlphaMax, __ldg(p.opac + prim) * g.Cx);
      if (alpha < kAlphaMin) return false;
      const float test_T = T * (1.0f - alpha);
      if (test_T < kTMin) return true;
      ++n_blend;
      p.density[prim] = 1.0f;
      compute_scaling(p, (int)prim, r);
      const float w = alpha * T;
      atomicMax(reinterpret_cast<int*>(p.max_blending) + prim, __float_as_int(w));
      N0 += g.n.x * w;
      N1 += g.n.y * w;
      N2 += g.n.z * w;
      const float3 c = sh_raw(p.shs, p.M, (int)prim, p.sh_degree, B);
      C0 += fmaxf(c.x, 0.f) * w;
      C1 += fmaxf(c.y, 0.f) * w;
      C2 += fmaxf(c.z, 0.f) * w;
      T = test_T;
      return false;
    });
    p.out_color[pix] = C0 + T * p.bg[0];
    p.out_color[HW + pix] = C1 + T * p.bg[1];
    p.out_color[2 * HW + pix] = C2 + T * p.bg[2];
    p.out_others[kDepthCh * HW + pix] = 0.0f;  // the reference never accumulates depth
    p.out_others[kAlphaCh * HW + pix] = 1.0f - T;
    p.out_others[(kNormalCh + 0) * HW + pix] = N0;
    p.out_others[(kNormalCh + 1) * HW + pix] = N1;
    p.out_others[(kNormalCh + 2) * HW + pix] = N2;
    p.out_others[kMidDepthCh * HW + pix] = 0.0f;
    p.out_others[kDistortionCh * HW + pix] = 0.0f;
  }
  add_stats(p.stats, n_rays, n_eval, n_blend);
}

// ---------------------------------------------------------------- adjoint
// Gradient of phi_max through the unit edge normals at the maximum and of the
// face normal (tritracer/backward.cu:104-189), in FP64; returns the 9 vertex
// gradients summed over both terms.
__device__ __forceinline__ void window_bwd_fp64(float4 a, float4 b, float4 c, const Geom& g, double dL_dphi,
                                                d3 dL_dn3, d3 (&gv)[3]) {
  const d3 V[3] = {tod(a), tod(b), tod(c)};
  gv[0] = gv[1] = gv[2] = mkd(0, 0, 0);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    if (fabs(g.d[k] - g.phi_max) > 1e-6) continue;
    const d3 p1 = V[k], p2 = V[(k + 1) % 3], p3 = V[(k + 2) % 3];
    const d3 n = cross(p1 - p3, p2 - p3);
    const d3 ne = cross(n, p1 - p2);
    const double inv = 1.0 / len(ne);
    const d3 Ne = ne * inv;
    // dL/dne = (I - Ne Ne^T) dL/dNe / |ne|
    const d3 dL_dNe = dL_dphi * (g.hp - p1);
    const d3 dL_dne = (dL_dNe - Ne * dot(Ne, dL_dNe)) * inv;
    // ne = ((p1-p3) x (p2-p3)) x (p1-p2), Jacobians in the form of
    // vecmath.h:2808-2859; v^T [u]x = v x u for the skew terms
    const d3 bb = p2 - p3, cc = p1 - p2, aa = p1 - p3;
    const d3 axb = cross(aa, bb);
    // v^T (b c^T - (b.c) I + [axb]x)
    const d3 g1 = mkd(dot(dL_dne, bb) * cc.x, dot(dL_dne, bb) * cc.y, dot(dL_dne, bb) * cc.z) -
                  dot(bb, cc) * dL_dne + cross(dL_dne, axb);
    // v^T ((a.c) I - a c^T - [axb]x)
    const d3 g2 = dot(aa, cc) * dL_dne - mkd(dot(dL_dne, aa) * cc.x, dot(dL_dne, aa) * cc.y, dot(dL_dne, aa) * cc.z) -
                  cross(dL_dne, axb);
    // v^T (c c^T - (c.c) I)
    const d3 g3 = mkd(dot(dL_dne, cc) * cc.x, dot(dL_dne, cc) * cc.y, dot(dL_dne, cc) * cc.z) - dot(cc, cc) * dL_dne;
    gv[k] = gv[k] + g1 - dL_dphi * Ne;
    gv[(k + 1) % 3] = gv[(k + 1) % 3] + g2;
    gv[(k + 2) % 3] = gv[(k + 2) % 3] + g3;
  }
  {
    const d3 p1 = V[0], p2 = V[1], p3 = V[2];
    const d3 n = cross(p1 - p3, p2 - p3);
    const double inv = 1.0 / len(n);
    const d3 Nn = n * inv;
    const d3 dL_dn = (dL_dn3 - Nn * dot(Nn, dL_dn3)) * inv;
    // n = (p1-p3) x (p2-p3): dn/dp1 = [p3-p2]x etc.; v^T [u]x = v x u
    gv[0] = gv[0] + cross(p3 - p2, dL_dn) * -1.0;
    gv[1] = gv[1] + cross(p1 - p3, dL_dn) * -1.0;
    gv[2] = gv[2] + cross(p2 - p1, dL_dn) * -1.0;
  }
}

__global__ void __launch_bounds__(kTraceThreads) k_backward(TraceParams p) {
  const Stack st = thread_stack();
  const int HW = p.H * p.W;
  int px, py;
  while (next_tile(p, px, py)) {
    if (px >= p.W || py >= p.H) continue;
    const int pix = py * p.W + px;
    const RayW r = load_ray(p.ray_o, p.ray_d, pix);
    const float3 u = unit_dir(r);
    float B[16];
    sh_basis(u.x, u.y, u.z, p.sh_degree, B);
    const float Cf0 = p.colors[pix], Cf1 = p.colors[HW + pix], Cf2 = p.colors[2 * HW + pix];
    const float Df = p.others[kDepthCh * HW + pix];
    const float Nf0 = p.others[(kNormalCh + 0) * HW + pix], Nf1 = p.others[(kNormalCh + 1) * HW + pix],
                Nf2 = p.others[(kNormalCh + 2) * HW + pix];
    const float g0 = p.dL_dpix[pix], g1 = p.dL_dpix[HW + pix], g2 = p.dL_dpix[2 * HW + pix];
    const float gD = p.dL_doth[kDepthCh * HW + pix];
    const float gN0 = p.dL_doth[(kNormalCh + 0) * HW + pix], gN1 = p.dL_doth[(kNormalCh + 1) * HW + pix],
                gN2 = p.dL_doth[(kNormalCh + 2) * HW + pix];
    float C0 = 0.f, C1 = 0.f, C2 = 0.f, N0 = 0.f, N1 = 0.f, N2 = 0.f, D = 0.f, T = 1.0f;
    march(p.bvh, r, p.tmin_inclusive, st, p.status, [&](uint32_t prim, float) -> bool {
      const float4* tr = p.bvh.tri_prim + 3 * (size_t)prim;
      const float4 va = __ldg(tr), vb = __ldg(tr + 1), vc = __ldg(tr + 2);
      const float sig = __ldg(p.sigma + prim);
      const Geom g = window_fp64(va, vb, vc, r, sig);
      const float opacity = __ldg(p.opac + prim);
      const float alpha = fminf(kAlphaMax, opacity * g.Cx);
      if (alpha < kAlphaMin) return false;
      const float test_T = T * (1.0f - alpha);
      if (test_T < kTMin) return true;
      const float w = alpha * T;
      const float3 raw = sh_raw(p.shs, p.M, (int)prim, p.sh_degree, B);
      const float c0 = fmaxf(raw.x, 0.f), c1 = fmaxf(raw.y, 0.f), c2 = fmaxf(raw.z, 0.f);
      C0 += c0 * w;
      C1 += c1 * w;
      C2 += c2 * w;
      N0 += g.n.x * w;
      N1 += g.n.y * w;
      N2 += g.n.z * w;
      const float ht = (float)g.t;
      D += w * ht;
      // backward.cu:296-312; C/N/D already include this hit
      const float inv1a = 1.0f / (1.0f - alpha);
      float dL_dalpha = g0 * (T * c0 - (Cf0 - C0) * inv1a) + g1 * (T * c1 - (Cf1 - C1) * inv1a) +
                        g2 * (T * c2 - (Cf2 - C2) * inv1a);
      dL_dalpha += gD * (T * ht - (Df - D) * inv1a);
      dL_dalpha += gN0 * (T * g.n.x - (Nf0 - N0) * inv1a) + gN1 * (T * g.n.y - (Nf1 - N1) * inv1a) +
                   gN2 * (T * g.n.z - (Nf2 - N2) * inv1a);
      red_add(p.d_opac + prim, dL_dalpha * g.Cx);
      const float dL_dC = opacity * dL_dalpha;
      if (g.phi_final > 0.0) red_add(p.d_sigma + prim, (float)((double)(dL_dC * g.Cx) * log(g.phi_final)));
      const double dL_dphi = (double)sig / g.phi_max * (double)dL_dC * (double)g.Cx;
      d3 gv[3];
      window_bwd_fp64(va, vb, vc, g, dL_dphi, mkd((double)gN0 * w, (double)gN1 * w, (double)gN2 * w), gv);
      float* dt = p.d_tri + 3 * (size_t)__ldg(p.cumsum + prim);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        red_add(dt + 3 * k + 0, (float)gv[k].x);
        red_add(dt + 3 * k + 1, (float)gv[k].y);
        red_add(dt + 3 * k + 2, (float)gv[k].z);
      }
      // SH: dRGB/dsh_k = B_k, masked where the colour was clamped at 0
      const float e0 = raw.x < 0.f ? 0.f : g0 * w, e1 = raw.y < 0.f ? 0.f : g1 * w, e2 = raw.z < 0.f ? 0.f : g2 * w;
      float* dsh = p.d_sh + (size_t)prim * p.M * 3;
      const int n = sh_count(p.sh_degree);
      if (p.M == 16 && n == 16) {
#pragma unroll
        for (int q = 0; q < 12; ++q) {
          float v4[4];
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int idx = 4 * q + j, k = idx / 3, ch = idx % 3;
            v4[j] = B[k] * (ch == 0 ? e0 : (ch == 1 ? e1 : e2));
          }
          red_add4(dsh + 4 * q, v4[0], v4[1], v4[2], v4[3]);
        }
      } else {
        for (int k = 0; k < n; ++k) {
          red_add(dsh + 3 * k + 0, B[k] * e0);
          red_add(dsh + 3 * k + 1, B[k] * e1);
          red_add(dsh + 3 * k + 2, B[k] * e2);
        }
      }
      T = test_T;
      return false;
    });
  }
}

// ---------------------------------------------------------------- hit stream
__global__ void __launch_bounds__(kTraceThreads) k_hit_stream(HitStreamParams p) {
  const Stack st = thread_stack();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.R) return;
  const RayW r = load_ray(p.ray_o, p.ray_d, i);
  unsigned long long key_min = 0ull;
  unsigned long long kb[kChunk];
  int count = 0;
  for (int chunk = 0; chunk < kMaxChunks; ++chunk) {
    float t_drop;
    query(p.bvh, r, key_min, kb, st, t_drop, p.status);
    int consumed = 0;
    unsigned long long last = 0;
#pragma unroll
    for (int j = 0; j < kChunk; ++j) {
      const unsigned long long key = kb[j];
      if (key == kEmptyKey || key_t(key) >= t_drop) break;
      if (count < p.max_hits) {
        p.ids[(size_t)i * p.max_hits + count] = key_prim(key);
        p.ts[(size_t)i * p.max_hits + count] = key_t(key);
      }
      ++count;
      ++consumed;
      last = key;
    }
    if (t_drop == INFINITY && consumed < kChunk) break;
    if (consumed == 0) {
      atomicOr(p.status, kStatusStack);
      break;
    }
    key_min = last + 1ull;
  }
  p.counts[i] = count;
}

}  // namespace

size_t trace_smem_bytes() { return (size_t)kStackDepth * kTraceThreads * 8; }

int trace_blocks_per_sm(int which) {
  int n = 0;
  const void* fn = which == 0 ? (const void*)k_forward : (const void*)k_backward;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, kTraceThreads, trace_smem_bytes()) != cudaSuccess) n = 1;
  return n > 0 ? n : 1;
}

cudaError_t launch_forward(const TraceParams& p, int grid, cudaStream_t s) {
  k_forward<<<grid, kTraceThreads, trace_smem_bytes(), s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_backward(const TraceParams& p, int grid, cudaStream_t s) {
  k_backward<<<grid, kTraceThreads, trace_smem_bytes(), s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_hit_stream(const HitStreamParams& p, cudaStream_t s) {
  const int grid = (p.R + kTraceThreads - 1) / kTraceThreads;
  if (grid == 0) return cudaSuccess;
  k_hit_stream<<<grid, kTraceThreads, trace_smem_bytes(), s>>>(p);
  return cudaGetLastError();
}

}  // namespace tt
