// Device-side definitions shared by the BVH builder and the trace kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace tt {

// ---------------------------------------------------------------- constants
// tritracer/config.h:10-11, auxiliary.h:9-10, forward.cu:129-134
constexpr int kChunk = 16;          // hits per k-closest query (CHUNK_SIZE)
constexpr double kStepEps = 1e-9;   // STEP_EPSILON, a double literal
constexpr float kNear = 0.2f;       // near_n
constexpr float kFar = 1000.0f;     // far_n
constexpr float kAlphaMax = 0.99f;
constexpr float kAlphaMin = 1.0f / 255.0f;
constexpr float kTMin = 0.0001f;    // transmittance cut-off
// side-output channels (config.h:16-20)
constexpr int kDepthCh = 0, kAlphaCh = 1, kNormalCh = 2, kMidDepthCh = 5, kDistortionCh = 6;

// BVH leaves hold up to this many triangles (a contiguous run of the
// Morton-sorted triangle records).
constexpr int kLeafMax = 3;
constexpr int kWide = 8;            // children per wide node
constexpr int kNodeF4 = 14;         // float4 words per wide node
constexpr uint32_t kLeafBit = 0x80000000u;
constexpr uint32_t kEmptyRef = 0x7FFFFFFFu;
constexpr int kMaxWideLevels = 72;  // > 64-bit key depth of the binary tree

// device status bits (tt_device_status)
constexpr int kStatusTimeout = 1;
constexpr int kStatusStack = 2;
constexpr int kStatusBounds = 4;
constexpr int kStatusCacheMiss = 8;  // the replay-only adjoint met a query its cache did not hold

// Debug builds (-DTT_BOUNDS_CHECK, `make bounds`): device index checks that
// record a violation in the status word and let the caller skip the access,
// instead of faulting. In normal builds the check is the constant true.
#ifdef TT_BOUNDS_CHECK
#define TT_IN_BOUNDS(status, cond) ((cond) ? true : (atomicOr((status), kStatusBounds), false))
#else
#define TT_IN_BOUNDS(status, cond) true
#endif

// Empty k-buffer slot: larger than every (t, id) key with t <= far.
constexpr unsigned long long kEmptyKey = 0xFFFFFFFFFFFFFFFFull;

__host__ __device__ inline uint32_t leaf_ref(uint32_t first, uint32_t count) {
  return kLeafBit | ((count - 1u) << 28) | first;
}
__host__ __device__ inline bool ref_is_leaf(uint32_t r) { return (r & kLeafBit) != 0u; }
__host__ __device__ inline uint32_t leaf_first(uint32_t r) { return r & 0x0FFFFFFFu; }
__host__ __device__ inline uint32_t leaf_count(uint32_t r) { return ((r >> 28) & 7u) + 1u; }

// Wide node layout in float4 words:
//   0,1 lo.x[8]  2,3 hi.x[8]  4,5 lo.y  6,7 hi.y  8,9 lo.z  10,11 hi.z
//   12,13 child refs (uint32 bits): internal wide-node index, leaf_ref(), or kEmptyRef
// Triangle records: 3 float4 per triangle (v0 | v1 | v2), w of word 0 holds
// the primitive index (as int bits) in the Morton-ordered copy.

struct BvhView {
  const float4* nodes;     // wide nodes
  const float4* tris;      // Morton-ordered triangle records
  const float4* tri_prim;  // primitive-ordered triangle records
  int P;
  int has_root;
  int wide_cap;  // wide nodes the node array holds (index bound)
};

// ---------------------------------------------------------------- key order
// A hit is the 64-bit key (bits(t) << 32) | primitive: for t >= +0 this is the
// (t, id) lexicographic order, which fixes the tie order the reference leaves
// to OptiX's traversal order.
__device__ __forceinline__ unsigned long long hit_key(float t, uint32_t prim) {
  return ((unsigned long long)__float_as_uint(t) << 32) | prim;
}
__device__ __forceinline__ float key_t(unsigned long long k) { return __uint_as_float((uint32_t)(k >> 32)); }
__device__ __forceinline__ uint32_t key_prim(unsigned long long k) { return (uint32_t)k; }

// ---------------------------------------------------------------- ray set-up
struct RayW {
  float ox, oy, oz;
  float dx, dy, dz;
  float ix, iy, iz;      // 1/d (components clamped away from 0)
  float oix, oiy, oiz;   // o * (1/d)
  int perm;              // watertight permutation: kx | ky << 2 | kz << 4
  float Sx, Sy, Sz;      // watertight shear
};

__device__ __forceinline__ float sel3(float x, float y, float z, int k) { return k == 0 ? x : (k == 1 ? y : z); }

__device__ __forceinline__ RayW make_ray(float3 o, float3 d) {
  RayW r;
  r.ox = o.x; r.oy = o.y; r.oz = o.z;
  r.dx = d.x; r.dy = d.y; r.dz = d.z;
  // Watertight set-up (Woop, Benthin, Wald, JCGT 2013): kz = axis of largest
  // |d|, kx/ky swapped when d[kz] < 0. Same expression tree as the oracle.
  const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
  int kz = (ax > ay) ? ((ax > az) ? 0 : 2) : ((ay > az) ? 1 : 2);
  int kx = kz + 1;
  if (kx == 3) kx = 0;
  int ky = kx + 1;
  if (ky == 3) ky = 0;
  const float dkz = sel3(d.x, d.y, d.z, kz);
  if (dkz < 0.0f) {
    const int tmp = kx;
    kx = ky;
    ky = tmp;
  }
  r.perm = kx | (ky << 2) | (kz << 4);
  r.Sx = __fdiv_rn(sel3(d.x, d.y, d.z, kx), dkz);
  r.Sy = __fdiv_rn(sel3(d.x, d.y, d.z, ky), dkz);
  r.Sz = __fdiv_rn(1.0f, dkz);
  auto safe_inv = [](float v) {
    const float m = fmaxf(fabsf(v), 1e-30f);
    return 1.0f / copysignf(m, v);
  };
  r.ix = safe_inv(d.x); r.iy = safe_inv(d.y); r.iz = safe_inv(d.z);
  r.oix = o.x * r.ix; r.oiy = o.y * r.iy; r.oiz = o.z * r.iz;
  return r;
}

// Axis permutation of the watertight test: the ray's own (kx, ky, kz), picked
// at run time ...
struct PermRt {
  int kx, ky, kz;
  __device__ __forceinline__ explicit PermRt(int pack) : kx(pack & 3), ky((pack >> 2) & 3), kz((pack >> 4) & 3) {}
  __device__ __forceinline__ float x(float a, float b, float c) const { return sel3(a, b, c, kx); }
  __device__ __forceinline__ float y(float a, float b, float c) const { return sel3(a, b, c, ky); }
  __device__ __forceinline__ float z(float a, float b, float c) const { return sel3(a, b, c, kz); }
};
// ... or fixed at compile time, for a warp whose rays all share it (the
// selects disappear; the arithmetic is the same).
template <int KX, int KY, int KZ>
struct PermCt {
  template <int K>
  __device__ __forceinline__ static float pick(float a, float b, float c) {
    return K == 0 ? a : (K == 1 ? b : c);
  }
  __device__ __forceinline__ float x(float a, float b, float c) const { return pick<KX>(a, b, c); }
  __device__ __forceinline__ float y(float a, float b, float c) const { return pick<KY>(a, b, c); }
  __device__ __forceinline__ float z(float a, float b, float c) const { return pick<KZ>(a, b, c); }
};

// Watertight, non-culling ray/triangle test in FP32 with the paper's FP64
// fall-back for zero edge functions. Every operation uses an explicit
// round-to-nearest intrinsic so nothing is contracted: t is bit-identical to
// the CPU oracle's evaluation of the same steps. `pm` must be the ray's own
// permutation (r.kx, r.ky, r.kz).
template <class Perm>
__device__ __forceinline__ bool isect_tri_p(const RayW& r, const Perm& pm, float4 a, float4 b, float4 c, float& t) {
  const float Ax0 = __fsub_rn(a.x, r.ox), Ay0 = __fsub_rn(a.y, r.oy), Az0 = __fsub_rn(a.z, r.oz);
  const float Bx0 = __fsub_rn(b.x, r.ox), By0 = __fsub_rn(b.y, r.oy), Bz0 = __fsub_rn(b.z, r.oz);
  const float Cx0 = __fsub_rn(c.x, r.ox), Cy0 = __fsub_rn(c.y, r.oy), Cz0 = __fsub_rn(c.z, r.oz);
  const float Akx = pm.x(Ax0, Ay0, Az0), Aky = pm.y(Ax0, Ay0, Az0), Akz = pm.z(Ax0, Ay0, Az0);
  const float Bkx = pm.x(Bx0, By0, Bz0), Bky = pm.y(Bx0, By0, Bz0), Bkz = pm.z(Bx0, By0, Bz0);
  const float Ckx = pm.x(Cx0, Cy0, Cz0), Cky = pm.y(Cx0, Cy0, Cz0), Ckz = pm.z(Cx0, Cy0, Cz0);
  const float Ax = __fsub_rn(Akx, __fmul_rn(r.Sx, Akz));
  const float Ay = __fsub_rn(Aky, __fmul_rn(r.Sy, Akz));
  const float Bx = __fsub_rn(Bkx, __fmul_rn(r.Sx, Bkz));
  const float By = __fsub_rn(Bky, __fmul_rn(r.Sy, Bkz));
  const float Cx = __fsub_rn(Ckx, __fmul_rn(r.Sx, Ckz));
  const float Cy = __fsub_rn(Cky, __fmul_rn(r.Sy, Ckz));
  float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
  float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
  float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
  if (U == 0.0f || V == 0.0f || W == 0.0f) {
    U = __double2float_rn(__dsub_rn(__dmul_rn((double)Cx, (double)By), __dmul_rn((double)Cy, (double)Bx)));
    V = __double2float_rn(__dsub_rn(__dmul_rn((double)Ax, (double)Cy), __dmul_rn((double)Ay, (double)Cx)));
    W = __double2float_rn(__dsub_rn(__dmul_rn((double)Bx, (double)Ay), __dmul_rn((double)By, (double)Ax)));
  }
  if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
  const float det = __fadd_rn(__fadd_rn(U, V), W);
  if (det == 0.0f) return false;
  const float Az = __fmul_rn(r.Sz, Akz);
  const float Bz = __fmul_rn(r.Sz, Bkz);
  const float Cz = __fmul_rn(r.Sz, Ckz);
  const float T = __fadd_rn(__fadd_rn(__fmul_rn(U, Az), __fmul_rn(V, Bz)), __fmul_rn(W, Cz));
  // + 0 turns a -0 distance (a ray starting on the triangle's plane, e.g. a
  // spawned secondary ray) into +0: hit keys are built from the float's
  // bits, where -0 would sort after every other hit
  t = __fadd_rn(__fdiv_rn(T, det), 0.0f);
  return true;
}

__device__ __forceinline__ bool isect_tri(const RayW& r, float4 a, float4 b, float4 c, float& t) {
  return isect_tri_p(r, PermRt(r.perm), a, b, c, t);
}

// Packed permutation: kx | ky << 2 | kz << 4. The six values the watertight
// set-up produces (kz = dominant axis; kx, ky the other two, swapped when the
// direction along kz is negative).
__device__ __forceinline__ int perm_pack(const RayW& r) { return r.perm; }
constexpr int kPerm12_0 = 1 | (2 << 2) | (0 << 4), kPerm21_0 = 2 | (1 << 2) | (0 << 4);
constexpr int kPerm20_1 = 2 | (0 << 2) | (1 << 4), kPerm02_1 = 0 | (2 << 2) | (1 << 4);
constexpr int kPerm01_2 = 0 | (1 << 2) | (2 << 4), kPerm10_2 = 1 | (0 << 2) | (2 << 4);

// Calls fn(perm) with a compile-time permutation when `pack` (warp-uniform)
// is one of the six, else with the ray's run-time one.
template <class Fn>
__device__ __forceinline__ void with_perm(int pack, const RayW& r, Fn&& fn) {
  switch (pack) {
    case kPerm12_0: fn(PermCt<1, 2, 0>{}); break;
    case kPerm21_0: fn(PermCt<2, 1, 0>{}); break;
    case kPerm20_1: fn(PermCt<2, 0, 1>{}); break;
    case kPerm02_1: fn(PermCt<0, 2, 1>{}); break;
    case kPerm01_2: fn(PermCt<0, 1, 2>{}); break;
    case kPerm10_2: fn(PermCt<1, 0, 2>{}); break;
    default: fn(PermRt(r.perm)); break;
  }
}

// ---------------------------------------------------------------- vectors
struct d3 {
  double x, y, z;
};
__device__ __forceinline__ d3 mkd(double x, double y, double z) { return d3{x, y, z}; }
__device__ __forceinline__ d3 tod(float4 v) { return d3{(double)v.x, (double)v.y, (double)v.z}; }
__device__ __forceinline__ d3 operator+(d3 a, d3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ d3 operator-(d3 a, d3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ d3 operator-(d3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ d3 operator*(d3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ d3 operator*(double s, d3 a) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ d3 cross(d3 a, d3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ double len(d3 v) { return sqrt(dot(v, v)); }
__device__ __forceinline__ d3 normalize(d3 v) { return v * (1.0 / sqrt(dot(v, v))); }

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }

// ---------------------------------------------------------------- atomics
__device__ __forceinline__ void red_add(float* p, float v) { atomicAdd(p, v); }
// Vector reduction (sm_90+): four consecutive, 16-byte aligned floats.
__device__ __forceinline__ void red_add4(float* p, float a, float b, float c, float d) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(a), "f"(b), "f"(c), "f"(d)
               : "memory");
}

}  // namespace tt
