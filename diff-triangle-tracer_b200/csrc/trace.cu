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
//  * k-buffer: the k nearest (t, primitive) pairs packed as 64-bit keys, kept
//    sorted in shared memory (one column per lane) by insertion, the largest
//    mirrored in a register;
//  * the chunked march of the reference is reproduced exactly on top of the
//    key stream: after every 16th visited hit the next query starts AT the
//    last hit's t (closed interval, optixTrace) or strictly after it;
//  * per hit, the window function runs in FP64 from the plane intersection
//    (the FP32 hit point loses ~4 digits on small triangles far from the
//    camera); SH, compositing and the side outputs are FP32 like the
//    reference; the adjoint re-traverses instead of storing hit lists.
#include <algorithm>
#include <cfloat>

#include "trace.cuh"

namespace tt {
namespace {

constexpr int kMaxChunks = 1 << 20;   // bound on re-traces per ray
constexpr int kMaxSteps = 1 << 24;    // bound on stack pops per query
// Resident blocks per SM the register budget must allow: 4 x 128 threads
// leave 128 registers a thread. Measured on 1M triangles, 4 x 800^2 rays,
// packets of 32: forward 19.0 / adjoint 21.6 ms at 4 blocks, 20.5 / 23.2 at
// 5 (96 registers, ~300 bytes of spills a thread), 21.8 / 24.9 at 6; later,
// with the forward at 18.2 ms at 4 blocks, 19.9 at 3 (168 registers, no
// spills, 12 warps per SM).
#ifndef TT_MIN_BLOCKS
#define TT_MIN_BLOCKS 4
#endif
constexpr int kMinBlocks = TT_MIN_BLOCKS;

// Per-lane traversal stack: the top SD entries in shared memory (strided by
// the block size, conflict-free), continued in thread-local memory for deep
// trees (only touched when the shared part is full).
constexpr int kSpill = 64;
struct Stack {
  uint32_t* ref;
  float* tn;
  int stride;
  __device__ __forceinline__ void put(int i, uint32_t r, float t) {
    ref[i * stride] = r;
    tn[i * stride] = t;
  }
};

// Sorted insert into the lane's k-buffer in shared memory (hits are rare
// next to box tests, so the buffer need not occupy 32 registers). `n` counts
// the valid keys (the slots from n on hold kEmptyKey): the insert shifts only
// the valid keys above the new one, not the empty tail, and once the buffer
// is full the largest key drops out. Returns true when the buffer is full
// after the insert (its last key then bounds the query).
template <int K>
__device__ __forceinline__ bool kb_insert_smem(unsigned long long* kb, int stride, unsigned long long key, int& n) {
  int i = n < K ? n : K - 1;
  while (i > 0) {
    const unsigned long long prev = kb[(i - 1) * stride];
    if (prev <= key) break;
    kb[i * stride] = prev;
    --i;
  }
  kb[i * stride] = key;
  if (n < K) ++n;
  return n == K;
}

// A candidate key enters a k-buffer holding n valid keys iff the buffer has
// room or the key is below its largest key.
template <int K>
__device__ __forceinline__ bool kb_accepts(const unsigned long long* kb, int stride, unsigned long long key, int n) {
  return n < K || key < kb[(K - 1) * stride];
}


struct Counters {
  unsigned nodes = 0, tris = 0, queries = 0, warp_nodes = 0;
  unsigned cont = 0, restart = 0;  // proposed intervals left by continuation / re-trace
  unsigned replays = 0;            // queries taken from the hit cache (adjoint)
  __device__ __forceinline__ void add_cont() { ++cont; }
  __device__ __forceinline__ void add_restart() { ++restart; }
};

// The packet drivers keep their counters in per-warp shared-memory words
// instead (warp-uniform updates by lane 0, shared atomics for the rare
// per-lane events), so the traversal carries no counter registers; they are
// folded into the thread's Counters when the warp is done.
constexpr int kWNodes = 0, kWTris = 1, kWWarpNodes = 2, kWQueries = 3, kWReplays = 4, kWCont = 5, kWRestart = 6,
              kWCounters = 8;
struct WarpCounters {
  unsigned* w;
  __device__ __forceinline__ void add_cont() { atomicAdd(w + kWCont, 1u); }
  __device__ __forceinline__ void add_restart() { atomicAdd(w + kWRestart, 1u); }
};

// Three-input FP32 min / max (one instruction on sm_100); min and max are
// exact, so the fold order does not change the result.
__device__ __forceinline__ float max3f(float a, float b, float c) {
  float d;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
  return d;
}
__device__ __forceinline__ float min3f(float a, float b, float c) {
  float d;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
  return d;
}

// Slab test of one ray against the 8 child boxes of a wide node:
// tn[c] = max(t_lo, near planes), tf[c] = min(tmax, far planes), the child is
// entered iff tn[c] <= tf[c]. The near and far plane of each axis are picked
// per ray by the sign of the direction (`nx`, `ny`, `nz`: word offset of the
// near planes; the far ones are at ^2). Two children's planes of one axis go
// through one packed FP32 FMA (each lane rounds like fmaf), and the three
// axes fold with 3-input min / max: 5 instructions per child where the
// scalar form takes 13, with bit-identical tn / tf.
__device__ __forceinline__ void slab8(const float4* __restrict__ nd, int nx, int ny, int nz, const RayW& r,
                                      float t_lo, float tmax, float (&tn)[8], float (&tf)[8]) {
  const float2 ix = make_float2(r.ix, r.ix), iy = make_float2(r.iy, r.iy), iz = make_float2(r.iz, r.iz);
  const float2 ox = make_float2(-r.oix, -r.oix), oy = make_float2(-r.oiy, -r.oiy), oz = make_float2(-r.oiz, -r.oiz);
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const float4 xn = __ldg(nd + nx + h), xf = __ldg(nd + (nx ^ 2) + h);
    const float4 yn = __ldg(nd + ny + h), yf = __ldg(nd + (ny ^ 2) + h);
    const float4 zn = __ldg(nd + nz + h), zf = __ldg(nd + (nz ^ 2) + h);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int c = 4 * h + 2 * q;
      const float2 axn = __ffma2_rn(q ? make_float2(xn.z, xn.w) : make_float2(xn.x, xn.y), ix, ox);
      const float2 ayn = __ffma2_rn(q ? make_float2(yn.z, yn.w) : make_float2(yn.x, yn.y), iy, oy);
      const float2 azn = __ffma2_rn(q ? make_float2(zn.z, zn.w) : make_float2(zn.x, zn.y), iz, oz);
      const float2 axf = __ffma2_rn(q ? make_float2(xf.z, xf.w) : make_float2(xf.x, xf.y), ix, ox);
      const float2 ayf = __ffma2_rn(q ? make_float2(yf.z, yf.w) : make_float2(yf.x, yf.y), iy, oy);
      const float2 azf = __ffma2_rn(q ? make_float2(zf.z, zf.w) : make_float2(zf.x, zf.y), iz, oz);
      tn[c] = fmaxf(max3f(axn.x, ayn.x, azn.x), t_lo);
      tn[c + 1] = fmaxf(max3f(axn.y, ayn.y, azn.y), t_lo);
      tf[c] = fminf(min3f(axf.x, ayf.x, azf.x), tmax);
      tf[c + 1] = fminf(min3f(axf.y, ayf.y, azf.y), tmax);
    }
  }
}

// The kChunk smallest hit keys >= key_min (t <= t_hi) along the ray, in
// ascending order, EMPTY-padded. If the stack overflowed, subtrees were
// dropped and t_drop is the smallest entry distance among them: only keys with
// t < t_drop are then guaranteed.
//
// Node visit: the near and far slab planes of each axis are picked per ray by
// the sign of the direction, so each child costs 6 FMAs and 6 min/max; child
// boxes are padded outward when written (k_wide_boxes) so the rounded test
// never culls a reported hit, and empty slots hold inverted boxes that never
// pass. Hit children are pushed in slot order with the nearest one on top.
template <int SD>
__device__ __forceinline__ void query(const BvhView& bvh, const RayW& r, unsigned long long key_min, float t_hi,
                                      unsigned long long* kb, int kstride, Stack st, float& t_drop, int* status,
                                      Counters& cnt, int count_work) {
  ++cnt.queries;
#pragma unroll
  for (int i = 0; i < kChunk; ++i) kb[i * kstride] = kEmptyKey;
  int kb_n = 0;
  t_drop = INFINITY;
  if (!bvh.has_root) return;
  const float t_lo = key_t(key_min);
  float tmax = t_hi;
  // word offsets of the near / far planes (lo at +0, hi at +2 within each axis)
  const int nx = r.ix >= 0.f ? 0 : 2, ny = r.iy >= 0.f ? 4 : 6, nz = r.iz >= 0.f ? 8 : 10;
  // entries at index >= SD live in thread-local memory
  uint32_t xref[kSpill];
  float xtn[kSpill];
  auto put = [&](int i, uint32_t r, float t) {
    if (i < SD) {
      st.put(i, r, t);
    } else {
      xref[i - SD] = r;
      xtn[i - SD] = t;
    }
  };
  int sp = 0;
  put(sp++, 0u, t_lo);
  int steps = 0;
  while (sp > 0) {
    if (++steps > kMaxSteps) {
      atomicOr(status, kStatusTimeout);
      break;
    }
    --sp;
    const uint32_t ref = sp < SD ? st.ref[sp * st.stride] : xref[sp - SD];
    if ((sp < SD ? st.tn[sp * st.stride] : xtn[sp - SD]) > tmax) continue;
    if (ref_is_leaf(ref)) {
      const uint32_t first = leaf_first(ref), ntri = leaf_count(ref);
      if (!TT_IN_BOUNDS(status, first + ntri <= (uint32_t)bvh.P)) continue;
      if (count_work) cnt.tris += ntri;
      for (uint32_t j = 0; j < ntri; ++j) {
        const float4* tr = bvh.tris + 3 * (size_t)(first + j);
        const float4 a = __ldg(tr), b = __ldg(tr + 1), c = __ldg(tr + 2);
        float t;
        if (!isect_tri(r, a, b, c, t)) continue;
        if (!(t >= t_lo) || !(t <= tmax)) continue;
        const unsigned long long key = hit_key(t, (uint32_t)__float_as_int(a.w));
        if (key >= key_min && kb_accepts<kChunk>(kb, kstride, key, kb_n)) {
          if (kb_insert_smem<kChunk>(kb, kstride, key, kb_n)) tmax = key_t(kb[(kChunk - 1) * kstride]);
        }
      }
      continue;
    }
    if (!TT_IN_BOUNDS(status, ref < (uint32_t)bvh.wide_cap)) continue;
    if (count_work) ++cnt.nodes;
    const float4* nd = bvh.nodes + (size_t)ref * kNodeF4;
    float tn[8], tf[8];
    bool hit[8];
    slab8(nd, nx, ny, nz, r, t_lo, tmax, tn, tf);
#pragma unroll
    for (int c = 0; c < 8; ++c) hit[c] = tn[c] <= tf[c];
    int nhit = 0, best = -1;
    float best_t = INFINITY;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      if (hit[c]) {
        ++nhit;
        if (tn[c] < best_t) {
          best_t = tn[c];
          best = c;
        }
      }
    }
    if (nhit == 0) continue;
    const float4 r0 = __ldg(nd + 12), r1 = __ldg(nd + 13);
    const uint32_t cref[8] = {__float_as_uint(r0.x), __float_as_uint(r0.y), __float_as_uint(r0.z),
                              __float_as_uint(r0.w), __float_as_uint(r1.x), __float_as_uint(r1.y),
                              __float_as_uint(r1.z), __float_as_uint(r1.w)};
    // nearest child last (top of the stack); on overflow drop the others and
    // remember the smallest distance dropped
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      if (!hit[c] || c == best) continue;
      if (sp < SD + kSpill - 1) {
        put(sp++, cref[c], tn[c]);
      } else {
        t_drop = fminf(t_drop, tn[c]);
      }
    }
    put(sp++, cref[best], best_t);
  }
}

// ---------------------------------------------------------------- packets
// Warp packet traversal for coherent rays (a warp = an 8x4-pixel tile of a
// pinhole camera, whose rays all cross nearly the same BVH nodes). The warp
// shares ONE stack in shared memory; an entry carries the node, the mask of
// lanes whose ray hit its box and the smallest entry distance among them.
// Every active lane tests its own ray (its own [t_lo, tmax] interval and
// k-buffer) against the 8 children; ballots give each child's lane mask and
// __reduce_min_sync its nearest entry distance; the triangles of hit leaf
// children are tested at once by the lanes that entered them, and hit
// interior children are ranked lane-parallel (lane c ranks child c) and
// pushed far-to-near, so the stack holds interior nodes only. Control flow is
// warp-uniform, so SIMT efficiency equals the fraction of lanes whose ray
// still needs the node, and every node/triangle record is read once per warp.
// Interior nodes only (leaf children are tested at their parent's visit):
// a BVH8 of depth d needs at most ~7d entries.
constexpr int kWarpStack = 96;

struct WarpStack {
  uint32_t* ref;
  unsigned* mask;
  float* tmin;
  unsigned* cnt;  // kWCounters words: the warp's traversal counters
};

template <int K>
__device__ __forceinline__ void packet_query(const BvhView& bvh, const RayW& r, bool want,
                                             unsigned long long key_min, float t_hi, unsigned long long* kb, int kstride,
                                             WarpStack ws, float& t_drop, int* status, int count_work) {
  const unsigned full = 0xFFFFFFFFu;
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int i = 0; i < K; ++i) kb[i * kstride] = kEmptyKey;
  int kb_n = 0;
  t_drop = INFINITY;
  const unsigned act = __ballot_sync(full, want);
  if (act == 0 || !bvh.has_root) return;
  if (lane == 0) ws.cnt[kWQueries] += __popc(act);
  const float t_lo = want ? key_t(key_min) : 0.f;
  float tmax = want ? t_hi : -1.0f;  // a lane without a query never passes a test
  const int nx = r.ix >= 0.f ? 0 : 2, ny = r.iy >= 0.f ? 4 : 6, nz = r.iz >= 0.f ? 8 : 10;
  // the rays of a packet nearly always share the watertight axis permutation:
  // then the triangle tests use it as a compile-time constant
  const int pk = perm_pack(r);
  const int pk0 = __shfl_sync(full, pk, __ffs(act) - 1);
  const int wperm = __all_sync(full, !want || pk == pk0) ? pk0 : -1;
  if (lane == 0) {
    ws.ref[0] = 0u;
    ws.mask[0] = act;
    ws.tmin[0] = 0.f;
  }
  __syncwarp();
  int sp = 1;
  for (int steps = 0; sp > 0; ++steps) {
    if (steps > kMaxSteps) {
      if (lane == 0) atomicOr(status, kStatusTimeout);
      break;
    }
    --sp;
    const uint32_t ref = ws.ref[sp];
    const float emin = ws.tmin[sp];
    // lanes whose interval now ends before the entry's nearest distance drop out
    const unsigned m = ws.mask[sp] & __ballot_sync(full, tmax >= emin);
    __syncwarp();
    if (m == 0) continue;
    if (!TT_IN_BOUNDS(status, ref < (uint32_t)bvh.wide_cap)) continue;  // ref is the same in every lane
    const bool on = (m >> lane) & 1u;
    if (count_work && lane == 0) {
      ws.cnt[kWNodes] += __popc(m);
      ws.cnt[kWWarpNodes] += 1u;
    }
    const float4* nd = bvh.nodes + (size_t)ref * kNodeF4;
    // lane c (c < 8) will push child c: fetch its reference with the boxes
    const uint32_t my_ref = lane < 8 ? __ldg(reinterpret_cast<const uint32_t*>(nd + 12) + lane) : kEmptyRef;
    float tn[8], tf[8];
    slab8(nd, nx, ny, nz, r, t_lo, tmax, tn, tf);
    // lane c (c < 8) collects child c: the mask of lanes entering it and
    // their nearest entry distance
    unsigned mymask = 0u;
    float mine = INFINITY;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const bool hit = on && tn[c] <= tf[c];
      const unsigned cm = __ballot_sync(full, hit);
      const unsigned cmin = __reduce_min_sync(full, hit ? __float_as_uint(tn[c]) : 0x7F800000u);
      if (lane == c) {
        mymask = cm;
        mine = __uint_as_float(cmin);
      }
    }
    // Leaf children are tested right away by the lanes that entered them (a
    // push and a pop saved per leaf); only interior children go on the stack.
    const bool my_leaf = mymask != 0u && ref_is_leaf(my_ref);
    for (unsigned lb = __ballot_sync(full, my_leaf); lb != 0u; lb &= lb - 1u) {
      const int lc = __ffs(lb) - 1;
      const uint32_t lref = __shfl_sync(full, my_ref, lc);
      const unsigned lm = __shfl_sync(full, mymask, lc);  // lanes entering the leaf
      const bool lon = (lm >> lane) & 1u;
      const uint32_t first = leaf_first(lref), ntri = leaf_count(lref);
      if (!TT_IN_BOUNDS(status, first + ntri <= (uint32_t)bvh.P)) continue;  // the same in every lane
      if (count_work && lane == 0) ws.cnt[kWTris] += __popc(lm) * ntri;
      with_perm(wperm, r, [&](const auto& pm) {
        for (uint32_t j = 0; j < ntri; ++j) {
          const float4* tr = bvh.tris + 3 * (size_t)(first + j);
          const float4 a = __ldg(tr), b = __ldg(tr + 1), c = __ldg(tr + 2);
          float t;
          if (!lon || !isect_tri_p(r, pm, a, b, c, t)) continue;
          if (!(t >= t_lo) || !(t <= tmax)) continue;
          const unsigned long long key = hit_key(t, (uint32_t)__float_as_int(a.w));
          if (key >= key_min && kb_accepts<K>(kb, kstride, key, kb_n)) {
            if (kb_insert_smem<K>(kb, kstride, key, kb_n)) tmax = key_t(kb[(K - 1) * kstride]);
          }
        }
      });
    }
    const unsigned pmask = my_leaf ? 0u : mymask;  // lane c: lanes entering interior child c
    const int nh = __popc(__ballot_sync(full, pmask != 0u));
    if (nh == 0) continue;
    // rank among the entered children by entry distance: distances are >= 0,
    // so their bit patterns order like the values; the low 3 bits make room
    // for the slot (near-ties go by slot, which only affects the visit order)
    const unsigned key = pmask != 0u ? ((__float_as_uint(mine) & ~7u) | (unsigned)lane) : 0xFFFFFFFFu;
    int rank = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) rank += __shfl_sync(full, key, c) < key ? 1 : 0;
    const int avail = kWarpStack - sp;
    const int npush = nh < avail ? nh : avail;
    if (pmask != 0u && rank < npush && TT_IN_BOUNDS(status, sp + npush - 1 - rank < kWarpStack)) {
      const int pos = sp + npush - 1 - rank;  // nearest on top
      ws.ref[pos] = my_ref;
      ws.mask[pos] = pmask;
      ws.tmin[pos] = mine;
    }
    if (nh > avail) {
      // stack full: the farthest children are dropped; their rays only trust
      // keys nearer than the dropped entry distance
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const unsigned m = __shfl_sync(full, pmask, c);
        const float e = __shfl_sync(full, mine, c);
        const int rk = __shfl_sync(full, rank, c);
        if (m != 0u && rk >= npush && ((m >> lane) & 1u)) t_drop = fminf(t_drop, e);
      }
    }
    __syncwarp();
    sp += npush;
  }
}

// ---------------------------------------------------------------- shading
// Per-hit geometry. The ray/plane intersection (t and the hit point relative
// to vertex A) is solved in FP64; everything after that works in FP32 on
// triangle-sized, A-relative coordinates, where FP32 keeps ~7 digits of the
// inradius (an FP32 hit point o + t d at distance ~3 keeps only ~3).
struct Geom {
  float Cx;
  float3 n;          // unit face normal
  float phi_final, phi_max;
  float d[3];        // signed edge distances of the hit point
  float3 q;          // hit point - A
  float3 e1, e2;     // B - A, C - A
  float t;           // hit distance from the FP64 solve
};

__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float fdot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 fcross(float3 a, float3 b) {
  return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float flen(float3 v) { return sqrtf(fdot(v, v)); }
__device__ __forceinline__ float3 fnormalize(float3 v) { return v * rsqrtf(fdot(v, v)); }

// FP32 operations with explicit round-to-nearest and no contraction, for
// code that repeats the reference's FP32 expression trees operation by
// operation (the sphere variants' set-up, the reference-arithmetic window
// function).
namespace vf {
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float3 add(float3 a, float3 b) { return make_float3(add(a.x, b.x), add(a.y, b.y), add(a.z, b.z)); }
__device__ __forceinline__ float3 sub(float3 a, float3 b) { return make_float3(sub(a.x, b.x), sub(a.y, b.y), sub(a.z, b.z)); }
__device__ __forceinline__ float3 scale(float3 a, float s) { return make_float3(mul(a.x, s), mul(a.y, s), mul(a.z, s)); }
__device__ __forceinline__ float dot(float3 a, float3 b) { return add(add(mul(a.x, b.x), mul(a.y, b.y)), mul(a.z, b.z)); }
__device__ __forceinline__ float3 cross(float3 a, float3 b) {
  return make_float3(sub(mul(a.y, b.z), mul(a.z, b.y)), sub(mul(a.z, b.x), mul(a.x, b.z)),
                     sub(mul(a.x, b.y), mul(a.y, b.x)));
}
__device__ __forceinline__ float3 normalize(float3 v) { return scale(v, div(1.0f, __fsqrt_rn(dot(v, v)))); }
__device__ __forceinline__ float3 neg(float3 v) { return make_float3(-v.x, -v.y, -v.z); }
// vecmath.h reflect: i - (2 n) dot(n, i)
__device__ __forceinline__ float3 reflect(float3 i, float3 n) { return sub(i, scale(scale(n, 2.0f), dot(n, i))); }

// common.h:116-141
__device__ __forceinline__ bool hit_sphere(float r, float3 cnt, float3 o, float3 d, float& t) {
  const float3 op = sub(o, cnt);
  const float a = dot(d, d);
  if (a <= 0.0f) return false;
  const float b = dot(op, d);
  const float c = sub(dot(op, op), mul(r, r));
  float det = sub(mul(b, b), mul(c, a));
  if (det < 0.0f) return false;
  det = __fsqrt_rn(det);
  t = div(sub(-b, det), a);
  if ((double)t < kStepEps) {
    t = div(add(-b, det), a);
    if ((double)t < kStepEps) return false;
  }
  return true;
}

// refract.cu:24-45, kept as written (square roots where Snell's law has
// squares; the same double/float mix)
__device__ __forceinline__ bool refract_dir(float3& out, float3 in, float3 n, float eta_org) {
  const float cos_i = dot(in, n);
  float eta = eta_org;
  if ((double)cos_i > 0.0) {
    eta = __double2float_rn(__drcp_rn((double)eta_org));
    n = neg(n);
  }
  const float sin2_i = __double2float_rn(fmax(0.0, __dsub_rn(1.0, (double)sqrtf(cos_i))));
  const float sin2_t = div(sin2_i, __fsqrt_rn(eta));
  if (sin2_t >= 1.0f) return false;
  const float cos_t = __double2float_rn(sqrt(fmax(0.0, __dsub_rn(1.0, (double)sin2_t))));
  out = add(scale(in, div(1.0f, eta)), scale(n, sub(div(-cos_i, eta), cos_t)));
  return true;
}

// envlight.cu:25-51
__device__ __forceinline__ float lcg(uint32_t& u) {
  u = u * 1664525u + 1013904223u;
  return mul((float)(u & 0x00FFFFFFu), 1.0f / 16777216.0f);
}
__device__ __forceinline__ float3 cosine_hemisphere(uint32_t& seed, float3 n) {
  const float u = lcg(seed);
  const float v = lcg(seed);
  const float z = __fsqrt_rn(u);
  const float rr = __fsqrt_rn(fmaxf(0.0f, __double2float_rn(__dsub_rn(1.0, (double)mul(z, z)))));
  const float phi = mul(v, 6.2831853071795864769f);
  const float3 dir = make_float3(mul(rr, cosf(phi)), mul(rr, sinf(phi)), z);
  const float3 up = fabsf(n.z) < 0.999f ? make_float3(0.f, 0.f, 1.f) : make_float3(0.f, 1.f, 0.f);
  const float3 t = normalize(cross(up, n));
  const float3 b = normalize(cross(n, t));
  return normalize(add(add(scale(t, dir.x), scale(b, dir.y)), scale(n, dir.z)));
}
}  // namespace vf

// Window function of tritracer/common.h:57-114: edge normals
// normalize(edge_cross x (p_i - p_{i+1})), edge 0 oriented by the incenter,
// phi = max edge distance, phi_final = phi / dist(incenter, edge 0),
// Cx = max(0, phi_final^sigma) with a negative base giving 0.
__device__ __forceinline__ Geom window_fn(float4 a, float4 b, float4 c, float3 o, float3 d, float sigma) {
  Geom g;
  const double e1x = (double)b.x - a.x, e1y = (double)b.y - a.y, e1z = (double)b.z - a.z;
  const double e2x = (double)c.x - a.x, e2y = (double)c.y - a.y, e2z = (double)c.z - a.z;
  const double nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
  const double ox = (double)o.x - a.x, oy = (double)o.y - a.y, oz = (double)o.z - a.z;  // o - A
  const double t = -(ox * nx + oy * ny + oz * nz) / ((double)d.x * nx + (double)d.y * ny + (double)d.z * nz);
  g.t = (float)t;
  g.q = make_float3((float)(ox + t * d.x), (float)(oy + t * d.y), (float)(oz + t * d.z));
  g.e1 = make_float3((float)e1x, (float)e1y, (float)e1z);
  g.e2 = make_float3((float)e2x, (float)e2y, (float)e2z);
  const float3 e1 = g.e1, e2 = g.e2;
  const float la = flen(e1 - e2), lb = flen(e2), lc = flen(e1);
  const float3 inc = (lb * e1 + lc * e2) * (1.0f / (la + lb + lc));  // A is the origin
  const float3 ec = fcross(e1, e2);
  g.n = fnormalize(ec);
  float3 en0 = fnormalize(fcross(ec, -e1));
  float dist = fdot(en0, inc);
  if (dist > 0.0f) {
    en0 = -en0;
    dist = -dist;
  }
  const float3 en1 = fnormalize(fcross(ec, e1 - e2));
  const float3 en2 = fnormalize(fcross(ec, e2));
  g.d[0] = fdot(en0, g.q);
  g.d[1] = fdot(en1, g.q - e1);
  g.d[2] = fdot(en2, g.q - e2);
  g.phi_max = fmaxf(fmaxf(g.d[0], g.d[1]), g.d[2]);
  g.phi_final = g.phi_max / dist;
  // __powf of the reference is NaN for a negative base and then clamped to 0
  g.Cx = (g.phi_final >= 0.0f) ? powf(g.phi_final, sigma) : 0.0f;
  return g;
}

// The window function in the reference's own FP32 arithmetic
// (tritracer/common.h:57-114 on the hit point o + t d of forward.cu:118, t
// the FP32 hit distance): absolute coordinates, each operation rounded to
// nearest in the order of the reference's expressions, no multiply-add
// fusion. It reproduces the reference's FP32 results, including the noise of
// its edge distances (dot(n, hit) + offset cancels most of its digits on
// small triangles far from the origin), for direct comparison with the
// reference's code; the default mode solves the hit point in FP64 instead.
__device__ __forceinline__ Geom window_fn_ref(float4 a4, float4 b4, float4 c4, float3 o, float3 d, float t,
                                              float sigma) {
  using namespace vf;
  Geom g;
  const float3 A = make_float3(a4.x, a4.y, a4.z), B = make_float3(b4.x, b4.y, b4.z), C = make_float3(c4.x, c4.y, c4.z);
  const float3 hit = add(o, scale(d, t));
  const float la = __fsqrt_rn(dot(sub(B, C), sub(B, C)));
  const float lb = __fsqrt_rn(dot(sub(A, C), sub(A, C)));
  const float lc = __fsqrt_rn(dot(sub(A, B), sub(A, B)));
  const float3 num = add(add(scale(A, la), scale(B, lb)), scale(C, lc));
  const float3 inc = scale(num, div(1.0f, add(add(la, lb), lc)));
  const float3 ec = cross(sub(B, A), sub(C, A));
  g.n = normalize(ec);
  const float3 P[3] = {A, B, C};
  float dist = 0.f, phi = -INFINITY;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const float3 p1 = P[i], p2 = P[(i + 1) % 3];
    float3 en = normalize(cross(ec, sub(p1, p2)));
    float offset = -dot(en, p1);
    if (i == 0) {
      dist = add(dot(en, inc), offset);
      if (dist > 0.0f) {
        en = neg(en);
        offset = -offset;
        dist = -dist;
      }
    }
    const float ed = add(dot(en, hit), offset);
    phi = fmaxf(phi, ed);
    g.d[i] = ed;
  }
  g.phi_max = phi;
  g.phi_final = div(phi, dist);
  g.Cx = (g.phi_final >= 0.0f) ? powf(g.phi_final, sigma) : 0.0f;
  g.q = sub(hit, A);
  g.e1 = sub(B, A);
  g.e2 = sub(C, A);
  g.t = t;
  return g;
}

// Geometry of a hit in the given shading mode.
template <int MODE>
__device__ __forceinline__ Geom shade_geom(float4 a, float4 b, float4 c, float3 o, float3 d, float t, float sigma) {
  if constexpr (MODE == kShadeRefArith)
    return window_fn_ref(a, b, c, o, d, t, sigma);
  else
    return window_fn(a, b, c, o, d, sigma);
}

__device__ __constant__ float c_sh2[5] = {1.0925484305920792f, -1.0925484305920792f, 0.31539156525252005f,
                                          -1.0925484305920792f, 0.5462742152960396f};
__device__ __constant__ float c_sh3[7] = {-0.5900435899266435f, 2.890611442640554f, -0.4570457994644658f,
                                          0.3731763325901154f, -0.4570457994644658f, 1.445305721320277f,
                                          -0.5900435899266435f};
constexpr float kSH0 = 0.28209479177387814f;
constexpr float kSH1 = 0.4886025119029199f;

// Degree-<=3 SH basis (tritracer/common.h:16-55, auxiliary.h:13-30).
__device__ __forceinline__ void sh_basis(float3 u, int deg, float (&B)[16]) {
  const float x = u.x, y = u.y, z = u.z;
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
    const float4* q = reinterpret_cast<const float4*>(base);  // 192-byte rows, 16-byte aligned
#pragma unroll
    for (int i = 0; i < 12; ++i) {
      const float4 w = __ldg(q + i);
      const float v[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int idx = 4 * i + j, k = idx / 3, ch = idx % 3;
        if (ch == 0) r = fmaf(B[k], v[j], r);
        else if (ch == 1) g = fmaf(B[k], v[j], g);
        else b = fmaf(B[k], v[j], b);
      }
    }
  } else {
    const int n = sh_count(deg);
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      if (k < n) {
        r = fmaf(B[k], __ldg(base + 3 * k), r);
        g = fmaf(B[k], __ldg(base + 3 * k + 1), g);
        b = fmaf(B[k], __ldg(base + 3 * k + 2), b);
      }
    }
  }
  return make_float3(r + 0.5f, g + 0.5f, b + 0.5f);
}

__device__ __forceinline__ float3 unit(float3 d) {
  const float inv = 1.0f / sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
  return make_float3(d.x * inv, d.y * inv, d.z * inv);
}

// computeScaling of tritracer/forward.cu:25-74 (first blending ray records the
// largest angle the vertices subtend around the centroid direction), in FP64.
__device__ __noinline__ void compute_scaling(float* __restrict__ scaling, const float* __restrict__ verts,
                                             const int* __restrict__ cumsum, const int* __restrict__ num_points,
                                             int prim, float3 of) {
  if (scaling[prim] > 0.0f) return;
  const int off = cumsum[prim], np = num_points[prim];
  const d3 o = mkd(of.x, of.y, of.z);
  d3 cen = mkd(0, 0, 0);
  for (int i = 0; i < np; ++i) {
    const float* v = verts + 3 * (size_t)(off + i);
    cen = cen + mkd(v[0], v[1], v[2]);
  }
  cen = cen * (1.0 / (double)np);
  const d3 t2o = cen - o;
  double best = 0.0;
  for (int i = 0; i < np; ++i) {
    const float* v = verts + 3 * (size_t)(off + i);
    const d3 a = mkd(v[0], v[1], v[2]) - o;
    const double lab = len(a) * len(t2o);
    double ang = 0.0;
    if (!(lab < 1e-12)) ang = acos(fmax(-1.0, fmin(1.0, dot(a, t2o) / lab)));
    best = fmax(ang, best);
  }
  scaling[prim] = (float)best;
}

// computeScaling in the reference's own FP32 arithmetic (forward.cu:25-74:
// centroid as a sum times 1/n, angle = acos of the clamped cosine), for the
// reference-arithmetic mode; the default computes it in FP64 above.
__device__ __noinline__ void compute_scaling_ref(float* __restrict__ scaling, const float* __restrict__ verts,
                                                 const int* __restrict__ cumsum, const int* __restrict__ num_points,
                                                 int prim, float3 o) {
  using namespace vf;
  if (scaling[prim] > 0.0f) return;
  const int off = cumsum[prim], np = num_points[prim];
  float3 cen = make_float3(0.f, 0.f, 0.f);
  for (int i = 0; i < np; ++i) {
    const float* v = verts + 3 * (size_t)(off + i);
    cen = add(cen, make_float3(v[0], v[1], v[2]));
  }
  cen = scale(cen, div(1.0f, (float)np));
  const float3 t2o = sub(cen, o);
  const float lt = __fsqrt_rn(dot(t2o, t2o));
  float best = 0.0f;
  for (int i = 0; i < np; ++i) {
    const float* v = verts + 3 * (size_t)(off + i);
    const float3 a = sub(make_float3(v[0], v[1], v[2]), o);
    const float lab = mul(__fsqrt_rn(dot(a, a)), lt);
    float ang = 0.0f;
    if (!(lab < 1e-12f)) ang = acosf(fmaxf(-1.0f, fminf(1.0f, div(dot(a, t2o), lab))));
    best = fmaxf(ang, best);
  }
  scaling[prim] = best;
}

// ---------------------------------------------------------------- the march
// Per-thread shared memory: the traversal stack and the 16 keys of the
// current chunk (staged out of registers before shading starts).
struct Smem {
  Stack st;
  unsigned long long* keys;
  int stride;
};

template <int SD>
__device__ __forceinline__ Smem thread_smem() {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem s;
  const int nt = blockDim.x;
  unsigned long long* keys = reinterpret_cast<unsigned long long*>(smem_raw);
  uint32_t* refs = reinterpret_cast<uint32_t*>(smem_raw + (size_t)kChunk * nt * 8);
  float* tns = reinterpret_cast<float*>(refs + (size_t)SD * nt);
  s.keys = keys + threadIdx.x;
  s.stride = nt;
  s.st.ref = refs + threadIdx.x;
  s.st.tn = tns + threadIdx.x;
  s.st.stride = nt;
  return s;
}

// Where a ray's next k-closest query starts, where it is inside the
// reference's 16-hit chunk, and the far bound of its queries (the far plane,
// or the end of a proposed interval until the ray leaves it).
struct Cursor {
  unsigned long long key_min;
  float last_hit_t;
  float t_hi;
  int ref_pos;
  int chunks;
};

__device__ __forceinline__ unsigned long long first_key(int tmin_inclusive) {
  return tmin_inclusive ? 0ull : (1ull << 32);
}

__device__ __forceinline__ Cursor first_cursor(int tmin_inclusive) {
  Cursor c;
  c.key_min = first_key(tmin_inclusive);
  c.last_hit_t = 0.f;
  c.t_hi = kFar;
  c.ref_pos = 0;
  c.chunks = 0;
  return c;
}

// Clips a ray's first query to the proposed interval [t_near, t_far]
// (interval planes [2][H][W]); a NaN or out-of-range bound falls back to the
// plain one.
__device__ __forceinline__ void clip_cursor(Cursor& c, const float* interval, int HW, int pix) {
  const float tn = __ldg(interval + pix), tf = __ldg(interval + HW + pix);
  if (tn > 0.f && tn < kFar) c.key_min = max(c.key_min, (unsigned long long)__float_as_uint(tn) << 32);
  if (tf >= 0.f && tf < kFar) c.t_hi = tf;
}

// Visits the keys of one query (K keys, ascending, staged in shared memory)
// in the reference's chunk order (forward.cu:99-154) and calls sh.visit(prim)
// for each hit at or beyond the near plane; visit returns true to end the ray
// (transmittance cut-off). Returns true when the ray is finished, else leaves
// in `cur` where the next query starts.
//
// The reference re-traces after every 16th visited hit from last_hit_t
// (closed interval: the hit(s) at last_hit_t come again) or just after it
// (open). A query buffer holds EVERY key between its lower bound and its last
// key, so the position "first key >= the new bound" is found inside the
// buffer whenever the buffer reaches it, and only otherwise does the next
// query start at that bound; after a full or truncated buffer the stream
// resumes right after the last key taken. The query size K is therefore a
// performance choice that never changes the visited sequence.
//
// Proposed intervals: when a clipped stream runs out (no key left below
// cur.t_hi) before the ray terminated, the ray is not finished: its queries go
// on from the next key with the far plane as bound (a continuation, counted
// in cnt.cont), or, if the interval held no hit at all, from the start of the
// ray (a plain re-trace, cnt.restart). Either way every hit at or beyond
// t_near is visited in the plain order.
template <int K, class Shader, class Cnt>
__device__ __forceinline__ bool consume_chunk(const Smem& sm, float t_drop, Cursor& cur, int tmin_inclusive,
                                              int* status, Shader& sh, Cnt& cnt) {
  const bool truncated = t_drop < INFINITY;
  auto trusted = [&](unsigned long long key) {
    return key != kEmptyKey && !(truncated && key_t(key) >= t_drop);
  };
  unsigned long long last_key = 0;
  bool any = false;
  // the stream ran out below cur.t_hi; `next` is where it would resume. A
  // shader that cannot end a ray (the collecting pass) stops there too: the
  // shading pass decides on continuations and re-traces.
  auto exhausted = [&](unsigned long long next) {
    if (cur.t_hi >= kFar || Shader::kStopsAtClip) return true;
    cur.t_hi = kFar;
    if (!any && cur.chunks == 0) {
      cur.key_min = first_key(tmin_inclusive);
      cnt.add_restart();
    } else {
      cur.key_min = next;
      cnt.add_cont();
    }
    return false;
  };
  int boundaries = 0;
  sh.prepare();
  int i = 0;
  while (i < K) {
    const unsigned long long key = sm.keys[i * sm.stride];
    if (!trusted(key)) break;
    any = true;
    last_key = key;
    const float t = key_t(key);
    // fmaxf(last + STEP_EPSILON, t) with the sum in double (forward.cu:111)
    cur.last_hit_t = fmaxf(__double2float_rn(__dadd_rn((double)cur.last_hit_t, kStepEps)), t);
    ++cur.ref_pos;
    if (!TT_IN_BOUNDS(status, key_prim(key) < (uint32_t)sh.p.bvh.P)) return true;
    if (t >= kNear && visit_slot(sh, key_prim(key), t, i, 0)) return true;
    if (cur.ref_pos == kChunk) {
      // the reference's next optixTrace starts at last_hit_t
      cur.ref_pos = 0;
      const unsigned long long tb = __float_as_uint(cur.last_hit_t);
      const unsigned long long bound = tmin_inclusive ? (tb << 32) : ((tb + 1ull) << 32);
      if (++boundaries > K) {  // 16+ hits at one t under the closed interval: no progress
        atomicOr(status, kStatusTimeout);
        return true;
      }
      int j = 0;
      while (j < K && trusted(sm.keys[j * sm.stride]) && sm.keys[j * sm.stride] < bound) ++j;
      if (j < K && trusted(sm.keys[j * sm.stride])) {
        i = j;  // continue inside the buffer
        continue;
      }
      if (j < K && sm.keys[j * sm.stride] == kEmptyKey && !truncated) return exhausted(bound);
      cur.key_min = bound;
      return false;
    }
    ++i;
  }
  if (i < K && sm.keys[i * sm.stride] == kEmptyKey && !truncated)
    return exhausted(any ? last_key + 1ull : cur.key_min);
  if (!any) {
    atomicOr(status, kStatusStack);  // a truncated query that trusted nothing
    return true;
  }
  cur.key_min = last_key + 1ull;
  return false;
}

// View holding global tile `tile` (views are stored in tile order).
__device__ __forceinline__ int find_view(const TraceParams& p, int tile) {
  int lo = 0, hi = p.nviews - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (p.views[mid].tile_begin <= tile)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// Hit cache (HitCacheHeader): the forward stores every query of a ray, the
// adjoint replays them. Rows are written and read once, so they bypass L2
// residency (streaming stores / loads) and leave it to the BVH.
__device__ __forceinline__ HitCacheHeader* cache_header_ptr(const TraceParams& p) {
  return static_cast<HitCacheHeader*>(p.hit_cache);
}
__device__ __forceinline__ unsigned long long* cache_main(const TraceParams& p) {
  return reinterpret_cast<unsigned long long*>(static_cast<char*>(p.hit_cache) + sizeof(HitCacheHeader));
}
template <int K>
__device__ __forceinline__ unsigned long long* cache_pool(const TraceParams& p) {
  return cache_main(p) + (size_t)(K + 1) * p.cache_rays;
}

template <int K>
__device__ __forceinline__ bool cache_replays(const TraceParams& p) {
  if (p.cache_mode != kCacheRead && p.cache_mode != kCacheFill) return false;
  const HitCacheHeader* h = cache_header_ptr(p);
  return h->magic == kHitCacheMagic && (h->k & ~kCacheColorsFlag) == (uint32_t)K && h->rays == p.cache_rays &&
         h->gen == p.cache_gen && h->pool_cap == p.cache_pool_cap;
}

// The forward stored every query it made: no pool entry was refused (a
// missing query always follows a refusal, and pool_used counts refused
// requests too). The adjoint can then replay every query of every march.
template <int K>
__device__ __forceinline__ bool cache_complete(const TraceParams& p) {
  return cache_replays<K>(p) && cache_header_ptr(p)->pool_used <= p.cache_pool_cap;
}

// Hit colours beside the queries (plain forward / adjoint of the packet
// drivers): the forward's shading kernels store them, the adjoint reads them
// when the header says they were written.
__device__ __forceinline__ bool cache_colors_on(const TraceParams& p) {
  if (!p.cache_colors || p.cols) return false;
  return p.cache_mode != kCacheRead || (cache_header_ptr(p)->k & kCacheColorsFlag) != 0u;
}
// Colour rows of the main-part entry of ray g or of pool entry e (row 3i + c
// holds channel c of slot i; `stride` floats between rows). Both counts fit
// an int: every entry takes over 400 bytes of the buffer.
template <int K>
__device__ __forceinline__ float* cache_color_rows(const TraceParams& p, bool main_part, long long g, uint32_t e,
                                                   int& stride) {
  if (main_part) {
    stride = (int)p.cache_rays;
    return p.cache_colors + g;
  }
  stride = (int)p.cache_pool_cap;
  return p.cache_colors + (size_t)3 * K * p.cache_rays + e;
}

// Shaders that use the colour rows take them and the hit's slot; the others
// ignore both.
template <class S>
__device__ __forceinline__ auto set_color_rows(S& sh, float* rows, int stride, int) -> decltype(sh.set_colors(rows, stride)) {
  sh.set_colors(rows, stride);
}
template <class S>
__device__ __forceinline__ void set_color_rows(S&, float*, int, long) {}
template <class S>
__device__ __forceinline__ auto visit_slot(S& sh, uint32_t prim, float t, int slot, int) -> decltype(sh.visit(prim, t, slot)) {
  return sh.visit(prim, t, slot);
}
template <class S>
__device__ __forceinline__ bool visit_slot(S& sh, uint32_t prim, float t, int, long) {
  return sh.visit(prim, t);
}

// Forward, first query of ray g. Returns where the entry of its next query
// gets linked (the high half of row k).
template <int K>
__device__ __forceinline__ uint32_t* cache_put_first(const TraceParams& p, long long g, const Smem& sm, float t_drop) {
  unsigned long long* rows = cache_main(p) + g;
  const size_t R = (size_t)p.cache_rays;
#pragma unroll 4
  for (int i = 0; i < K; ++i) __stcs(rows + i * R, sm.keys[i * sm.stride]);
  unsigned long long* w = rows + K * R;
  __stcs(w, ((unsigned long long)kNoEntry << 32) | __float_as_uint(t_drop));
  return reinterpret_cast<uint32_t*>(w) + 1;
}

// Forward, a later query into pool entry e (< pool_cap), linked from `link`.
template <int K>
__device__ __forceinline__ uint32_t* cache_put_more(const TraceParams& p, uint32_t e, unsigned long long key_min,
                                                    const Smem& sm, float t_drop, uint32_t* link) {
  unsigned long long* rows = cache_pool<K>(p) + e;
  const size_t C = p.cache_pool_cap;
#pragma unroll 4
  for (int i = 0; i < K; ++i) __stcs(rows + i * C, sm.keys[i * sm.stride]);
  unsigned long long* w = rows + K * C;
  __stcs(w, ((unsigned long long)kNoEntry << 32) | __float_as_uint(t_drop));
  __stcs(rows + (K + 1) * C, key_min);
  *link = e;
  return reinterpret_cast<uint32_t*>(w) + 1;
}

// Forward: pool entries for the lanes in `want` (one atomic per warp).
__device__ __forceinline__ uint32_t cache_alloc(const TraceParams& p, bool want) {
  const unsigned m = __ballot_sync(0xFFFFFFFFu, want);
  if (m == 0u) return kNoEntry;
  const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
  uint32_t base = 0u;
  if (lane == leader) base = atomicAdd(&cache_header_ptr(p)->pool_used, (uint32_t)__popc(m));
  base = __shfl_sync(0xFFFFFFFFu, base, leader);
  return want ? base + (uint32_t)__popc(m & ((1u << lane) - 1u)) : kNoEntry;
}

// Adjoint: fills the lane's query buffer from the first query of ray g or
// from pool entry e; returns t_drop and the entry of the next query.
template <int K>
__device__ __forceinline__ float cache_get(const TraceParams& p, bool first, long long g, uint32_t e, const Smem& sm,
                                           uint32_t& next) {
  const unsigned long long* rows = first ? cache_main(p) + g : cache_pool<K>(p) + e;
  const size_t S = first ? (size_t)p.cache_rays : (size_t)p.cache_pool_cap;
#pragma unroll 4
  for (int i = 0; i < K; ++i) sm.keys[i * sm.stride] = __ldcs(rows + i * S);
  const unsigned long long w = __ldcs(rows + K * S);
  next = (uint32_t)(w >> 32);
  return __uint_as_float((uint32_t)w);
}

// Fill mode: the word where the entry of the query after the one replayed
// from the main part (first) or from pool entry e gets linked.
template <int K>
__device__ __forceinline__ uint32_t* cache_link_of(const TraceParams& p, bool first, long long g, uint32_t e) {
  unsigned long long* w = first ? cache_main(p) + g + (size_t)K * p.cache_rays
                                : cache_pool<K>(p) + e + (size_t)K * p.cache_pool_cap;
  return reinterpret_cast<uint32_t*>(w) + 1;
}

// Adjoint: does pool entry e hold the query that starts at key_min?
template <int K>
__device__ __forceinline__ bool cache_has(const TraceParams& p, uint32_t e, unsigned long long key_min) {
  return e < p.cache_pool_cap && __ldcs(cache_pool<K>(p) + (size_t)(K + 1) * p.cache_pool_cap + e) == key_min;
}

template <int K>
__device__ __forceinline__ void cache_header(const TraceParams& p, bool colors = false) {
  if (p.cache_mode == kCacheWrite && blockIdx.x == 0 && threadIdx.x == 0) {
    HitCacheHeader* h = cache_header_ptr(p);  // pool_used was zeroed by the host
    h->magic = kHitCacheMagic;
    h->k = K | (colors ? kCacheColorsFlag : 0u);  // colours: the shading kernels store them
    h->rays = p.cache_rays;
    h->gen = p.cache_gen;
    h->pool_cap = p.cache_pool_cap;
  }
}

// Persistent warp driver. Each round: lanes without a ray take the next rays
// of the tile-ordered image (8x4 pixels per 32 slots) from the global counter,
// then every lane holding a ray runs its k-closest query, then every such lane
// shades its chunk. Traversal and shading never mix inside a warp, and lanes
// whose ray finished are refilled instead of idling.
template <int SD, class Shader>
__device__ __forceinline__ void drive(const TraceParams& p, const Smem& sm, Shader& sh, Counters& cnt) {
  constexpr int K = kChunk;  // hits per per-lane query
  const unsigned full = 0xFFFFFFFFu;
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  const int total = p.ntiles * 32;
  bool have = false, exhausted = false;
  Cursor cur = first_cursor(p.tmin_inclusive);
  float3 o = make_float3(0.f, 0.f, 0.f), d = o;
  long long g = 0;              // hit cache index of the lane's ray
  uint32_t* link = nullptr;     // forward: where the entry of the ray's next query gets linked
  uint32_t next = kNoEntry;     // adjoint: entry of the ray's next query
  const bool replay = cache_replays<K>(p);
  for (;;) {
    const unsigned need = __ballot_sync(full, !have && !exhausted);
    if (need) {
      const int leader = __ffs(need) - 1;
      int base = 0;
      if (lane == leader) base = atomicAdd(p.work, __popc(need));
      base = __shfl_sync(full, base, leader);
      if (!have && !exhausted) {
        const int slot = base + __popc(need & lt);
        if (slot >= total) {
          exhausted = true;
        } else {
          const int tile = slot >> 5, l = slot & 31;
          const ViewDesc& v = p.views[find_view(p, tile)];
          const int lt = tile - v.tile_begin;
          const int px = (lt % v.ntx) * 8 + (l & 7), py = (lt / v.ntx) * 4 + (l >> 3);
          if (px < v.W && py < v.H) {
            const int pix = py * v.W + px;
            o = make_float3(v.ray_o[3 * pix], v.ray_o[3 * pix + 1], v.ray_o[3 * pix + 2]);
            d = make_float3(v.ray_d[3 * pix], v.ray_d[3 * pix + 1], v.ray_d[3 * pix + 2]);
            g = v.ray_begin + pix;
            cur = first_cursor(p.tmin_inclusive);
            if (v.interval) clip_cursor(cur, v.interval, v.H * v.W, pix);
            if (sh.begin(&v, pix, o, d))
              have = true;
            else
              sh.end();
          }
        }
      }
    }
    if (__ballot_sync(full, have) == 0) {
      if (__all_sync(full, exhausted)) break;
      continue;
    }
    float t_drop = INFINITY;
    if (have) {
      const bool first = cur.chunks == 0;  // the ray's queries are numbered by its chunks
      if (replay && (first || cache_has<K>(p, next, cur.key_min))) {  // as the forward found it
        if (p.cache_mode == kCacheFill) link = cache_link_of<K>(p, first, g, next);
        t_drop = cache_get<K>(p, first, g, next, sm, next);
        ++cnt.replays;
      } else {
        next = kNoEntry;
        const RayW r = make_ray(o, d);
        query<SD>(p.bvh, r, cur.key_min, cur.t_hi, sm.keys, sm.stride, sm.st, t_drop, p.status, cnt, p.count_work);
        if (p.cache_mode == kCacheWrite || p.cache_mode == kCacheFill) {
          if (first) {
            link = cache_put_first<K>(p, g, sm, t_drop);
          } else if (link) {
            const uint32_t e = atomicAdd(&cache_header_ptr(p)->pool_used, 1u);
            link = e < p.cache_pool_cap ? cache_put_more<K>(p, e, cur.key_min, sm, t_drop, link) : nullptr;
          }
        }
      }
    }
    __syncwarp();
    if (have) {
      bool done = consume_chunk<K>(sm, t_drop, cur, p.tmin_inclusive, p.status, sh, cnt);
      if (!done && ++cur.chunks >= kMaxChunks) {
        atomicOr(p.status, kStatusTimeout);
        done = true;
      }
      // the collecting pass stores at most collect_queries queries a ray
      if (Shader::kStopsAtClip && p.collect_queries > 0 && cur.chunks >= p.collect_queries) done = true;
      if (done) {
        if (sh.next(o, d)) {  // another ray of the same pixel (envlight samples)
          cur = first_cursor(p.tmin_inclusive);
        } else {
          sh.end();
          have = false;
        }
      }
    }
  }
}

// Packet driver: a warp takes an 8x4-pixel tile, then runs rounds of one
// packet query (all lanes whose ray is unfinished) and one shading pass until
// every ray of the tile is done.
__device__ __forceinline__ WarpStack warp_stack(unsigned char* base) {
  const int w = threadIdx.x >> 5;
  WarpStack ws;
  ws.ref = reinterpret_cast<uint32_t*>(base) + w * kWarpStack;
  ws.mask = reinterpret_cast<unsigned*>(base + (size_t)(blockDim.x / 32) * kWarpStack * 4) + w * kWarpStack;
  ws.tmin = reinterpret_cast<float*>(base + (size_t)(blockDim.x / 32) * kWarpStack * 8) + w * kWarpStack;
  ws.cnt = reinterpret_cast<unsigned*>(base + (size_t)(blockDim.x / 32) * kWarpStack * 12) + w * kWCounters;
  return ws;
}

// kReplayOnly: every query comes from the hit cache (the adjoint given a
// complete cache); the build carries no traversal code, which leaves the
// shading arithmetic more registers. A query the cache lacks (which a
// complete cache never does) ends that ray and sets kStatusCacheMiss.
template <int K, class Shader, bool kReplayOnly = false>
__device__ __forceinline__ void drive_packets(const TraceParams& p, const Smem& sm, WarpStack ws, Shader& sh,
                                              Counters& cnt) {
  const unsigned full = 0xFFFFFFFFu;
  const int lane = threadIdx.x & 31;
  const bool replay = cache_replays<K>(p);
  const bool colors = cache_colors_on(p);
  if (lane < kWCounters) ws.cnt[lane] = 0u;
  __syncwarp();
  WarpCounters wc{ws.cnt};
  for (;;) {
    int tile = 0;
    if (lane == 0) tile = atomicAdd(p.work, 1);
    tile = __shfl_sync(full, tile, 0);
    if (tile >= p.ntiles) break;
    const ViewDesc& v = p.views[find_view(p, tile)];
    const int lt = tile - v.tile_begin;
    const int px = (lt % v.ntx) * 8 + (lane & 7), py = (lt / v.ntx) * 4 + (lane >> 3);
    bool active = px < v.W && py < v.H;
    float3 o = make_float3(0.f, 0.f, 1.f), d = make_float3(0.f, 0.f, 1.f);
    Cursor cur = first_cursor(p.tmin_inclusive);
    long long g = 0;  // hit cache index of the lane's ray
    if (active) {
      const int pix = py * v.W + px;
      g = v.ray_begin + pix;
      o = make_float3(v.ray_o[3 * pix], v.ray_o[3 * pix + 1], v.ray_o[3 * pix + 2]);
      d = make_float3(v.ray_d[3 * pix], v.ray_d[3 * pix + 1], v.ray_d[3 * pix + 2]);
      if (v.interval) clip_cursor(cur, v.interval, v.H * v.W, pix);
      sh.begin(&v, pix, o, d);  // the plain shaders always trace their one ray
    }
    const RayW r = make_ray(o, d);
    uint32_t* link = nullptr;  // forward: where the entry of the ray's next query gets linked
    uint32_t next = kNoEntry;  // adjoint: entry of the ray's next query
    for (bool first = true; __any_sync(full, active); first = false) {
      float t_drop = INFINITY;
      // lanes whose query the forward stored replay it; the others traverse
      const bool rep = replay && active && (first || cache_has<K>(p, next, cur.key_min));
      const bool trav = active && !rep;
      if constexpr (kReplayOnly) {
        if (trav) {
          atomicOr(p.status, kStatusCacheMiss);
          active = false;
        }
      } else {
        if (__any_sync(full, trav))
          packet_query<K>(p.bvh, r, trav, cur.key_min, cur.t_hi, sm.keys, sm.stride, ws, t_drop, p.status,
                          p.count_work);
      }
      const unsigned nrep = __popc(__ballot_sync(full, rep));
      if (lane == 0) ws.cnt[kWReplays] += nrep;
      // the cache entry holding this query, if any: its colour rows
      bool in_main = false;
      uint32_t entry = kNoEntry;
      if (rep) {
        in_main = first;
        entry = next;
        if (p.cache_mode == kCacheFill) link = cache_link_of<K>(p, first, g, next);
        t_drop = cache_get<K>(p, first, g, next, sm, next);
      } else {
        next = kNoEntry;
      }
      if (p.cache_mode == kCacheWrite || p.cache_mode == kCacheFill) {
        if (first) {
          if (trav) {
            link = cache_put_first<K>(p, g, sm, t_drop);
            in_main = true;
          }
        } else {
          const bool more = trav && link != nullptr;
          const uint32_t e = cache_alloc(p, more);
          if (more) {
            link = e < p.cache_pool_cap ? cache_put_more<K>(p, e, cur.key_min, sm, t_drop, link) : nullptr;
            if (e < p.cache_pool_cap) entry = e;
          }
        }
      }
      if (colors) {
        int stride = 0;
        float* rows = (in_main || entry != kNoEntry) ? cache_color_rows<K>(p, in_main, g, entry, stride) : nullptr;
        set_color_rows(sh, rows, stride, 0);
      }
      if (active) {
        bool done = consume_chunk<K>(sm, t_drop, cur, p.tmin_inclusive, p.status, sh, wc);
        if (!done && ++cur.chunks >= kMaxChunks) {
          atomicOr(p.status, kStatusTimeout);
          done = true;
        }
        // the collecting pass stores at most collect_queries queries a ray
        if (Shader::kStopsAtClip && p.collect_queries > 0 && cur.chunks >= p.collect_queries) done = true;
        if (done) {
          sh.end();
          active = false;
        }
      }
    }
  }
  // the warp's counters into lane 0's Counters (summed over the warp later)
  __syncwarp();
  if (lane == 0) {
    cnt.nodes += ws.cnt[kWNodes];
    cnt.tris += ws.cnt[kWTris];
    cnt.warp_nodes += ws.cnt[kWWarpNodes];
    cnt.queries += ws.cnt[kWQueries];
    cnt.replays += ws.cnt[kWReplays];
    cnt.cont += ws.cnt[kWCont];
    cnt.restart += ws.cnt[kWRestart];
  }
}

template <int K>
__device__ __forceinline__ Smem packet_smem(unsigned char*& rest) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem s;
  s.keys = reinterpret_cast<unsigned long long*>(smem_raw) + threadIdx.x;
  s.stride = blockDim.x;
  s.st.ref = nullptr;
  s.st.tn = nullptr;
  s.st.stride = 0;
  rest = smem_raw + (size_t)K * blockDim.x * 8;
  return s;
}

// Traversal configurations the kernels are instantiated for (the autotuner
// picks one per workload): warp packets with 16 or 32 hits per query, or
// independent lanes with a 32- or 24-entry stack per ray.
template <int CFG>
struct TraversalCfg;
template <>
struct TraversalCfg<kCfgLanes32> {
  static constexpr bool packets = false;
  static constexpr int K = 16, SD = 32;
};
template <>
struct TraversalCfg<kCfgPackets16> {
  static constexpr bool packets = true;
  static constexpr int K = 16, SD = 0;
};
template <>
struct TraversalCfg<kCfgPackets32> {
  static constexpr bool packets = true;
  static constexpr int K = 32, SD = 0;
};
template <>
struct TraversalCfg<kCfgLanes24> {
  static constexpr bool packets = false;
  static constexpr int K = 16, SD = 24;
};

template <int CFG>
constexpr size_t smem_bytes_for() {
  using C = TraversalCfg<CFG>;
  return C::packets ? (size_t)kTraceThreads * C::K * 8 + (size_t)(kTraceThreads / 32) * (kWarpStack * 12 + kWCounters * 4)
                    : (size_t)kTraceThreads * (C::SD * 8 + kChunk * 8);
}

// Exact-adjoint forward: per-thread shared-memory words after the traversal's
// shared memory (FwdShader<true>).
constexpr int kXD = 0, kXWsum = 1, kXWt2 = 2, kXMid = 3, kXDist2 = 4, kXMidSet = 5, kExactSlots = 6;
constexpr size_t kExactSmemBytes = (size_t)kTraceThreads * kExactSlots * 4;

template <int CFG, class Shader, bool kReplayOnly = false>
__device__ __forceinline__ void run(const TraceParams& p, Shader& sh, Counters& cnt) {
  using C = TraversalCfg<CFG>;
  if constexpr (C::packets) {
    unsigned char* rest;
    const Smem sm = packet_smem<C::K>(rest);
    drive_packets<C::K, Shader, kReplayOnly>(p, sm, warp_stack(rest), sh, cnt);
  } else {
    drive<C::SD>(p, thread_smem<C::SD>(), sh, cnt);
  }
}

// ---------------------------------------------------------------- forward
__device__ __forceinline__ void add_stats(unsigned long long* stats, unsigned rays, unsigned evals, unsigned blends,
                                          const Counters& c) {
  const unsigned v[kNumStats] = {rays,         evals,   blends,    c.nodes,   c.tris,
                                 c.queries,    c.warp_nodes, c.cont, c.restart, c.replays};
#pragma unroll
  for (int i = 0; i < kNumStats; ++i) {
    const unsigned s = __reduce_add_sync(0xFFFFFFFFu, v[i]);
    if ((threadIdx.x & 31) == 0) atomicAdd(stats + i, (unsigned long long)s);
  }
}

// forward.cu:109-152 per hit and :204-214 per ray. EXACT (no reference
// counterpart) also fills the channels the reference leaves at 0: depth
// sum w t, middepth (t of the hit after which T <= 0.5) and distortion
// sum_{i<j} w_i w_j (t_i - t_j)^2 (running sums of w and w t^2).
template <int MODE>
struct FwdShader {
  static constexpr bool EXACT = MODE == kShadeExact;
  static constexpr bool kStopsAtClip = false;
  const TraceParams& p;
  const ViewDesc* v;
  int pix;
  float3 o, d;
  float C0, C1, C2, N0, N1, N2, T;
  // EXACT only: the ray's depth sums, middepth and distortion live in a
  // per-thread shared-memory slot (kExactSlots words, stride blockDim.x), so
  // the traversal between two shading passes does not carry them in registers
  float* xs = nullptr;
  // colour rows of the current query's hit-cache entry (raw colour of the
  // hit in slot i at rows 3i..3i+2, `cstride` floats apart), or nullptr
  float* crow = nullptr;
  int cstride = 0;
  unsigned n_rays = 0, n_eval = 0, n_blend = 0;
  unsigned first_eval = 0;  // value of n_eval at the ray's first hit (record only)

  __device__ FwdShader(const TraceParams& params, size_t exact_offset) : p(params) {
    if (EXACT) {
      extern __shared__ __align__(16) unsigned char smem_raw[];
      xs = reinterpret_cast<float*>(smem_raw + exact_offset) + threadIdx.x;
    }
  }
  __device__ __forceinline__ float& x(int i) { return xs[i * blockDim.x]; }

  __device__ __forceinline__ bool begin(const ViewDesc* view, int pixel, float3 ro, float3 rd) {
    v = view;
    pix = pixel;
    o = ro;
    d = rd;
    C0 = C1 = C2 = N0 = N1 = N2 = 0.f;
    if (EXACT) {
#pragma unroll
      for (int i = 0; i < kExactSlots; ++i) x(i) = 0.f;
    }
    T = 1.0f;
    ++n_rays;
    if (v->record) {
      // t of the first and last hit visited, and whether the ray terminated
      const int HW = v->H * v->W;
      v->record[pix] = INFINITY;
      v->record[HW + pix] = INFINITY;
      v->record[2 * HW + pix] = 0.0f;
      first_eval = n_eval + 1;
    }
    return true;
  }

  __device__ __forceinline__ bool next(float3&, float3&) { return false; }

  __device__ __forceinline__ void prepare() {}

  __device__ __forceinline__ void set_colors(float* rows, int stride) {
    crow = rows;
    cstride = stride;
  }

  __device__ __forceinline__ bool visit(uint32_t prim, float t) { return visit(prim, t, -1); }

  // `slot`: the hit's position in its query (colour rows), -1 if unknown
  __device__ __forceinline__ bool visit(uint32_t prim, float t, int slot) {
    const float4* tr = p.bvh.tri_prim + 3 * (size_t)prim;
    const Geom g = shade_geom<MODE>(__ldg(tr), __ldg(tr + 1), __ldg(tr + 2), o, d, t, __ldg(p.sigma + prim));
    ++n_eval;
    float* rec = v->record;
    const int HW = v->H * v->W;
    if (rec) {
      if (n_eval == first_eval) rec[pix] = t;
      rec[HW + pix] = t;
    }
    const float alpha = fminf(kAlphaMax, __ldg(p.opac + prim) * g.Cx);
    if (alpha < kAlphaMin) return false;
    const float test_T = T * (1.0f - alpha);
    if (test_T < kTMin) {
      if (rec) rec[2 * HW + pix] = 1.0f;
      return true;
    }
    ++n_blend;
    p.density[prim] = 1.0f;
    if constexpr (MODE == kShadeRefArith)
      compute_scaling_ref(p.scaling, p.verts, p.cumsum, p.num_points, (int)prim, o);
    else
      compute_scaling(p.scaling, p.verts, p.cumsum, p.num_points, (int)prim, o);
    const float w = alpha * T;
    atomicMax(reinterpret_cast<int*>(p.max_blending) + prim, __float_as_int(w));
    N0 += g.n.x * w;
    N1 += g.n.y * w;
    N2 += g.n.z * w;
    if (EXACT) {
      const float ht = g.t;
      const float D = x(kXD), Wsum = x(kXWsum), Wt2 = x(kXWt2);
      x(kXDist2) += w * (ht * ht * Wsum - 2.0f * ht * D + Wt2);
      x(kXWsum) = Wsum + w;
      x(kXD) = D + w * ht;
      x(kXWt2) = Wt2 + w * ht * ht;
      if (x(kXMidSet) == 0.f && test_T <= 0.5f) {
        x(kXMid) = ht;
        x(kXMidSet) = 1.f;
      }
    }
    float3 c;
    if (p.cols) {  // precomputed colours in place of SH
      c = make_float3(__ldg(p.cols + 3 * prim), __ldg(p.cols + 3 * prim + 1), __ldg(p.cols + 3 * prim + 2));
    } else {
      float B[16];
      sh_basis(unit(d), p.sh_degree, B);
      const float3 raw = sh_raw(p.shs, p.M, (int)prim, p.sh_degree, B);
      c = make_float3(fmaxf(raw.x, 0.f), fmaxf(raw.y, 0.f), fmaxf(raw.z, 0.f));
      if (crow && slot >= 0) {  // for the adjoint, which then reads it instead of the SH
        crow[(size_t)(3 * slot) * cstride] = raw.x;
        crow[(size_t)(3 * slot + 1) * cstride] = raw.y;
        crow[(size_t)(3 * slot + 2) * cstride] = raw.z;
      }
    }
    C0 += c.x * w;
    C1 += c.y * w;
    C2 += c.z * w;
    T = test_T;
    return false;
  }

  __device__ __forceinline__ void end() {
    const int HW = v->H * v->W;
    v->out_color[pix] = C0 + T * p.bg[0];
    v->out_color[HW + pix] = C1 + T * p.bg[1];
    v->out_color[2 * HW + pix] = C2 + T * p.bg[2];
    v->out_others[kDepthCh * HW + pix] = EXACT ? x(kXD) : 0.0f;  // the reference never accumulates depth
    v->out_others[kAlphaCh * HW + pix] = 1.0f - T;
    v->out_others[(kNormalCh + 0) * HW + pix] = N0;
    v->out_others[(kNormalCh + 1) * HW + pix] = N1;
    v->out_others[(kNormalCh + 2) * HW + pix] = N2;
    v->out_others[kMidDepthCh * HW + pix] = EXACT ? x(kXMid) : 0.0f;
    v->out_others[kDistortionCh * HW + pix] = EXACT ? x(kXDist2) : 0.0f;
  }
};

// Blocks per SM the replay-only builds are compiled for (shading pass and
// adjoint): 4, as the traversing builds; at 5 the adjoint spilled 240 bytes
// a thread and took 5.4 ms instead of 5.0 on C2.
#ifndef TT_REPLAY_BLOCKS
#define TT_REPLAY_BLOCKS 4
#endif
constexpr int kReplayBlocks = TT_REPLAY_BLOCKS;

// REPLAY: the replay-only build for the shading pass of a split forward
// whose traversal-only pass stored every query of every march; launched as a
// pair with the traversing build (p.fwd_pair), like the adjoint.
template <int CFG, int MODE, bool REPLAY = false>
__global__ void __launch_bounds__(kTraceThreads, REPLAY ? kReplayBlocks : kMinBlocks) k_forward(const __grid_constant__ TraceParams p) {
  if (p.fwd_pair && cache_complete<TraversalCfg<CFG>::K>(p) != REPLAY) return;
  cache_header<TraversalCfg<CFG>::K>(p, TraversalCfg<CFG>::packets && p.cache_colors != nullptr);
  Counters cnt;
  FwdShader<MODE> sh(p, smem_bytes_for<CFG>());
  run<CFG, FwdShader<MODE>, REPLAY>(p, sh, cnt);
  // queries = those the march used, traversed here or replayed from the
  // collecting pass; hit_cache_replays counts the adjoint's replays only
  cnt.queries += cnt.replays;
  cnt.replays = 0;
  add_stats(p.stats, sh.n_rays, sh.n_eval, sh.n_blend, cnt);
}

// ---------------------------------------------------------------- collect
// Traversal-only pass of the split forward (plain program with a hit cache).
// It runs every ray's march with a shader that shades nothing and never ends
// a ray early, so it makes, and stores in the hit cache, every k-closest
// query the plain march would make. The shading pass (k_forward reading the
// cache) then replays each query its own march asks for; a ray that ends on
// the transmittance cut-off simply leaves its later queries unread, and a
// query the cache could not hold (pool full) is traversed again there. With
// no shading state or code the pass needs far fewer registers than the fused
// kernel, so more warps per SM hide the latency of the node and triangle
// loads, which is what bounds the traversal.
// 6 blocks of 128 threads (80 registers, ~60 bytes of spills a thread since
// the packet drivers keep their counters in shared memory): 24 warps per SM
// against the fused kernel's 16. Measured on 1M triangles, 4 x 800^2 rays,
// split forward storing two queries a ray: 15.4 ms at 6 blocks, 16.5 at 5
// (95 registers, no spills), fused 19.0 (one run, same box). With the
// counters in registers the 6-block build spilled ~170 bytes and was no
// faster than 5 blocks.
#ifndef TT_COLLECT_BLOCKS
#define TT_COLLECT_BLOCKS 6
#endif
constexpr int kCollectBlocks = TT_COLLECT_BLOCKS;

struct MarchShader {
  static constexpr bool kStopsAtClip = true;
  const TraceParams& p;
  __device__ explicit MarchShader(const TraceParams& params) : p(params) {}
  __device__ __forceinline__ bool begin(const ViewDesc*, int, float3, float3) { return true; }
  __device__ __forceinline__ bool next(float3&, float3&) { return false; }
  __device__ __forceinline__ void prepare() {}
  __device__ __forceinline__ bool visit(uint32_t, float) { return false; }
  __device__ __forceinline__ void end() {}
};

template <int CFG>
__global__ void __launch_bounds__(kTraceThreads, kCollectBlocks) k_collect(const __grid_constant__ TraceParams p) {
  cache_header<TraversalCfg<CFG>::K>(p, TraversalCfg<CFG>::packets && p.cache_colors != nullptr);
  Counters cnt;
  MarchShader sh(p);
  run<CFG>(p, sh, cnt);
  // the traversal work (node visits, triangle tests) only: rays, hits and the
  // queries the march used are counted by the shading pass
  cnt.queries = 0;
  add_stats(p.stats, 0u, 0u, 0u, cnt);
}

// ---------------------------------------------------------------- variants
// Sphere variants of the reference (tritracer/reflect.cu, refract.cu,
// envlight.cu, common.h:116-148), forward only as there. The analytic sphere
// is extra = [r, cx, cy, cz, samples]. The secondary-ray set-up repeats the
// reference's FP32 expressions with explicit round-to-nearest operations (no
// contraction), so the bent rays equal the oracle's.

struct VarShader {
  static constexpr bool kStopsAtClip = false;
  const TraceParams& p;
  const ViewDesc* v;
  int pix;
  float3 o, d;
  float C0, C1, C2, T;
  // envlight: the bent surface point, sample index and running radiance
  bool env;
  int sample;
  float3 so;
  float A0, A1, A2;
  unsigned n_rays = 0, n_eval = 0, n_blend = 0;

  __device__ explicit VarShader(const TraceParams& params) : p(params) {}

  __device__ __forceinline__ void env_ray(float3& ro, float3& rd) {
    const float3 cnt = make_float3(p.sph_cx, p.sph_cy, p.sph_cz);
    const float3 n = vf::normalize(vf::sub(so, cnt));
    uint32_t seed = ((uint32_t)(pix + 1u) * 9781u) ^ ((uint32_t)(sample + 1u) * 6271u);
    rd = vf::cosine_hemisphere(seed, n);
    ro = vf::add(so, vf::scale(rd, (float)kStepEps));
  }

  __device__ __forceinline__ bool begin(const ViewDesc* view, int pixel, float3& ro, float3& rd) {
    v = view;
    pix = pixel;
    C0 = C1 = C2 = 0.f;
    T = 1.0f;
    env = false;
    A0 = A1 = A2 = 0.f;
    ++n_rays;
    const float3 cnt = make_float3(p.sph_cx, p.sph_cy, p.sph_cz);
    const float eps = (float)kStepEps;
    float st;
    const bool hit = vf::hit_sphere(p.sph_r, cnt, ro, rd, st);
    if (p.variant == 1) {  // reflect.cu:42-48
      if (hit) {
        ro = vf::add(ro, vf::scale(rd, st));
        const float3 n = vf::normalize(vf::sub(ro, cnt));
        ro = vf::add(ro, vf::scale(n, eps));
        rd = vf::reflect(vf::normalize(rd), n);
      }
    } else if (p.variant == 2) {  // refract.cu:47-71
      if (hit) {
        const float3 hp = vf::add(ro, vf::scale(rd, st));
        const float3 n = vf::normalize(vf::sub(hp, cnt));
        const float3 in = vf::normalize(rd);
        const float ior = vf::div(1.5f, 1.0003f);
        float3 nd = in;
        if (!vf::refract_dir(nd, in, n, ior)) nd = vf::reflect(in, vf::dot(in, n) < 0.0f ? n : vf::neg(n));
        ro = vf::add(hp, vf::scale(n, eps));
        rd = nd;
      }
    } else if (hit) {  // envlight.cu:116-166
      so = vf::add(ro, vf::scale(rd, st));
      so = vf::add(so, vf::scale(vf::normalize(vf::sub(so, cnt)), eps));
      env = true;
      sample = 0;
      if (p.samples <= 0) return false;
      env_ray(ro, rd);
    }
    o = ro;
    d = rd;
    return true;
  }

  __device__ __forceinline__ void prepare() {}

  __device__ __forceinline__ bool visit(uint32_t prim, float) {
    const float4* tr = p.bvh.tri_prim + 3 * (size_t)prim;
    const Geom g = window_fn(__ldg(tr), __ldg(tr + 1), __ldg(tr + 2), o, d, __ldg(p.sigma + prim));
    ++n_eval;
    const float alpha = fminf(kAlphaMax, __ldg(p.opac + prim) * g.Cx);
    if (alpha < kAlphaMin) return false;
    const float test_T = T * (1.0f - alpha);
    if (test_T < kTMin) return true;
    ++n_blend;
    const float w = alpha * T;
    float B[16];
    sh_basis(unit(d), p.sh_degree, B);
    const float3 c = sh_raw(p.shs, p.M, (int)prim, p.sh_degree, B);
    C0 += fmaxf(c.x, 0.f) * w;
    C1 += fmaxf(c.y, 0.f) * w;
    C2 += fmaxf(c.z, 0.f) * w;
    T = test_T;
    return false;
  }

  __device__ __forceinline__ bool next(float3& ro, float3& rd) {
    if (!env) return false;
    A0 += C0 + T * p.bg[0];
    A1 += C1 + T * p.bg[1];
    A2 += C2 + T * p.bg[2];
    if (++sample >= p.samples) return false;
    C0 = C1 = C2 = 0.f;
    T = 1.0f;
    env_ray(ro, rd);
    o = ro;
    d = rd;
    return true;
  }

  __device__ __forceinline__ void end() {
    const int HW = v->H * v->W;
    if (env) {  // mean sample radiance; transmittance 0
      const float inv = 1.0f / (float)p.samples;
      C0 = A0 * inv;
      C1 = A1 * inv;
      C2 = A2 * inv;
      T = 0.0f;
    }
    v->out_color[pix] = C0 + T * p.bg[0];
    v->out_color[HW + pix] = C1 + T * p.bg[1];
    v->out_color[2 * HW + pix] = C2 + T * p.bg[2];
#pragma unroll
    for (int c = 0; c < 7; ++c) v->out_others[c * HW + pix] = 0.0f;  // variants write colour only
  }
};

__global__ void __launch_bounds__(kTraceThreads, 4) k_variant(const __grid_constant__ TraceParams p) {
  Counters cnt;
  VarShader sh(p);
  drive<32>(p, thread_smem<32>(), sh, cnt);
  add_stats(p.stats, sh.n_rays, sh.n_eval, sh.n_blend, cnt);
}

// ---------------------------------------------------------------- adjoint
// Gradient of phi_max through the unit edge normal of each edge at the maximum
// (|d_k - phi_max| <= 1e-6) and of the face normal, as in
// tritracer/backward.cu:104-189, in A-relative FP32 coordinates. Returns the
// 9 vertex gradients summed over both terms.
__device__ __forceinline__ void window_bwd(const Geom& g, float dL_dphi, float3 dL_dn3, float3 (&gv)[3]) {
  const float3 V[3] = {make_float3(0.f, 0.f, 0.f), g.e1, g.e2};
  gv[0] = gv[1] = gv[2] = make_float3(0.f, 0.f, 0.f);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    if (fabsf(g.d[k] - g.phi_max) > 1e-6f) continue;
    const float3 p1 = V[k], p2 = V[(k + 1) % 3], p3 = V[(k + 2) % 3];
    const float3 aa = p1 - p3, bb = p2 - p3, cc = p1 - p2;
    const float3 n = fcross(aa, bb);
    const float3 ne = fcross(n, cc);
    const float inv = 1.0f / flen(ne);
    const float3 Ne = ne * inv;
    // dL/dne = (I - Ne Ne^T) dL/dNe / |ne|
    const float3 dL_dNe = dL_dphi * (g.q - p1);
    const float3 v = (dL_dNe - Ne * fdot(Ne, dL_dNe)) * inv;
    // ne = ((p1-p3) x (p2-p3)) x (p1-p2); Jacobians in the form of
    // vecmath.h:2808-2859, with v^T [u]x = v x u for the skew terms
    const float3 axb = n;
    const float3 g1 = fdot(v, bb) * cc - fdot(bb, cc) * v + fcross(v, axb);
    const float3 g2 = fdot(aa, cc) * v - fdot(v, aa) * cc - fcross(v, axb);
    const float3 g3 = fdot(v, cc) * cc - fdot(cc, cc) * v;
    gv[k] = gv[k] + g1 - dL_dphi * Ne;
    gv[(k + 1) % 3] = gv[(k + 1) % 3] + g2;
    gv[(k + 2) % 3] = gv[(k + 2) % 3] + g3;
  }
  {
    // n = (p1-p3) x (p2-p3): dn/dp1 = [p3-p2]x etc.; v^T [u]x = v x u
    const float3 n = fcross(V[0] - V[2], V[1] - V[2]);
    const float inv = 1.0f / flen(n);
    const float3 Nn = n * inv;
    const float3 v = (dL_dn3 - Nn * fdot(Nn, dL_dn3)) * inv;
    gv[0] = gv[0] + fcross(v, V[2] - V[1]);
    gv[1] = gv[1] + fcross(v, V[0] - V[2]);
    gv[2] = gv[2] + fcross(v, V[1] - V[0]);
  }
}

// Exact adjoint of the window function (no reference counterpart), written
// from its definition in A-relative coordinates (P0 = 0, P1 = e1, P2 = e2,
// hit point q): edge k's unit normal en_k = s_k normalize(nc x (P_k - P_k+1))
// with nc = e1 x e2, d_k = en_k . (q - P_k), phi = max d_k,
// dist = en_0 . (I - P0), I the incenter, phi_final = phi / dist; the face
// normal normalize(nc); q = o - A + t dir with t solving q . nc = 0. Inputs:
// dL/dphi, dL/dCx sigma Cx (for dist), dL/dn and the depth term dL/dt.
__device__ __noinline__ void window_bwd_exact(const Geom& g, float3 dir, float dL_dphi, float G, float3 dL_dn3,
                                              float dL_dt_depth, float3 (&gv)[3]) {
  const float3 P[3] = {make_float3(0.f, 0.f, 0.f), g.e1, g.e2};
  const float3 nc = fcross(g.e1, g.e2);
  const float la = flen(g.e1 - g.e2), lb = flen(g.e2), lc = flen(g.e1), sum = la + lb + lc;
  const float3 inc = (lb * g.e1 + lc * g.e2) * (1.0f / sum);
  float3 en[3];
  en[0] = fnormalize(fcross(nc, -g.e1));
  float dist = fdot(en[0], inc);
  const bool flip0 = dist > 0.0f;
  if (flip0) {
    en[0] = -en[0];
    dist = -dist;
  }
  en[1] = fnormalize(fcross(nc, g.e1 - g.e2));
  en[2] = fnormalize(fcross(nc, g.e2));
  const float dL_ddist = -G / dist;
  gv[0] = gv[1] = gv[2] = make_float3(0.f, 0.f, 0.f);
  float3 g_nc = make_float3(0.f, 0.f, 0.f);
  auto edge_bwd = [&](int k, float3 g_en) {
    const float3 e = P[k] - P[(k + 1) % 3];
    const float3 ne = fcross(nc, e);
    const float inv = 1.0f / flen(ne);
    const float3 raw = ne * inv;
    const float3 gr = (k == 0 && flip0) ? -g_en : g_en;
    const float3 v = (gr - raw * fdot(raw, gr)) * inv;  // dL/d(ne)
    g_nc = g_nc + fcross(e, v);
    const float3 ge = fcross(v, nc);
    gv[k] = gv[k] + ge;
    gv[(k + 1) % 3] = gv[(k + 1) % 3] - ge;
  };
  float3 g_p = make_float3(0.f, 0.f, 0.f);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    if (fabsf(g.d[k] - g.phi_max) > 1e-6f) continue;
    edge_bwd(k, dL_dphi * (g.q - P[k]));
    g_p = g_p + dL_dphi * en[k];
    gv[k] = gv[k] - dL_dphi * en[k];
  }
  {
    edge_bwd(0, dL_ddist * inc);
    const float3 gI = dL_ddist * en[0];
    gv[0] = gv[0] - gI;
    gv[0] = gv[0] + (la / sum) * gI;
    gv[1] = gv[1] + (lb / sum) * gI;
    gv[2] = gv[2] + (lc / sum) * gI;
    const float ga = fdot(gI, P[0] - inc) / sum, gb = fdot(gI, P[1] - inc) / sum, gc = fdot(gI, P[2] - inc) / sum;
    const float3 bc = P[1] - P[2], ca = P[2] - P[0], ab = P[0] - P[1];
    gv[1] = gv[1] + (ga / la) * bc;
    gv[2] = gv[2] - (ga / la) * bc;
    gv[2] = gv[2] + (gb / lb) * ca;
    gv[0] = gv[0] - (gb / lb) * ca;
    gv[0] = gv[0] + (gc / lc) * ab;
    gv[1] = gv[1] - (gc / lc) * ab;
  }
  {
    const float inv = 1.0f / flen(nc);
    const float3 n = nc * inv;
    g_nc = g_nc + (dL_dn3 - n * fdot(n, dL_dn3)) * inv;
  }
  {
    const float dL_dt = fdot(g_p, dir) + dL_dt_depth;
    const float sc = -dL_dt / fdot(dir, nc);
    const float3 fB = fcross(g.e2, g.q), fC = fcross(g.q, g.e1);
    gv[0] = gv[0] + sc * (-nc - fB - fC);
    gv[1] = gv[1] + sc * fB;
    gv[2] = gv[2] + sc * fC;
  }
  {
    const float3 g1 = fcross(g.e2, g_nc), g2 = fcross(g_nc, g.e1);
    gv[1] = gv[1] + g1;
    gv[2] = gv[2] + g2;
    gv[0] = gv[0] - g1 - g2;
  }
}

// backward.cu:191-350: the same march, running C/N/D that include the current
// hit, dL/dalpha from the final values, scattered gradients. EXACT: the full
// chain rule of window_bwd_exact, and no gradient through a clamped alpha.
template <int MODE>
struct BwdShader {
  static constexpr bool EXACT = MODE == kShadeExact;
  static constexpr bool kStopsAtClip = false;
  const TraceParams& p;
  const ViewDesc* v;
  int pix;
  float3 o, d;
  // per-ray finals and upstream gradients, loaded for each chunk (so they do
  // not occupy registers during traversal)
  float Cf0, Cf1, Cf2, Df, Nf0, Nf1, Nf2;
  float g0, g1, g2, gD, gN0, gN1, gN2;
  float C0, C1, C2, N0, N1, N2, D, T;
  // EXACT: middepth / distortion (finals per chunk, running sum S, mid flag)
  float Wf, distf, gMid, gDist, S;
  bool mid_seen;

  __device__ explicit BwdShader(const TraceParams& params) : p(params) {}

  __device__ __forceinline__ bool begin(const ViewDesc* view, int pixel, float3 ro, float3 rd) {
    v = view;
    pix = pixel;
    o = ro;
    d = rd;
    C0 = C1 = C2 = N0 = N1 = N2 = D = 0.f;
    T = 1.0f;
    S = 0.f;
    mid_seen = false;
    return true;
  }

  __device__ __forceinline__ bool next(float3&, float3&) { return false; }

  __device__ __forceinline__ void prepare() {
    const int HW = v->H * v->W;
    Cf0 = __ldg(v->colors + pix);
    Cf1 = __ldg(v->colors + HW + pix);
    Cf2 = __ldg(v->colors + 2 * HW + pix);
    Df = __ldg(v->others + kDepthCh * HW + pix);
    Nf0 = __ldg(v->others + (kNormalCh + 0) * HW + pix);
    Nf1 = __ldg(v->others + (kNormalCh + 1) * HW + pix);
    Nf2 = __ldg(v->others + (kNormalCh + 2) * HW + pix);
    g0 = __ldg(v->dL_dpix + pix);
    g1 = __ldg(v->dL_dpix + HW + pix);
    g2 = __ldg(v->dL_dpix + 2 * HW + pix);
    gD = __ldg(v->dL_doth + kDepthCh * HW + pix);
    gN0 = __ldg(v->dL_doth + (kNormalCh + 0) * HW + pix);
    gN1 = __ldg(v->dL_doth + (kNormalCh + 1) * HW + pix);
    gN2 = __ldg(v->dL_doth + (kNormalCh + 2) * HW + pix);
    if (EXACT) {
      Wf = __ldg(v->others + kAlphaCh * HW + pix);
      distf = __ldg(v->others + kDistortionCh * HW + pix);
      gMid = __ldg(v->dL_doth + kMidDepthCh * HW + pix);
      gDist = __ldg(v->dL_doth + kDistortionCh * HW + pix);
    }
  }

  // colour rows of the current query's hit-cache entry (the forward's raw
  // colour of each blended hit), or nullptr: then the SH are evaluated
  float* crow = nullptr;
  int cstride = 0;
  __device__ __forceinline__ void set_colors(float* rows, int stride) {
    crow = rows;
    cstride = stride;
  }

  __device__ __forceinline__ bool visit(uint32_t prim, float t) { return visit(prim, t, -1); }

  __device__ __forceinline__ bool visit(uint32_t prim, float t, int slot) {
    const float4* tr = p.bvh.tri_prim + 3 * (size_t)prim;
    const float sig = __ldg(p.sigma + prim);
    const Geom g = shade_geom<MODE>(__ldg(tr), __ldg(tr + 1), __ldg(tr + 2), o, d, t, sig);
    const float opacity = __ldg(p.opac + prim);
    const float alpha = fminf(kAlphaMax, opacity * g.Cx);
    if (alpha < kAlphaMin) return false;
    const float test_T = T * (1.0f - alpha);
    if (test_T < kTMin) return true;
    const float w = alpha * T;
    float B[16];
    float3 raw;
    if (p.cols) {  // precomputed colours in place of SH
      raw = make_float3(__ldg(p.cols + 3 * prim), __ldg(p.cols + 3 * prim + 1), __ldg(p.cols + 3 * prim + 2));
    } else {
      sh_basis(unit(d), p.sh_degree, B);
      if (crow && slot >= 0)
        raw = make_float3(crow[(size_t)(3 * slot) * cstride], crow[(size_t)(3 * slot + 1) * cstride],
                          crow[(size_t)(3 * slot + 2) * cstride]);
      else
        raw = sh_raw(p.shs, p.M, (int)prim, p.sh_degree, B);
    }
    const float c0 = p.cols ? raw.x : fmaxf(raw.x, 0.f), c1 = p.cols ? raw.y : fmaxf(raw.y, 0.f),
                c2 = p.cols ? raw.z : fmaxf(raw.z, 0.f);
    C0 += c0 * w;
    C1 += c1 * w;
    C2 += c2 * w;
    N0 += g.n.x * w;
    N1 += g.n.y * w;
    N2 += g.n.z * w;
    D += w * g.t;
    // backward.cu:296-312; C/N/D already include this hit
    const float inv1a = 1.0f / (1.0f - alpha);
    float dL_dalpha = g0 * (T * c0 - (Cf0 - C0) * inv1a) + g1 * (T * c1 - (Cf1 - C1) * inv1a) +
                      g2 * (T * c2 - (Cf2 - C2) * inv1a);
    dL_dalpha += gD * (T * g.t - (Df - D) * inv1a);
    dL_dalpha += gN0 * (T * g.n.x - (Nf0 - N0) * inv1a) + gN1 * (T * g.n.y - (Nf1 - N1) * inv1a) +
                 gN2 * (T * g.n.z - (Nf2 - N2) * inv1a);
    float dL_dt = gD * w;
    if (EXACT) {
      // distortion: dD/dalpha_k = T_k E_k - (2 D_f - S_k) / (1 - alpha_k),
      // E_k = t^2 W_f - 2 t B_f + C_f, C_f = (D_f + B_f^2) / W_f; dD/dt_k = 2 w (t W_f - B_f)
      const float Cf = Wf > 0.f ? (distf + Df * Df) / Wf : 0.f;
      const float E = g.t * g.t * Wf - 2.0f * g.t * Df + Cf;
      S += w * E;
      dL_dalpha += gDist * (T * E - (2.0f * distf - S) * inv1a);
      dL_dt += gDist * 2.0f * w * (g.t * Wf - Df);
      if (!mid_seen && test_T <= 0.5f) {
        mid_seen = true;
        dL_dt += gMid;
      }
    }
    const bool live = !EXACT || opacity * g.Cx < kAlphaMax;
    const float dL_dC = live ? opacity * dL_dalpha : 0.0f;
    if (live) red_add(p.d_opac + prim, dL_dalpha * g.Cx);
    if (g.phi_final > 0.0f) red_add(p.d_sigma + prim, dL_dC * g.Cx * logf(g.phi_final));
    const float dL_dphi = sig / g.phi_max * dL_dC * g.Cx;
    float3 gv[3];
    if (EXACT)
      window_bwd_exact(g, d, dL_dphi, dL_dC * sig * g.Cx, make_float3(gN0 * w, gN1 * w, gN2 * w), dL_dt, gv);
    else
      window_bwd(g, dL_dphi, make_float3(gN0 * w, gN1 * w, gN2 * w), gv);
    float* dt = p.d_tri + 3 * (size_t)__ldg(p.cumsum + prim);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      red_add(dt + 3 * k + 0, gv[k].x);
      red_add(dt + 3 * k + 1, gv[k].y);
      red_add(dt + 3 * k + 2, gv[k].z);
    }
    if (p.cols) {
      red_add(p.d_cols + 3 * prim + 0, g0 * w);
      red_add(p.d_cols + 3 * prim + 1, g1 * w);
      red_add(p.d_cols + 3 * prim + 2, g2 * w);
      T = test_T;
      return false;
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
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        if (k < n) {
          red_add(dsh + 3 * k + 0, B[k] * e0);
          red_add(dsh + 3 * k + 1, B[k] * e1);
          red_add(dsh + 3 * k + 2, B[k] * e2);
        }
      }
    }
    T = test_T;
    return false;
  }

  __device__ __forceinline__ void end() {}
};

// The adjoint. REPLAY: the replay-only build (packet configurations), which
// needs a complete hit cache. Given a cache, the host launches the two builds
// back to back (p.bwd_pair): the replay-only one works when the cache is
// complete, the traversing one otherwise, and the other returns at once;
// the choice is read on the device, so nothing synchronises.
template <int CFG, int MODE, bool REPLAY = false>
__global__ void __launch_bounds__(kTraceThreads, REPLAY ? kReplayBlocks : kMinBlocks) k_backward(const __grid_constant__ TraceParams p) {
  if (p.bwd_pair && cache_complete<TraversalCfg<CFG>::K>(p) != REPLAY) return;
  Counters cnt;
  BwdShader<MODE> sh(p);
  run<CFG, BwdShader<MODE>, REPLAY>(p, sh, cnt);
  const unsigned s = __reduce_add_sync(0xFFFFFFFFu, cnt.replays);
  if ((threadIdx.x & 31) == 0 && s != 0u) atomicAdd(p.stats + kStatReplays, (unsigned long long)s);
}

// ---------------------------------------------------------------- secondary rays
// Secondary-ray passes over a device ray queue (no reference counterpart; the
// reference bends rays only at one analytic sphere). Per pixel a tree of
// rays: the first blended hit of a ray of depth < max_depth on a triangle of
// material 1 spawns a reflected and (unless totally reflected) a refracted
// ray from the exact hit point, and that hit's colour is
// F L(reflected) + (1 - F) L(refracted) instead of its SH colour; rays that
// leave the scene see a lat-long environment map in place of bg. One launch
// per level traces the level's rays from its queue and appends their
// children to the next level's queue (atomic slot counter); resolve launches
// then add each child's radiance to its parent, deepest level first, and
// write the pixel colours. The adjoint traces every ray of every level in one
// launch with upstream gradient tau dL/dpixel, taking the spawning hit's
// colour from the children's resolved radiance.

// Per-lane persistent driver over `total` queue items (item order = record
// order); lanes refill as their rays finish.
template <int SD, class Shader>
__device__ __forceinline__ void drive_items(const TraceParams& p, const Smem& sm, Shader& sh, Counters& cnt,
                                            int total) {
  constexpr int K = kChunk;
  const unsigned full = 0xFFFFFFFFu;
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  bool have = false, exhausted = false;
  Cursor cur = first_cursor(p.tmin_inclusive);
  float3 o = make_float3(0.f, 0.f, 0.f), d = o;
  uint32_t* link = nullptr;  // forward: where the entry of the ray's next query gets linked
  uint32_t next = kNoEntry;  // adjoint: entry of the ray's next query
  const bool replay = cache_replays<K>(p);
  for (;;) {
    const unsigned need = __ballot_sync(full, !have && !exhausted);
    if (need) {
      const int leader = __ffs(need) - 1;
      int base = 0;
      if (lane == leader) base = atomicAdd(p.work, __popc(need));
      base = __shfl_sync(full, base, leader);
      if (!have && !exhausted) {
        const int item = base + __popc(need & lt);
        if (item >= total) {
          exhausted = true;
        } else {
          sh.begin_item(item, o, d);
          cur = first_cursor(p.tmin_inclusive);
          have = true;
        }
      }
    }
    if (__ballot_sync(full, have) == 0) {
      if (__all_sync(full, exhausted)) break;
      continue;
    }
    float t_drop = INFINITY;
    if (have) {
      // Hit cache: a level-0 ray (record = pixel) keeps its first query in
      // the main part; a deeper ray starts its chain in the pool, linked from
      // its queue record
      const bool first = cur.chunks == 0;
      const bool main_part = first && sh.ridx < p.cache_rays;
      uint32_t* rec_link = &p.sec.rec[sh.ridx].cache_link;
      if (replay && first && !main_part) next = __ldcg(rec_link);
      if (replay && (main_part || cache_has<K>(p, next, cur.key_min))) {
        if (p.cache_mode == kCacheFill) link = cache_link_of<K>(p, main_part, sh.ridx, next);
        t_drop = cache_get<K>(p, main_part, sh.ridx, next, sm, next);
        ++cnt.replays;
      } else {
        next = kNoEntry;
        const RayW r = make_ray(o, d);
        query<SD>(p.bvh, r, cur.key_min, cur.t_hi, sm.keys, sm.stride, sm.st, t_drop, p.status, cnt, p.count_work);
        if (p.cache_mode == kCacheWrite || p.cache_mode == kCacheFill) {
          if (main_part) {
            link = cache_put_first<K>(p, sh.ridx, sm, t_drop);
          } else {
            if (first) link = rec_link;
            if (link) {
              const uint32_t e = atomicAdd(&cache_header_ptr(p)->pool_used, 1u);
              link = e < p.cache_pool_cap ? cache_put_more<K>(p, e, cur.key_min, sm, t_drop, link) : nullptr;
            }
          }
        }
      }
    }
    __syncwarp();
    if (have) {
      bool done = consume_chunk<K>(sm, t_drop, cur, p.tmin_inclusive, p.status, sh, cnt);
      if (!done && ++cur.chunks >= kMaxChunks) {
        atomicOr(p.status, kStatusTimeout);
        done = true;
      }
      // the collecting pass stores at most collect_queries queries a ray
      if (Shader::kStopsAtClip && p.collect_queries > 0 && cur.chunks >= p.collect_queries) done = true;
      if (done) {
        sh.end();
        have = false;
      }
    }
  }
}

// FP64 with explicit round-to-nearest operations (no contraction), in the
// oracle's operation order, so both spawn the same FP32 rays.
namespace sd {
struct V {
  double x, y, z;
};
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ V vsub(V a, V b) { return {sub(a.x, b.x), sub(a.y, b.y), sub(a.z, b.z)}; }
__device__ __forceinline__ V vadd(V a, V b) { return {add(a.x, b.x), add(a.y, b.y), add(a.z, b.z)}; }
__device__ __forceinline__ V vscale(V a, double s) { return {mul(a.x, s), mul(a.y, s), mul(a.z, s)}; }
__device__ __forceinline__ double dot(V a, V b) { return add(add(mul(a.x, b.x), mul(a.y, b.y)), mul(a.z, b.z)); }
__device__ __forceinline__ V cross(V a, V b) {
  return {sub(mul(a.y, b.z), mul(a.z, b.y)), sub(mul(a.z, b.x), mul(a.x, b.z)), sub(mul(a.x, b.y), mul(a.y, b.x))};
}
__device__ __forceinline__ V from(float4 v) { return {(double)v.x, (double)v.y, (double)v.z}; }
__device__ __forceinline__ V from(float3 v) { return {(double)v.x, (double)v.y, (double)v.z}; }
__device__ __forceinline__ float3 to_f(V v) {
  return make_float3(__double2float_rn(v.x), __double2float_rn(v.y), __double2float_rn(v.z));
}
}  // namespace sd

struct SpawnDev {
  float3 o, r, t;
  bool refracts;
  float F;
};

// Reflected / refracted rays at the hit of (o, d) on the triangle (a, b, c)
// with index of refraction ior: Schlick's Fresnel term, the exact hit point
// of an FP64 plane solve.
__device__ __noinline__ SpawnDev spawn_rays(float4 a4, float4 b4, float4 c4, float3 of, float3 df, float ior_f) {
  using namespace sd;
  const V A = from(a4), B = from(b4), C = from(c4), o = from(of), d = from(df);
  const V nc = cross(vsub(B, A), vsub(C, A));
  const double te = __ddiv_rn(dot(vsub(A, o), nc), dot(d, nc));
  const V x = vadd(o, vscale(d, te));
  const V n = vscale(nc, __ddiv_rn(1.0, __dsqrt_rn(dot(nc, nc))));
  const V du = vscale(d, __ddiv_rn(1.0, __dsqrt_rn(dot(d, d))));
  const double ior = (double)ior_f;
  const double cosi = dot(du, n);
  const bool entering = cosi < 0.0;
  const V nf = entering ? n : V{-n.x, -n.y, -n.z};
  const double c = entering ? -cosi : cosi;
  const double ei = entering ? 1.0 : ior, et = entering ? ior : 1.0;
  const double eta = __ddiv_rn(ei, et);
  const double q = __ddiv_rn(sub(ei, et), add(ei, et));
  const double r0 = mul(q, q);
  const double k = sub(1.0, mul(mul(eta, eta), sub(1.0, mul(c, c))));
  SpawnDev sp;
  sp.o = to_f(x);
  sp.r = to_f(vadd(du, vscale(nf, mul(2.0, c))));
  sp.refracts = k >= 0.0;
  double F = 1.0;
  V t = du;
  if (sp.refracts) {
    const double m = sub(1.0, c);
    const double m2 = mul(m, m);
    F = add(r0, mul(sub(1.0, r0), mul(mul(m2, m2), m)));
    t = vadd(vscale(du, eta), vscale(nf, sub(mul(eta, c), __dsqrt_rn(k))));
  }
  sp.t = to_f(t);
  sp.F = __double2float_rn(F);
  return sp;
}

// Lat-long lookup: longitude atan2(d.z, d.x) over the columns (wrapping),
// colatitude acos(d.y) over the rows (clamped), bilinear between texel centres.
// env_texels gives the four texels (word offsets of their RGB) and the
// bilinear fractions; the adjoint scatters into the same four.
struct EnvTexels {
  size_t t00, t01, t10, t11;
  float ax, ay;
};

__device__ __forceinline__ EnvTexels env_texels(const SecParams& s, float3 d) {
  const float kPi = 3.14159265358979f;
  const float len = sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
  const float u = atan2f(d.z, d.x) * (0.5f / kPi) + 0.5f;
  const float v = acosf(fminf(1.f, fmaxf(-1.f, d.y / len))) * (1.0f / kPi);
  float fx = u * (float)s.env_w - 0.5f, fy = v * (float)s.env_h - 0.5f;
  if (!(fabsf(fx) <= (float)s.env_w)) fx = 0.f;  // NaN direction: any texel, never out of bounds
  if (!(fabsf(fy) <= (float)s.env_h)) fy = 0.f;
  const float x0f = floorf(fx), y0f = floorf(fy);
  const int W = s.env_w, H = s.env_h;
  const int x0 = (((int)x0f % W) + W) % W, x1 = (x0 + 1) % W;
  const int y0 = max(0, min(H - 1, (int)y0f)), y1 = max(0, min(H - 1, (int)y0f + 1));
  EnvTexels t;
  t.ax = fx - x0f;
  t.ay = fy - y0f;
  t.t00 = ((size_t)y0 * W + x0) * 3;
  t.t01 = ((size_t)y0 * W + x1) * 3;
  t.t10 = ((size_t)y1 * W + x0) * 3;
  t.t11 = ((size_t)y1 * W + x1) * 3;
  return t;
}

__device__ __forceinline__ float3 env_lookup(const SecParams& s, float3 d) {
  const EnvTexels t = env_texels(s, d);
  const float ax = t.ax, ay = t.ay;
  const float* e = s.env;
  float out[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float t00 = __ldg(e + t.t00 + c), t01 = __ldg(e + t.t01 + c);
    const float t10 = __ldg(e + t.t10 + c), t11 = __ldg(e + t.t11 + c);
    out[c] = (1.f - ay) * ((1.f - ax) * t00 + ax * t01) + ay * ((1.f - ax) * t10 + ax * t11);
  }
  return make_float3(out[0], out[1], out[2]);
}

// Adjoint of T env(d) in a ray's radiance: dL/d(texel) += g T (bilinear weight).
__device__ __forceinline__ void env_lookup_bwd(const SecParams& s, float3 d, float T, float g0, float g1, float g2) {
  const EnvTexels t = env_texels(s, d);
  const float ax = t.ax, ay = t.ay;
  const float wt[4] = {(1.f - ay) * (1.f - ax), (1.f - ay) * ax, ay * (1.f - ax), ay * ax};
  const size_t at[4] = {t.t00, t.t01, t.t10, t.t11};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float f = T * wt[k];
    red_add(s.d_env + at[k] + 0, g0 * f);
    red_add(s.d_env + at[k] + 1, g1 * f);
    red_add(s.d_env + at[k] + 2, g2 * f);
  }
}

// d F / d ior of Schlick's reflected share F at a refracting hit:
// F = r0 + (1 - r0) (1 - cos)^5 with r0 = ((ior - 1) / (ior + 1))^2 (either
// side of the interface), so dF/dior = dr0/dior (1 - F) / (1 - r0) and
// dr0/dior = 4 (ior - 1) / (ior + 1)^3.
__device__ __forceinline__ float fresnel_dF_dior(float n, float F) {
  const float q = (n - 1.f) / (n + 1.f);
  const float n1 = n + 1.f;
  return 4.f * (n - 1.f) / (n1 * n1 * n1) * (1.f - F) / (1.f - q * q);
}

// The rays of one level: trace, composite, spawn children into the next level.
struct SecShader {
  static constexpr bool kStopsAtClip = false;
  const TraceParams& p;
  const ViewDesc* v;
  int ridx, pix, level;
  float3 o, d;
  float C0, C1, C2, N0, N1, N2, T, tau;
  bool spawned;
  unsigned n_rays = 0, n_eval = 0, n_blend = 0;

  __device__ explicit SecShader(const TraceParams& params) : p(params), v(&params.views[0]), level(params.sec.level) {}

  __device__ __forceinline__ void begin_item(int i, float3& ro, float3& rd) {
    const SecParams& s = p.sec;
    ridx = s.base[level] + (level > 0 && s.order ? (int)__ldg(s.order + i) : i);
    SecRecord* r = s.rec + ridx;
    if (level == 0) {
      pix = i;
      ro = make_float3(v->ray_o[3 * pix], v->ray_o[3 * pix + 1], v->ray_o[3 * pix + 2]);
      rd = make_float3(v->ray_d[3 * pix], v->ray_d[3 * pix + 1], v->ray_d[3 * pix + 2]);
      tau = 1.0f;
      r->pixel = pix;
      r->tau = 1.0f;
    } else {
      ro = make_float3(r->o[0], r->o[1], r->o[2]);
      rd = make_float3(r->d[0], r->d[1], r->d[2]);
      pix = r->pixel;
      tau = r->tau;
    }
    r->child_r = r->child_t = -1;
    r->F = r->w = 0.f;
    o = ro;
    d = rd;
    C0 = C1 = C2 = N0 = N1 = N2 = 0.f;
    T = 1.0f;
    spawned = false;
    ++n_rays;
  }

  // The packet driver's entry (level 0): the primary ray of `pixel`.
  __device__ __forceinline__ bool begin(const ViewDesc*, int pixel, float3, float3) {
    float3 ro, rd;
    begin_item(pixel, ro, rd);
    return true;
  }

  __device__ __forceinline__ void prepare() {}

  __device__ __forceinline__ int push_child(float3 co, float3 cd, float ctau) {
    const SecParams& s = p.sec;
    const int slot = atomicAdd(s.count + level + 1, 1);
    if (slot >= s.cap[level + 1]) {
      atomicOr(p.status, kStatusStack);
      return -1;
    }
    SecRecord* c = s.rec + s.base[level + 1] + slot;
    c->o[0] = co.x;
    c->o[1] = co.y;
    c->o[2] = co.z;
    c->d[0] = cd.x;
    c->d[1] = cd.y;
    c->d[2] = cd.z;
    c->pixel = pix;
    c->tau = ctau;
    c->cache_link = kNoEntry;
    return slot;
  }

  __device__ __forceinline__ bool visit(uint32_t prim, float) {
    const float4* tr = p.bvh.tri_prim + 3 * (size_t)prim;
    const float4 a = __ldg(tr), b = __ldg(tr + 1), c = __ldg(tr + 2);
    const Geom g = window_fn(a, b, c, o, d, __ldg(p.sigma + prim));
    ++n_eval;
    const float alpha = fminf(kAlphaMax, __ldg(p.opac + prim) * g.Cx);
    if (alpha < kAlphaMin) return false;
    const float test_T = T * (1.0f - alpha);
    if (test_T < kTMin) return true;
    ++n_blend;
    const float w = alpha * T;
    if (level == 0) {
      p.density[prim] = 1.0f;
      compute_scaling(p.scaling, p.verts, p.cumsum, p.num_points, (int)prim, o);
      atomicMax(reinterpret_cast<int*>(p.max_blending) + prim, __float_as_int(w));
      N0 += g.n.x * w;
      N1 += g.n.y * w;
      N2 += g.n.z * w;
    }
    const SecParams& s = p.sec;
    if (!spawned && level < s.max_depth && __ldg(s.material + prim) == 1) {
      // the hit's colour comes from its children at the resolve
      spawned = true;
      const SpawnDev sp = spawn_rays(a, b, c, o, d, __ldg(s.ior + prim));
      SecRecord* r = s.rec + ridx;
      r->F = sp.F;
      r->w = w;
      r->child_r = push_child(sp.o, sp.r, tau * w * sp.F);
      if (sp.refracts) r->child_t = push_child(sp.o, sp.t, tau * w * (1.0f - sp.F));
    } else {
      float B[16];
      sh_basis(unit(d), p.sh_degree, B);
      const float3 col = sh_raw(p.shs, p.M, (int)prim, p.sh_degree, B);
      C0 += fmaxf(col.x, 0.f) * w;
      C1 += fmaxf(col.y, 0.f) * w;
      C2 += fmaxf(col.z, 0.f) * w;
    }
    T = test_T;
    return false;
  }

  __device__ __forceinline__ void end() {
    const float3 e = env_lookup(p.sec, d);
    SecRecord* r = p.sec.rec + ridx;
    r->L[0] = C0 + T * e.x;
    r->L[1] = C1 + T * e.y;
    r->L[2] = C2 + T * e.z;
    if (level == 0) {
      const int HW = v->H * v->W;
      v->out_others[kDepthCh * HW + pix] = 0.0f;
      v->out_others[kAlphaCh * HW + pix] = 1.0f - T;
      v->out_others[(kNormalCh + 0) * HW + pix] = N0;
      v->out_others[(kNormalCh + 1) * HW + pix] = N1;
      v->out_others[(kNormalCh + 2) * HW + pix] = N2;
      v->out_others[kMidDepthCh * HW + pix] = 0.0f;
      v->out_others[kDistortionCh * HW + pix] = 0.0f;
    }
  }
};

__device__ __forceinline__ int sec_level_size(const TraceParams& p, int level) {
  return level == 0 ? p.views[0].H * p.views[0].W : min(__ldcg(p.sec.count + level), p.sec.cap[level]);
}

// Level 0: the primary rays are camera-coherent, so they are traced as warp
// packets of 8x4 pixels (with the hit cache's 16 hits per query), in a kernel
// of their own (the lane driver's registers would spill in the same kernel).
__global__ void __launch_bounds__(kTraceThreads, kMinBlocks) k_sec_primary(const __grid_constant__ TraceParams p) {
  cache_header<kChunk>(p);  // the deeper levels append to the same cache
  Counters cnt;
  SecShader sh(p);
  unsigned char* rest;
  const Smem sm = packet_smem<kChunk>(rest);
  drive_packets<kChunk>(p, sm, warp_stack(rest), sh, cnt);
  cnt.queries += cnt.replays;  // replayed from the traversal pass (split schedule): used by the march all the same
  cnt.replays = 0;
  add_stats(p.stats, sh.n_rays, sh.n_eval, sh.n_blend, cnt);
}

// Levels >= 1: spawned rays, incoherent: one ray per lane, with a
// kSecStack-entry stack in shared memory per lane (continued in local
// memory) and kSecBlocks blocks per SM.
#ifndef TT_SEC_STACK
#define TT_SEC_STACK 32
#endif
#ifndef TT_SEC_BLOCKS
#define TT_SEC_BLOCKS 4
#endif
constexpr int kSecStack = TT_SEC_STACK, kSecBlocks = TT_SEC_BLOCKS;
constexpr size_t sec_trace_smem() { return (size_t)kTraceThreads * (kSecStack * 8 + kChunk * 8); }

__global__ void __launch_bounds__(kTraceThreads, kSecBlocks) k_sec_trace(const __grid_constant__ TraceParams p) {
  Counters cnt;
  SecShader sh(p);
  drive_items<kSecStack>(p, thread_smem<kSecStack>(), sh, cnt, sec_level_size(p, p.sec.level));
  cnt.queries += cnt.replays;  // replayed from the traversal pass (split schedule): used by the march all the same
  cnt.replays = 0;
  add_stats(p.stats, sh.n_rays, sh.n_eval, sh.n_blend, cnt);
}

// Traversal pass of a spawned level (split schedule): the level's rays, in
// the same order, with a shader that shades and spawns nothing, storing every
// query in the ray tree's hit cache (the chain starts at the ray's record);
// k_sec_trace then replays them in fill mode. Like k_collect for primary
// rays: without the shading and spawning code the pass needs fewer
// registers, and with a shorter shared-memory stack per lane (continued in
// local memory) more blocks fit an SM.
#ifndef TT_SEC_COLLECT_STACK
#define TT_SEC_COLLECT_STACK 16
#endif
#ifndef TT_SEC_COLLECT_BLOCKS
#define TT_SEC_COLLECT_BLOCKS 6
#endif
constexpr int kSecCollectStack = TT_SEC_COLLECT_STACK, kSecCollectBlocks = TT_SEC_COLLECT_BLOCKS;
constexpr size_t sec_collect_smem() { return (size_t)kTraceThreads * (kSecCollectStack * 8 + kChunk * 8); }

struct SecMarchShader {
  static constexpr bool kStopsAtClip = true;
  const TraceParams& p;
  int ridx = 0;
  __device__ explicit SecMarchShader(const TraceParams& params) : p(params) {}
  __device__ __forceinline__ void begin_item(int i, float3& ro, float3& rd) {
    const SecParams& s = p.sec;
    ridx = s.base[s.level] + (s.order ? (int)__ldg(s.order + i) : i);
    const SecRecord* r = s.rec + ridx;
    ro = make_float3(r->o[0], r->o[1], r->o[2]);
    rd = make_float3(r->d[0], r->d[1], r->d[2]);
  }
  __device__ __forceinline__ void prepare() {}
  __device__ __forceinline__ bool visit(uint32_t, float) { return false; }
  __device__ __forceinline__ void end() {}
};

__global__ void __launch_bounds__(kTraceThreads, kSecCollectBlocks) k_sec_collect(const __grid_constant__ TraceParams p) {
  Counters cnt;
  SecMarchShader sh(p);
  drive_items<kSecCollectStack>(p, thread_smem<kSecCollectStack>(), sh, cnt, sec_level_size(p, p.sec.level));
  cnt.queries = 0;  // counted by the shading pass (k_sec_trace), like k_collect
  add_stats(p.stats, 0u, 0u, 0u, cnt);
}

// Sort keys of the spawned rays of level p.sec.level: the direction in 16 x
// 16 octahedral bins (8 bits) over the Morton code of the origin, 7 bits an
// axis, within the root box of the BVH (21 bits); slots past the level's
// count get 0xFFFFFFFF and sort after every ray. On C3 this order traces the
// spawned levels in 29.9 ms a step against 30.7 with the direction octant
// over a 27-bit Morton code and 32.5 with the origin first; finer direction
// bins (1024, 4096) or coarser origins were slower.
__device__ __forceinline__ uint32_t spread3(uint32_t v) {  // 9 bits -> every third of 27
  v &= 0x1FFu;
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

__global__ void k_sec_sort_keys(const __grid_constant__ TraceParams p, uint32_t* __restrict__ keys,
                                uint32_t* __restrict__ vals) {
  const SecParams& s = p.sec;
  const int level = s.level, cap = s.cap[level];
  const int n = min(__ldcg(s.count + level), cap);
  // the root's box: the union of its 8 child boxes (empty slots are inverted)
  float lo[3] = {0.f, 0.f, 0.f}, ext[3] = {1.f, 1.f, 1.f};
  if (p.bvh.has_root && p.bvh.P >= 2) {
    const float* nd = reinterpret_cast<const float*>(p.bvh.nodes);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      float l = INFINITY, h = -INFINITY;
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        l = fminf(l, __ldg(nd + 16 * a + c));
        h = fmaxf(h, __ldg(nd + 16 * a + 8 + c));
      }
      if (l < h) {
        lo[a] = l;
        ext[a] = h - l;
      }
    }
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += gridDim.x * blockDim.x) {
    uint32_t key = 0xFFFFFFFFu;
    if (i < n) {
      const SecRecord& r = s.rec[s.base[level] + i];
      uint32_t q[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) q[a] = (uint32_t)fminf(fmaxf((r.o[a] - lo[a]) / ext[a] * 512.f, 0.f), 511.f);
      // octahedral map of the direction onto [-1, 1]^2 (lower hemisphere folded out)
      const float ad = fabsf(r.d[0]) + fabsf(r.d[1]) + fabsf(r.d[2]);
      float ux = ad > 0.f ? r.d[0] / ad : 0.f, uy = ad > 0.f ? r.d[1] / ad : 0.f;
      if (r.d[2] < 0.f) {
        const float fx = (1.f - fabsf(uy)) * (ux >= 0.f ? 1.f : -1.f);
        const float fy = (1.f - fabsf(ux)) * (uy >= 0.f ? 1.f : -1.f);
        ux = fx;
        uy = fy;
      }
      const uint32_t bx = (uint32_t)fminf(fmaxf((ux * 0.5f + 0.5f) * 16.f, 0.f), 15.f);
      const uint32_t by = (uint32_t)fminf(fmaxf((uy * 0.5f + 0.5f) * 16.f, 0.f), 15.f);
      key = (((bx << 4) | by) << 21) | (spread3(q[0] >> 2) << 2) | (spread3(q[1] >> 2) << 1) | spread3(q[2] >> 2);
    }
    keys[i] = key;
    vals[i] = (uint32_t)i;
  }
}

// Adds each record's children's radiance to it (their level is complete) and,
// for level 0, writes the pixel colours.
__global__ void k_sec_resolve(const __grid_constant__ TraceParams p) {
  const SecParams& s = p.sec;
  const int level = s.level;
  const int n = sec_level_size(p, level);
  const ViewDesc& v = p.views[0];
  const int HW = v.H * v.W;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    SecRecord* r = s.rec + s.base[level] + i;
    float L0 = r->L[0], L1 = r->L[1], L2 = r->L[2];
    if (r->child_r >= 0 || r->child_t >= 0) {
      float lr[3] = {0.f, 0.f, 0.f}, lt[3] = {0.f, 0.f, 0.f};
      if (r->child_r >= 0) {
        const SecRecord* c = s.rec + s.base[level + 1] + r->child_r;
        lr[0] = c->L[0];
        lr[1] = c->L[1];
        lr[2] = c->L[2];
      }
      if (r->child_t >= 0) {
        const SecRecord* c = s.rec + s.base[level + 1] + r->child_t;
        lt[0] = c->L[0];
        lt[1] = c->L[1];
        lt[2] = c->L[2];
      }
      const float F = r->F, w = r->w;
      L0 += w * (F * lr[0] + (1.0f - F) * lt[0]);
      L1 += w * (F * lr[1] + (1.0f - F) * lt[1]);
      L2 += w * (F * lr[2] + (1.0f - F) * lt[2]);
      r->L[0] = L0;
      r->L[1] = L1;
      r->L[2] = L2;
    }
    if (level == 0) {
      v.out_color[i] = L0;
      v.out_color[HW + i] = L1;
      v.out_color[2 * HW + i] = L2;
    }
  }
}

// Adjoint of every ray of every level (backward.cu's per-hit formulas with
// upstream gradient tau dL/dpixel; the spawning hit's colour is the
// children's resolved radiance and it has no SH gradient).
struct SecBwdShader {
  static constexpr bool kStopsAtClip = false;
  const TraceParams& p;
  const ViewDesc* v;
  int ridx, pix, level;
  float3 o, d;
  float Cf0, Cf1, Cf2, Df, Nf0, Nf1, Nf2;
  float g0, g1, g2, gD, gN0, gN1, gN2;
  float C0, C1, C2, N0, N1, N2, D, T;
  bool spawned;

  __device__ explicit SecBwdShader(const TraceParams& params) : p(params), v(&params.views[0]) {}

  __device__ __forceinline__ void begin_item(int item, float3& ro, float3& rd) {
    const SecParams& s = p.sec;
    level = 0;
    int i = item;
    while (level < s.max_depth && i >= sec_level_size(p, level)) {
      i -= sec_level_size(p, level);
      ++level;
    }
    // spawned levels in the order the forward traced them (neighbouring
    // items then gather the same triangles)
    const uint32_t* ord = level > 0 ? s.bwd_order[level] : nullptr;
    ridx = s.base[level] + (ord ? (int)__ldg(ord + i) : i);
    const SecRecord* r = s.rec + ridx;
    const int HW = v->H * v->W;
    float tau;
    if (level == 0) {
      pix = i;
      ro = make_float3(v->ray_o[3 * pix], v->ray_o[3 * pix + 1], v->ray_o[3 * pix + 2]);
      rd = make_float3(v->ray_d[3 * pix], v->ray_d[3 * pix + 1], v->ray_d[3 * pix + 2]);
      tau = 1.0f;
      Df = __ldg(v->others + kDepthCh * HW + pix);
      Nf0 = __ldg(v->others + (kNormalCh + 0) * HW + pix);
      Nf1 = __ldg(v->others + (kNormalCh + 1) * HW + pix);
      Nf2 = __ldg(v->others + (kNormalCh + 2) * HW + pix);
      gD = __ldg(v->dL_doth + kDepthCh * HW + pix);
      gN0 = __ldg(v->dL_doth + (kNormalCh + 0) * HW + pix);
      gN1 = __ldg(v->dL_doth + (kNormalCh + 1) * HW + pix);
      gN2 = __ldg(v->dL_doth + (kNormalCh + 2) * HW + pix);
    } else {
      ro = make_float3(r->o[0], r->o[1], r->o[2]);
      rd = make_float3(r->d[0], r->d[1], r->d[2]);
      pix = r->pixel;
      tau = r->tau;
      Df = Nf0 = Nf1 = Nf2 = gD = gN0 = gN1 = gN2 = 0.f;
    }
    Cf0 = r->L[0];
    Cf1 = r->L[1];
    Cf2 = r->L[2];
    g0 = tau * __ldg(v->dL_dpix + pix);
    g1 = tau * __ldg(v->dL_dpix + HW + pix);
    g2 = tau * __ldg(v->dL_dpix + 2 * HW + pix);
    o = ro;
    d = rd;
    C0 = C1 = C2 = N0 = N1 = N2 = D = 0.f;
    T = 1.0f;
    spawned = false;
  }

  __device__ __forceinline__ void prepare() {}

  __device__ __forceinline__ bool visit(uint32_t prim, float) {
    const float4* tr = p.bvh.tri_prim + 3 * (size_t)prim;
    const float sig = __ldg(p.sigma + prim);
    const Geom g = window_fn(__ldg(tr), __ldg(tr + 1), __ldg(tr + 2), o, d, sig);
    const float opacity = __ldg(p.opac + prim);
    const float alpha = fminf(kAlphaMax, opacity * g.Cx);
    if (alpha < kAlphaMin) return false;
    const float test_T = T * (1.0f - alpha);
    if (test_T < kTMin) return true;
    const float w = alpha * T;
    const SecParams& s = p.sec;
    float c0, c1, c2;
    float raw0 = 0.f, raw1 = 0.f, raw2 = 0.f;
    float B[16];
    const bool spawn = !spawned && level < s.max_depth && __ldg(s.material + prim) == 1;
    if (spawn) {
      spawned = true;
      const SecRecord* r = s.rec + ridx;
      const float F = r->F;
      float lr[3] = {0.f, 0.f, 0.f}, lt[3] = {0.f, 0.f, 0.f};
      if (r->child_r >= 0) {
        const SecRecord* c = s.rec + s.base[level + 1] + r->child_r;
        lr[0] = c->L[0];
        lr[1] = c->L[1];
        lr[2] = c->L[2];
      }
      if (r->child_t >= 0) {
        const SecRecord* c = s.rec + s.base[level + 1] + r->child_t;
        lt[0] = c->L[0];
        lt[1] = c->L[1];
        lt[2] = c->L[2];
      }
      c0 = F * lr[0] + (1.0f - F) * lt[0];
      c1 = F * lr[1] + (1.0f - F) * lt[1];
      c2 = F * lr[2] + (1.0f - F) * lt[2];
      if (s.d_ior && r->child_t >= 0) {  // a refracting hit: the colour depends on ior through F
        const float dL_dF = w * (g0 * (lr[0] - lt[0]) + g1 * (lr[1] - lt[1]) + g2 * (lr[2] - lt[2]));
        red_add(s.d_ior + prim, dL_dF * fresnel_dF_dior(__ldg(s.ior + prim), F));
      }
    } else {
      sh_basis(unit(d), p.sh_degree, B);
      const float3 raw = sh_raw(p.shs, p.M, (int)prim, p.sh_degree, B);
      raw0 = raw.x;
      raw1 = raw.y;
      raw2 = raw.z;
      c0 = fmaxf(raw.x, 0.f);
      c1 = fmaxf(raw.y, 0.f);
      c2 = fmaxf(raw.z, 0.f);
    }
    C0 += c0 * w;
    C1 += c1 * w;
    C2 += c2 * w;
    N0 += g.n.x * w;
    N1 += g.n.y * w;
    N2 += g.n.z * w;
    D += w * g.t;
    const float inv1a = 1.0f / (1.0f - alpha);
    float dL_dalpha = g0 * (T * c0 - (Cf0 - C0) * inv1a) + g1 * (T * c1 - (Cf1 - C1) * inv1a) +
                      g2 * (T * c2 - (Cf2 - C2) * inv1a);
    // The exact adjoint differentiates the outputs the passes compute: the
    // depth channel is 0 there (as in the reference), so it has no gradient,
    // and a clamped alpha passes none; the reference-style adjoint keeps
    // backward.cu's depth term and differentiates through the clamp.
    const bool exact = p.mode == kShadeExact;
    if (!exact) dL_dalpha += gD * (T * g.t - (Df - D) * inv1a);
    dL_dalpha += gN0 * (T * g.n.x - (Nf0 - N0) * inv1a) + gN1 * (T * g.n.y - (Nf1 - N1) * inv1a) +
                 gN2 * (T * g.n.z - (Nf2 - N2) * inv1a);
    const bool live = !exact || opacity * g.Cx < kAlphaMax;
    const float dL_dC = live ? opacity * dL_dalpha : 0.0f;
    if (live) red_add(p.d_opac + prim, dL_dalpha * g.Cx);
    if (g.phi_final > 0.0f) red_add(p.d_sigma + prim, dL_dC * g.Cx * logf(g.phi_final));
    const float dL_dphi = sig / g.phi_max * dL_dC * g.Cx;
    float3 gv[3];
    if (exact)  // the full chain rule of the window function and the face normal; spawn geometry held constant
      window_bwd_exact(g, d, dL_dphi, dL_dC * sig * g.Cx, make_float3(gN0 * w, gN1 * w, gN2 * w), 0.0f, gv);
    else
      window_bwd(g, dL_dphi, make_float3(gN0 * w, gN1 * w, gN2 * w), gv);
    float* dt = p.d_tri + 3 * (size_t)__ldg(p.cumsum + prim);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      red_add(dt + 3 * k + 0, gv[k].x);
      red_add(dt + 3 * k + 1, gv[k].y);
      red_add(dt + 3 * k + 2, gv[k].z);
    }
    if (!spawn) {
      const float e0 = raw0 < 0.f ? 0.f : g0 * w, e1 = raw1 < 0.f ? 0.f : g1 * w, e2 = raw2 < 0.f ? 0.f : g2 * w;
      float* dsh = p.d_sh + (size_t)prim * p.M * 3;
      const int n = sh_count(p.sh_degree);
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        if (k < n) {
          red_add(dsh + 3 * k + 0, B[k] * e0);
          red_add(dsh + 3 * k + 1, B[k] * e1);
          red_add(dsh + 3 * k + 2, B[k] * e2);
        }
      }
    }
    T = test_T;
    return false;
  }

  // the environment term T env(d) of the ray's radiance
  __device__ __forceinline__ void end() {
    if (p.sec.d_env) env_lookup_bwd(p.sec, d, T, g0, g1, g2);
  }
};

__global__ void __launch_bounds__(kTraceThreads, 4) k_sec_backward(const __grid_constant__ TraceParams p) {
  Counters cnt;
  SecBwdShader sh(p);
  int total = 0;
  for (int l = 0; l <= p.sec.max_depth; ++l) total += sec_level_size(p, l);
  drive_items<32>(p, thread_smem<32>(), sh, cnt, total);
  const unsigned s = __reduce_add_sync(0xFFFFFFFFu, cnt.replays);
  if ((threadIdx.x & 31) == 0 && s != 0u) atomicAdd(p.stats + kStatReplays, (unsigned long long)s);
}

// ---------------------------------------------------------------- hit stream
__global__ void __launch_bounds__(kTraceThreads) k_hit_stream(HitStreamParams p) {
  const Smem sm = thread_smem<kStackDepth>();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.R) return;
  const float3 o = make_float3(p.ray_o[3 * i], p.ray_o[3 * i + 1], p.ray_o[3 * i + 2]);
  const float3 d = make_float3(p.ray_d[3 * i], p.ray_d[3 * i + 1], p.ray_d[3 * i + 2]);
  const RayW r = make_ray(o, d);
  unsigned long long key_min = 0ull;
  int count = 0;
  for (int chunk = 0; chunk < kMaxChunks; ++chunk) {
    float t_drop;
    Counters cnt;
    query<kStackDepth>(p.bvh, r, key_min, kFar, sm.keys, sm.stride, sm.st, t_drop, p.status, cnt, 0);
    int consumed = 0;
    unsigned long long last = 0;
#pragma unroll
    for (int j = 0; j < kChunk; ++j) {
      const unsigned long long key = sm.keys[j * sm.stride];
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

size_t trace_smem_bytes(int cfg) {
  switch (cfg) {
    case kCfgPackets16: return smem_bytes_for<kCfgPackets16>();
    case kCfgPackets32: return smem_bytes_for<kCfgPackets32>();
    case kCfgLanes24: return smem_bytes_for<kCfgLanes24>();
    default: return smem_bytes_for<kCfgLanes32>();
  }
}

namespace {
template <int CFG>
const void* fwd_fn() { return (const void*)k_forward<CFG, kShadeRef>; }
template <int CFG>
const void* bwd_fn() { return (const void*)k_backward<CFG, kShadeRef>; }
const void* collect_fn(int cfg) {
  switch (cfg) {
    case kCfgPackets16: return (const void*)k_collect<kCfgPackets16>;
    case kCfgPackets32: return (const void*)k_collect<kCfgPackets32>;
    case kCfgLanes24: return (const void*)k_collect<kCfgLanes24>;
    default: return (const void*)k_collect<kCfgLanes32>;
  }
}
const void* kernel_for(int which, int cfg) {
  switch (cfg) {
    case kCfgPackets16: return which == 0 ? fwd_fn<kCfgPackets16>() : bwd_fn<kCfgPackets16>();
    case kCfgPackets32: return which == 0 ? fwd_fn<kCfgPackets32>() : bwd_fn<kCfgPackets32>();
    case kCfgLanes24: return which == 0 ? fwd_fn<kCfgLanes24>() : bwd_fn<kCfgLanes24>();
    default: return which == 0 ? fwd_fn<kCfgLanes32>() : bwd_fn<kCfgLanes32>();
  }
}
}  // namespace

int trace_blocks_per_sm(int which, int cfg) {
  int n = 0;
  const void* fn = which == 2 ? (const void*)k_variant : (which == 3 ? collect_fn(cfg) : kernel_for(which, cfg));
  const size_t smem = which == 2 ? smem_bytes_for<kCfgLanes32>() : trace_smem_bytes(cfg);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, kTraceThreads, smem) != cudaSuccess) n = 1;
  return n > 0 ? n : 1;
}

// The exact-adjoint forward's accumulators take kExactSmemBytes after the
// traversal's shared memory, which takes the lane configurations past the
// default 48 KB of dynamic shared memory: opt those kernels in.
cudaError_t trace_init() {
  cudaError_t e = cudaSuccess;
  auto opt_in = [&](const void* fn, size_t bytes) {
    if (e == cudaSuccess && bytes > 48 * 1024)
      e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  };
  opt_in((const void*)k_forward<kCfgPackets16, kShadeExact>, smem_bytes_for<kCfgPackets16>() + kExactSmemBytes);
  opt_in((const void*)k_forward<kCfgPackets32, kShadeExact>, smem_bytes_for<kCfgPackets32>() + kExactSmemBytes);
  opt_in((const void*)k_forward<kCfgPackets16, kShadeExact, true>, smem_bytes_for<kCfgPackets16>() + kExactSmemBytes);
  opt_in((const void*)k_forward<kCfgPackets32, kShadeExact, true>, smem_bytes_for<kCfgPackets32>() + kExactSmemBytes);
  opt_in((const void*)k_forward<kCfgLanes24, kShadeExact>, smem_bytes_for<kCfgLanes24>() + kExactSmemBytes);
  opt_in((const void*)k_forward<kCfgLanes32, kShadeExact>, smem_bytes_for<kCfgLanes32>() + kExactSmemBytes);
  return e;
}

// Grid of a replay-only build: the traversing build's grid (SMs x its blocks
// per SM) at the replay build's blocks per SM.
inline int replay_grid(int grid) { return grid / kMinBlocks * kReplayBlocks; }

template <int MODE>
cudaError_t launch_forward_t(const TraceParams& p, int grid, cudaStream_t s) {
  const size_t extra = MODE == kShadeExact ? kExactSmemBytes : 0;
  if (p.fwd_pair) {
    if (p.cfg == kCfgPackets16)
      k_forward<kCfgPackets16, MODE, true><<<replay_grid(grid), kTraceThreads, smem_bytes_for<kCfgPackets16>() + extra, s>>>(p);
    else
      k_forward<kCfgPackets32, MODE, true><<<replay_grid(grid), kTraceThreads, smem_bytes_for<kCfgPackets32>() + extra, s>>>(p);
  }
  switch (p.cfg) {
    case kCfgPackets16: k_forward<kCfgPackets16, MODE><<<grid, kTraceThreads, smem_bytes_for<kCfgPackets16>() + extra, s>>>(p); break;
    case kCfgPackets32: k_forward<kCfgPackets32, MODE><<<grid, kTraceThreads, smem_bytes_for<kCfgPackets32>() + extra, s>>>(p); break;
    case kCfgLanes24: k_forward<kCfgLanes24, MODE><<<grid, kTraceThreads, smem_bytes_for<kCfgLanes24>() + extra, s>>>(p); break;
    default: k_forward<kCfgLanes32, MODE><<<grid, kTraceThreads, smem_bytes_for<kCfgLanes32>() + extra, s>>>(p); break;
  }
  return cudaGetLastError();
}

template <int MODE>
cudaError_t launch_backward_t(const TraceParams& p, int grid, cudaStream_t s) {
  if (p.bwd_pair) {
    if (p.cfg == kCfgPackets16)
      k_backward<kCfgPackets16, MODE, true><<<replay_grid(grid), kTraceThreads, smem_bytes_for<kCfgPackets16>(), s>>>(p);
    else
      k_backward<kCfgPackets32, MODE, true><<<replay_grid(grid), kTraceThreads, smem_bytes_for<kCfgPackets32>(), s>>>(p);
  }
  switch (p.cfg) {
    case kCfgPackets16: k_backward<kCfgPackets16, MODE><<<grid, kTraceThreads, smem_bytes_for<kCfgPackets16>(), s>>>(p); break;
    case kCfgPackets32: k_backward<kCfgPackets32, MODE><<<grid, kTraceThreads, smem_bytes_for<kCfgPackets32>(), s>>>(p); break;
    case kCfgLanes24: k_backward<kCfgLanes24, MODE><<<grid, kTraceThreads, smem_bytes_for<kCfgLanes24>(), s>>>(p); break;
    default: k_backward<kCfgLanes32, MODE><<<grid, kTraceThreads, smem_bytes_for<kCfgLanes32>(), s>>>(p); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_collect(const TraceParams& p, int grid, cudaStream_t s) {
  switch (p.cfg) {
    case kCfgPackets16: k_collect<kCfgPackets16><<<grid, kTraceThreads, smem_bytes_for<kCfgPackets16>(), s>>>(p); break;
    case kCfgPackets32: k_collect<kCfgPackets32><<<grid, kTraceThreads, smem_bytes_for<kCfgPackets32>(), s>>>(p); break;
    case kCfgLanes24: k_collect<kCfgLanes24><<<grid, kTraceThreads, smem_bytes_for<kCfgLanes24>(), s>>>(p); break;
    default: k_collect<kCfgLanes32><<<grid, kTraceThreads, smem_bytes_for<kCfgLanes32>(), s>>>(p); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_forward(const TraceParams& p, int grid, cudaStream_t s) {
  if (p.variant != 0) {
    k_variant<<<grid, kTraceThreads, smem_bytes_for<kCfgLanes32>(), s>>>(p);
    return cudaGetLastError();
  }
  switch (p.mode) {
    case kShadeExact: return launch_forward_t<kShadeExact>(p, grid, s);
    case kShadeRefArith: return launch_forward_t<kShadeRefArith>(p, grid, s);
    default: return launch_forward_t<kShadeRef>(p, grid, s);
  }
}

cudaError_t launch_backward(const TraceParams& p, int grid, cudaStream_t s) {
  switch (p.mode) {
    case kShadeExact: return launch_backward_t<kShadeExact>(p, grid, s);
    case kShadeRefArith: return launch_backward_t<kShadeRefArith>(p, grid, s);
    default: return launch_backward_t<kShadeRef>(p, grid, s);
  }
}

int sec_blocks_per_sm(int which) {
  int n = 0;
  const void* fn = which == 0 ? (const void*)k_sec_trace
                              : (which == 1 ? (const void*)k_sec_backward
                                            : (which == 2 ? (const void*)k_sec_primary : (const void*)k_sec_collect));
  const size_t smem = which == 2 ? smem_bytes_for<kCfgPackets16>()
                                 : (which == 0 ? sec_trace_smem()
                                               : (which == 3 ? sec_collect_smem() : smem_bytes_for<kCfgLanes32>()));
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, kTraceThreads, smem) != cudaSuccess) n = 1;
  return n > 0 ? n : 1;
}

cudaError_t launch_sec_trace(const TraceParams& p, int grid, cudaStream_t s) {
  k_sec_trace<<<grid, kTraceThreads, sec_trace_smem(), s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_sec_collect(const TraceParams& p, int grid, cudaStream_t s) {
  k_sec_collect<<<grid, kTraceThreads, sec_collect_smem(), s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_sec_primary(const TraceParams& p, int grid, cudaStream_t s) {
  k_sec_primary<<<grid, kTraceThreads, smem_bytes_for<kCfgPackets16>(), s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_sec_resolve(const TraceParams& p, cudaStream_t s) {
  const long long cap = p.sec.level == 0 ? (long long)p.views[0].H * p.views[0].W : p.sec.cap[p.sec.level];
  const int grid = (int)std::min<long long>((cap + 255) / 256, 4096);
  if (grid == 0) return cudaSuccess;
  k_sec_resolve<<<grid, 256, 0, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_sec_sort_keys(const TraceParams& p, uint32_t* keys, uint32_t* vals, cudaStream_t s) {
  const int cap = p.sec.cap[p.sec.level];
  const int grid = std::min((cap + 255) / 256, 148 * 8);
  if (grid == 0) return cudaSuccess;
  k_sec_sort_keys<<<grid, 256, 0, s>>>(p, keys, vals);
  return cudaGetLastError();
}

cudaError_t launch_sec_backward(const TraceParams& p, int grid, cudaStream_t s) {
  k_sec_backward<<<grid, kTraceThreads, smem_bytes_for<kCfgLanes32>(), s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_hit_stream(const HitStreamParams& p, cudaStream_t s) {
  const int grid = (p.R + kTraceThreads - 1) / kTraceThreads;
  if (grid == 0) return cudaSuccess;
  k_hit_stream<<<grid, kTraceThreads, smem_bytes_for<kCfgLanes32>(), s>>>(p);
  return cudaGetLastError();
}

}  // namespace tt
