// Proposal network: batched inference and one training step (forward, loss,
// backward, weight gradients, Adam) of the ray-interval MLP on the
// 5th-generation tensor cores. No reference counterpart: the reference traces
// every ray from the camera to the far plane.
//
// Tensor-core scheme (4 warps per CTA, 128 rays per tile = MMA M):
//  * every operand sits in shared memory in the no-swizzle core-matrix
//    layout: 8x8 BF16 blocks of 128 contiguous bytes (8 rows of 16 bytes),
//    the blocks of one group of 8 columns stacked over all R rows, column
//    groups R*16 bytes apart. A tile read with K along its columns is a
//    K-major operand; the SAME tile read with K along its rows (second
//    descriptor, leading/stride offsets swapped) is an MN-major operand. So
//    the forward product (act x W^T), the input gradient (dZ x W) and the
//    weight gradient (dZ^T x act) all read the one copy of each activation
//    and weight tile; nothing is transposed in memory;
//  * the bias of every layer is a weight column fed by a constant-1 input,
//    so the bias gradient comes out of the same weight-gradient MMA;
//  * one thread issues the MMAs and tcgen05.commit arrives on an mbarrier
//    that all threads wait on (bounded; a timeout sets the status word and
//    the CTA frees its tensor memory and returns); each thread then reads its
//    row of the FP32 accumulator with tcgen05.ld (32x32b);
//  * the training kernel keeps the four weight-gradient accumulators in
//    tensor memory across all of its tiles (M = 64 layout: row m in lane
//    m % 16 + 32 * (m / 16)) and writes them out once; the Adam kernel sums
//    the CTAs' partials in a fixed order (deterministic).
#include <cuda_bf16.h>

#include <cmath>
#include <mutex>

#include "proposal.cuh"
#include "tt_device.cuh"

namespace tt {
namespace mlp {
namespace {

constexpr int kThreads = 128;
constexpr int kActBytes = kTileRows * kIn * 2;  // one 128 x 80 BF16 activation tile
constexpr int kDzBytes = kTileRows * kHid * 2;  // one 128 x 64 BF16 gradient tile
constexpr int kWBytes = kParams * 2;
constexpr int kWaitLimit = 1 << 20;  // mbarrier polls before a wait gives up
constexpr uint32_t kInferCols = 128; // tensor-memory columns: two 128 x 64 accumulators (one per warp group)
constexpr uint32_t kTrainCols = 512; // accumulator + 4 weight-gradient accumulators (64 + 4 * 80)

__host__ __device__ constexpr int layer_rows(int l) { return l < 3 ? kHid : kOutRows; }
__host__ __device__ constexpr int layer_off(int l) { return l * kHid * kIn; }
__host__ __device__ constexpr uint32_t dw_col(int l) { return 64u + 80u * (uint32_t)l; }

// Byte offset of element (r, c) of an R-row BF16 tile in the core-matrix layout.
__host__ __device__ constexpr int core_off(int R, int r, int c) { return (c >> 3) * (R * 16) + r * 16 + (c & 7) * 2; }

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, no swizzle: start address, leading- and
// stride-dimension byte offsets (16-byte units), descriptor version 1.
__device__ __forceinline__ uint64_t make_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// R-row tile read with K along its columns (K-major) or along its rows (MN-major).
__device__ __forceinline__ uint64_t desc_k(uint32_t addr, int R) { return make_desc(addr, (uint32_t)R * 16u, 128u); }
__device__ __forceinline__ uint64_t desc_mn(uint32_t addr, int R) { return make_desc(addr, 128u, (uint32_t)R * 16u); }

// Instruction descriptor, kind::f16: BF16 A and B, FP32 accumulator, M x N.
__host__ __device__ constexpr uint32_t make_idesc(int M, int N, int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes -> visible to the tensor cores
__device__ __forceinline__ void fence_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t mbar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(1u) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (int i = 0; i < kWaitLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 16 consecutive FP32 columns of this thread's tensor-memory lane (the load
// and its completion wait in one statement, so no use can move above it).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// whole warp
__device__ __forceinline__ void tmem_alloc(uint32_t slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(ncols) : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&h);
}

// Distance s along the ray from its origin to the closest approach of its
// line to the centre c: the network sees o + s d (centred) and predicts t - s.
__device__ __forceinline__ float closest_offset(float3& o, float3 d, float cx, float cy, float cz) {
  o = make_float3(o.x - cx, o.y - cy, o.z - cz);
  const float dd = d.x * d.x + d.y * d.y + d.z * d.z;
  const float s = dd > 0.f ? -(o.x * d.x + o.y * d.y + o.z * d.z) / dd : 0.f;
  o = make_float3(fmaf(s, d.x, o.x), fmaf(s, d.y, o.y), fmaf(s, d.z, o.z));
  return s;
}

// The 80 inputs of one ray as 40 BF16 pairs: the 6 coordinates (centred
// closest-approach origin, scaled, and direction), then for k = 0..5 the sines
// and the cosines of 2^k pi x over the 6 coordinates, then the constant 1
// (bias input) and a zero.
__device__ __forceinline__ void encode(float3 o, float3 d, float scale, uint32_t (&x)[40]) {
  float f[kIn];
  const float v[6] = {o.x * scale, o.y * scale, o.z * scale, d.x, d.y, d.z};
#pragma unroll
  for (int j = 0; j < 6; ++j) f[j] = v[j];
  // octave 0 from sincospif, each next octave by the double-angle identities
  // sin 2a = 2 sin a cos a, cos 2a = (cos a - sin a)(cos a + sin a): a few
  // FMAs instead of a full sincospif per value. The error doubles per octave
  // (~1e-6 after five), far below the BF16 step (~4e-3) the inputs are
  // rounded to.
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    float s, c;
    sincospif(v[j], &s, &c);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      f[6 + 12 * k + j] = s;
      f[12 + 12 * k + j] = c;
      const float s2 = 2.0f * s * c, c2 = (c - s) * (c + s);
      s = s2;
      c = c2;
    }
  }
  f[78] = 1.0f;
  f[79] = 0.0f;
#pragma unroll
  for (int i = 0; i < 40; ++i) x[i] = pack_bf16(f[2 * i], f[2 * i + 1]);
}

// Row r of a 128-row tile with 8 * groups columns.
template <int G>
__device__ __forceinline__ void put_row(unsigned char* tile, int r, const uint32_t (&x)[4 * G]) {
#pragma unroll
  for (int g = 0; g < G; ++g)
    *reinterpret_cast<uint4*>(tile + core_off(kTileRows, r, 8 * g)) = make_uint4(x[4 * g], x[4 * g + 1], x[4 * g + 2], x[4 * g + 3]);
}

// ReLU of a 64-wide accumulator row, followed by the bias input.
__device__ __forceinline__ void hidden_row(uint32_t lane_base, uint32_t (&x)[40]) {
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    float z[16];
    tmem_ld16(lane_base + 16u * q, z);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const float a = z[2 * j] > 0.f ? z[2 * j] : 0.f, b = z[2 * j + 1] > 0.f ? z[2 * j + 1] : 0.f;
      x[8 * q + j] = pack_bf16(a, b);
    }
  }
  x[32] = pack_bf16(1.0f, 0.0f);
#pragma unroll
  for (int i = 33; i < 40; ++i) x[i] = 0u;
}

// D[128 x R] = act[128 x 80] * W^T (W: R x 80), K = 80 in 5 steps.
__device__ __forceinline__ void issue_forward(uint32_t d, uint32_t act, uint32_t w, int R) {
  const uint32_t id = make_idesc(kTileRows, R, 0, 0);
#pragma unroll
  for (int k = 0; k < kIn / 16; ++k)
    mma_bf16(d, desc_k(act + k * 2 * kTileRows * 16, kTileRows), desc_k(w + k * 2 * R * 16, R), id, k > 0 ? 1u : 0u);
}

// dW[64 x 80] (+)= dZ^T act: M = 64 output rows, N = 80 inputs, K = 128 rays.
__device__ __forceinline__ void issue_weight_grad(uint32_t d, uint32_t dz, uint32_t act, bool first) {
  const uint32_t id = make_idesc(64, kIn, 1, 1);
#pragma unroll
  for (int k = 0; k < kTileRows / 16; ++k)
    mma_bf16(d, desc_mn(dz + k * 256, kTileRows), desc_mn(act + k * 256, kTileRows), id, (!first || k > 0) ? 1u : 0u);
}

// dA[128 x 64] = dZ[128 x R] W[R x 64 of 80]: K = R rows of W.
__device__ __forceinline__ void issue_input_grad(uint32_t d, uint32_t dz, uint32_t w, int R) {
  const uint32_t id = make_idesc(kTileRows, kHid, 0, 1);
  for (int k = 0; k < R / 16; ++k)
    mma_bf16(d, desc_k(dz + k * 2 * kTileRows * 16, kTileRows), desc_mn(w + k * 256, R), id, k > 0 ? 1u : 0u);
}

__device__ __forceinline__ void load_weights(unsigned char* wsm, const uint16_t* w) {
  const uint4* src = reinterpret_cast<const uint4*>(w);
  for (int i = threadIdx.x; i < kWBytes / 16; i += blockDim.x) reinterpret_cast<uint4*>(wsm)[i] = __ldg(src + i);
}

__device__ __forceinline__ int find_set(const InferParams& p, int tile) {
  int lo = 0, hi = p.nsets - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (p.sets[mid].tile_begin <= tile)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// ------------------------------------------------------------- inference
// Two groups of 4 warps per CTA, each with its own activation tile, mbarrier
// and 64 tensor-memory columns, run independent tiles over the one shared
// copy of the weights: while one group waits on its MMA chain (issue ->
// commit -> mbarrier -> tcgen05.ld -> epilogue -> next layer) the other one
// works, and the weights' shared memory is paid once for both. Groups
// synchronise on their own named barriers (1 and 2), the CTA only at the
// start and the end.
constexpr int kInferGroups = 2;
constexpr int kInferThreads = kThreads * kInferGroups;

__device__ __forceinline__ void group_sync(int g) {
  asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(kThreads) : "memory");
}
__device__ __forceinline__ bool group_and(int g, bool v) {
  int r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.s32 p, %1, 0;\n\tbar.red.and.pred q, %2, %3, p;\n\t"
      "selp.s32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"((int)v), "r"(1 + g), "r"(kThreads)
      : "memory");
  return r != 0;
}

__global__ void __launch_bounds__(kInferThreads, 3) k_infer(const __grid_constant__ InferParams p) {
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char* wsm = smem;
  uint64_t* mbars = reinterpret_cast<uint64_t*>(smem + kWBytes + kInferGroups * kActBytes);
  uint32_t* slot = reinterpret_cast<uint32_t*>(mbars + kInferGroups);
  const int warp = threadIdx.x >> 5, grp = warp >> 2, tid = threadIdx.x & (kThreads - 1);
  unsigned char* act = smem + kWBytes + grp * kActBytes;
  load_weights(wsm, p.w);
  if (threadIdx.x < kInferGroups) mbar_init(smem_addr(mbars + threadIdx.x));
  if (warp == 0) tmem_alloc(smem_addr(slot), kInferCols);
  fence_smem();
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tbase = *slot;
  const uint32_t tmem = tbase + 64u * (uint32_t)grp;  // this group's accumulator columns
  const uint32_t lane_base = tmem + ((uint32_t)((warp & 3) * 32) << 16);
  const uint32_t mb = smem_addr(mbars + grp), a_act = smem_addr(act), a_w = smem_addr(wsm);
  uint32_t phase = 0;
  bool ok = true;
  for (int tile = blockIdx.x * kInferGroups + grp; tile < p.ntiles && ok; tile += gridDim.x * kInferGroups) {
    const RaySet& rs = p.sets[find_set(p, tile)];
    const int r = (tile - rs.tile_begin) * kTileRows + tid;
    const bool valid = r < rs.n;
    float3 o = make_float3(0.f, 0.f, 0.f), d = make_float3(0.f, 0.f, 1.f);
    if (valid) {
      const float* po = rs.o + (size_t)r * rs.stride;
      const float* pd = rs.d + (size_t)r * rs.stride;
      o = make_float3(__ldg(po), __ldg(po + 1), __ldg(po + 2));
      d = make_float3(__ldg(pd), __ldg(pd + 1), __ldg(pd + 2));
    }
    const float s_off = closest_offset(o, d, p.cx, p.cy, p.cz);
    uint32_t x[40];
    encode(o, d, p.origin_scale, x);
    put_row<10>(act, tid, x);
    fence_smem();
    fence_before();
    group_sync(grp);
    for (int l = 0; l < 4; ++l) {
      if (tid == 0) {
        fence_after();
        issue_forward(tmem, a_act, a_w + 2 * layer_off(l), layer_rows(l));
        mma_commit(mb);
      }
      ok = mbar_wait(mb, phase);
      phase ^= 1u;
      ok = group_and(grp, ok);
      if (!ok) break;
      fence_after();
      if (l < 3) {
        hidden_row(lane_base, x);
        put_row<10>(act, tid, x);
        fence_smem();
      } else {
        float y[16];
        tmem_ld16(lane_base, y);
        if (valid) {
          // far_cap is measured from the closest approach, like the outputs
          const float t0 = fmaf(y[0], p.t_scale, p.t_shift) + s_off - p.margin_near;
          const float f1 = fmaf(y[1], p.t_scale, p.t_shift) + p.margin_far;
          const float t1 = f1 >= p.far_cap ? INFINITY : f1 + s_off;
          rs.out0[(size_t)r * rs.ostride] = t0;
          rs.out1[(size_t)r * rs.ostride] = t1;
        }
      }
      fence_before();
      group_sync(grp);
    }
  }
  if (!ok && tid == 0) atomicOr(p.status, kStatusTimeout);
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0) tmem_free(tbase, kInferCols);
}

// ------------------------------------------------------------- training
__global__ void __launch_bounds__(kThreads, 1) k_train(const __grid_constant__ TrainParams p) {
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char* wsm = smem;
  unsigned char* act = smem + kWBytes;  // 4 tiles: X, H1, H2, H3 (each with its bias input)
  unsigned char* dz = act + 4 * kActBytes;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(dz + kDzBytes);
  uint32_t* slot = reinterpret_cast<uint32_t*>(mbar + 1);
  __shared__ float red[kThreads / 32];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  load_weights(wsm, p.w);
  if (tid == 0) mbar_init(smem_addr(mbar));
  if (warp == 0) tmem_alloc(smem_addr(slot), kTrainCols);
  fence_smem();
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *slot;
  const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
  const uint32_t mb = smem_addr(mbar), a_w = smem_addr(wsm), a_dz = smem_addr(dz);
  uint32_t a_act[4];
#pragma unroll
  for (int l = 0; l < 4; ++l) a_act[l] = smem_addr(act + l * kActBytes);
  uint32_t phase = 0;
  bool ok = true;
  float loss = 0.f;
  const int t_begin = blockIdx.x * p.tiles_per_cta;
  const int t_end = min(t_begin + p.tiles_per_cta, p.ntiles);
  auto wait_mma = [&]() {
    if (tid == 0) mma_commit(mb);
    ok = mbar_wait(mb, phase);
    phase ^= 1u;
    ok = __syncthreads_and(ok);
    fence_after();
    return ok;
  };
  for (int tile = t_begin; tile < t_end && ok; ++tile) {
    const bool first = tile == t_begin;
    const int row = tile * kTileRows + tid;
    const bool valid = row < p.n;
    float3 o = make_float3(0.f, 0.f, 0.f), d = make_float3(0.f, 0.f, 1.f);
    float tg0 = 0.f, tg1 = 0.f;
    bool has_near = false;
    if (valid) {
      const float* pr = p.rays + (size_t)row * 6;
      o = make_float3(__ldg(pr), __ldg(pr + 1), __ldg(pr + 2));
      d = make_float3(__ldg(pr + 3), __ldg(pr + 4), __ldg(pr + 5));
    }
    const float s_off = closest_offset(o, d, p.cx, p.cy, p.cz);
    if (valid) {
      const float t_near = __ldg(p.targets + 2 * (size_t)row);
      has_near = t_near >= 0.f;
      tg0 = (t_near - s_off - p.t_shift) * p.inv_t_scale;
      tg1 = (__ldg(p.targets + 2 * (size_t)row + 1) - s_off - p.t_shift) * p.inv_t_scale;
    }
    uint32_t x[40];
    encode(o, d, p.origin_scale, x);
    put_row<10>(act, tid, x);
    fence_smem();
    fence_before();
    __syncthreads();
    // forward, keeping every layer's input tile
    float y0 = 0.f, y1 = 0.f;
    for (int l = 0; l < 4 && ok; ++l) {
      if (tid == 0) {
        fence_after();
        issue_forward(tmem, a_act[l], a_w + 2 * layer_off(l), layer_rows(l));
      }
      if (!wait_mma()) break;
      if (l < 3) {
        hidden_row(lane_base, x);
        put_row<10>(act + (l + 1) * kActBytes, tid, x);
        fence_smem();
      } else {
        float y[16];
        tmem_ld16(lane_base, y);
        y0 = y[0];
        y1 = y[1];
      }
      fence_before();
      __syncthreads();
    }
    if (!ok) break;
    // asymmetric squared loss: a t_near above its target (hits cut off)
    // weighs near_weight, a t_far below its target (a continuation)
    // far_weight; rays without hits have no t_near term
    const float e0 = y0 - tg0, e1 = y1 - tg1;
    const float w0 = has_near ? (e0 > 0.f ? p.near_weight : 1.0f) : 0.f;
    const float w1 = e1 < 0.f ? p.far_weight : 1.0f;
    if (valid) loss += w0 * e0 * e0 + w1 * e1 * e1;
    {
      uint32_t g[32];
      g[0] = valid ? pack_bf16(2.f * w0 * e0, 2.f * w1 * e1) : 0u;
#pragma unroll
      for (int i = 1; i < 32; ++i) g[i] = 0u;
      put_row<8>(dz, tid, g);
    }
    fence_smem();
    fence_before();
    __syncthreads();
    // backward: dW_l += dZ_l^T act_l; dZ_{l-1} = (dZ_l W_l) * [act_l > 0]
    for (int l = 3; l >= 0 && ok; --l) {
      if (tid == 0) {
        fence_after();
        issue_weight_grad(tmem + dw_col(l), a_dz, a_act[l], first);
        if (l > 0) issue_input_grad(tmem, a_dz, a_w + 2 * layer_off(l), layer_rows(l));
      }
      if (!wait_mma()) break;
      if (l > 0) {
        const unsigned char* h = act + l * kActBytes;  // the layer's input = previous layer's ReLU output
        uint32_t g[32];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          float da[16];
          tmem_ld16(lane_base + 16u * q, da);
#pragma unroll
          for (int half = 0; half < 2; ++half) {
            const uint4 hv = *reinterpret_cast<const uint4*>(h + core_off(kTileRows, tid, 16 * q + 8 * half));
            const uint32_t hw[4] = {hv.x, hv.y, hv.z, hv.w};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const float* v = da + 8 * half + 2 * j;
              const float a = (hw[j] & 0xFFFFu) ? v[0] : 0.f, b = (hw[j] >> 16) ? v[1] : 0.f;
              g[8 * q + 4 * half + j] = pack_bf16(a, b);
            }
          }
        }
        put_row<8>(dz, tid, g);
        fence_smem();
      }
      fence_before();
      __syncthreads();
    }
  }
  // write the weight gradients (zeros for a CTA without tiles) and the loss
  float* out = p.partial + (size_t)blockIdx.x * kPartial;
  const bool any = t_begin < t_end;
  for (int l = 0; l < 4; ++l) {
    const int m = 16 * warp + lane;
#pragma unroll
    for (int c0 = 0; c0 < kIn; c0 += 16) {
      float v[16];
      tmem_ld16(lane_base + dw_col(l) + (uint32_t)c0, v);
      if (lane < 16 && m < layer_rows(l)) {
#pragma unroll
        for (int j = 0; j < 16; ++j) out[layer_off(l) + m * kIn + c0 + j] = (any && ok) ? v[j] : 0.f;
      }
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) loss += __shfl_xor_sync(0xFFFFFFFFu, loss, off);
  if (lane == 0) red[warp] = loss;
  fence_before();
  __syncthreads();
  fence_after();
  if (tid == 0) {
    out[kParams] = ok ? red[0] + red[1] + red[2] + red[3] : 0.f;
    if (!ok) atomicOr(p.status, kStatusTimeout);
  }
  if (warp == 0) tmem_free(tmem, kTrainCols);
}

// ------------------------------------------------------------- Adam
__global__ void k_adam(const __grid_constant__ AdamParams p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kParams) {
    float w = p.master[i];
    if (p.adam) {
      float g = 0.f;
      for (int c = 0; c < p.nparts; ++c) g += p.partial[(size_t)c * kPartial + i];
      g *= p.grad_scale;
      const float m = p.beta1 * p.m[i] + (1.f - p.beta1) * g;
      const float v = p.beta2 * p.v[i] + (1.f - p.beta2) * g * g;
      p.m[i] = m;
      p.v[i] = v;
      w -= p.lr * (m * p.c1) / (sqrtf(v * p.c2) + p.eps);
      p.master[i] = w;
    }
    const int l = i < layer_off(1) ? 0 : (i < layer_off(2) ? 1 : (i < layer_off(3) ? 2 : 3));
    const int j = i - layer_off(l), r = j / kIn, c = j % kIn;
    p.w[layer_off(l) + core_off(layer_rows(l), r, c) / 2] = __bfloat16_as_ushort(__float2bfloat16_rn(w));
  } else if (i == kParams && p.adam && p.loss) {
    float s = 0.f;
    for (int c = 0; c < p.nparts; ++c) s += p.partial[(size_t)c * kPartial + kParams];
    *p.loss = s * p.grad_scale;
  }
}

}  // namespace

size_t infer_smem_bytes() { return (size_t)kWBytes + (size_t)kInferGroups * kActBytes + 8 * kInferGroups + 16; }
size_t train_smem_bytes() { return (size_t)kWBytes + 4 * kActBytes + kDzBytes + 16; }

namespace {
std::mutex g_attr_mu;
bool g_attr_done[64] = {};
cudaError_t set_attrs() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_attr_mu);
  if (dev >= 0 && dev < 64 && g_attr_done[dev]) return cudaSuccess;
  e = cudaFuncSetAttribute(k_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)infer_smem_bytes());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)train_smem_bytes());
  if (e == cudaSuccess && dev >= 0 && dev < 64) g_attr_done[dev] = true;
  return e;
}
}  // namespace

int infer_blocks_per_sm() {
  if (set_attrs() != cudaSuccess) return 1;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_infer, kInferThreads, infer_smem_bytes()) != cudaSuccess)
    n = 1;
  return n > 0 ? n : 1;
}

cudaError_t launch_infer(const InferParams& p, int grid, cudaStream_t s) {
  cudaError_t e = set_attrs();
  if (e != cudaSuccess) return e;
  if (p.ntiles == 0) return cudaSuccess;
  k_infer<<<grid, kInferThreads, infer_smem_bytes(), s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_train(const TrainParams& p, int grid, cudaStream_t s) {
  cudaError_t e = set_attrs();
  if (e != cudaSuccess) return e;
  k_train<<<grid, kThreads, train_smem_bytes(), s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_adam(const AdamParams& p, cudaStream_t s) {
  k_adam<<<(kParams + 1 + 255) / 256, 256, 0, s>>>(p);
  return cudaGetLastError();
}

}  // namespace mlp
}  // namespace tt
