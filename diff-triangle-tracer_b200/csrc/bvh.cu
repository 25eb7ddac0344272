// LBVH builder: replaces the OptiX GAS build/update of the reference
// (tritracer/pipeline.cpp:206-265, driven from tracer.cpp:53-69).
//
//   prep       triangle records (primitive order) + centroid bounds
//   morton     30-bit Morton codes of the centroids
//   sort       4-pass LSD radix sort (8-bit digits), stable, hand-written
//   records    triangle records in Morton order (traversal reads these)
//   karras     binary radix tree over (code, position) keys (Karras, HPG 2012)
//   bottom-up  node boxes, second arrival at each node merges its children
//   collapse   one launch per level: greedily open the largest child until a
//              node has 8 children; subtrees of <= kLeafMax triangles become
//              leaves (a contiguous run of Morton-ordered records)
//   boxes      each wide node's 8 child boxes from the binary boxes
// A refit re-runs prep/records/bottom-up/boxes over the same topology.
#include <algorithm>
#include <cstddef>
#include <cstdio>

#include <cstring>
#include <vector>

#include "bvh.cuh"

namespace tt {

cudaError_t DevBuf::reserve(size_t n) {
  if (n <= bytes && p) return cudaSuccess;
  release();
  cudaError_t e = cudaMalloc(&p, n ? n : 16);
  if (e != cudaSuccess) {
    p = nullptr;
    bytes = 0;
    return e;
  }
  bytes = n;
  return cudaSuccess;
}

void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
}

namespace {

constexpr int kBlock = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kBlock * kSortItems;

struct alignas(16) BinNode {
  float4 lo, hi;
  int left, right, first, last;
};

__device__ __forceinline__ int f2o(float f) {
  const int i = __float_as_int(f);
  return i >= 0 ? i : (i ^ 0x7FFFFFFF);
}
__device__ __forceinline__ float o2f(int i) { return __int_as_float(i >= 0 ? i : (i ^ 0x7FFFFFFF)); }

__device__ __forceinline__ uint32_t expand_bits(uint32_t v) {
  v = (v * 0x00010001u) & 0xFF0000FFu;
  v = (v * 0x00000101u) & 0x0F00F00Fu;
  v = (v * 0x00000011u) & 0xC30C30C3u;
  v = (v * 0x00000005u) & 0x49249249u;
  return v;
}

__global__ void k_bounds_init(int* b) {
  if (threadIdx.x < 3) b[threadIdx.x] = 0x7FFFFFFF;
  else if (threadIdx.x < 6) b[threadIdx.x] = (int)0x80000000;
}

// Triangle records in primitive order (and, when `cen` is set, centroids and
// their bounds for the Morton quantisation).
__global__ void k_prep(const float* __restrict__ verts, const int* __restrict__ cumsum, int P,
                       float4* __restrict__ tri_prim, float4* __restrict__ cen, int* __restrict__ bounds) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  float c[3] = {0.f, 0.f, 0.f};
  const bool ok = p < P;
  if (ok) {
    const float* v = verts + 3 * (size_t)cumsum[p];
    float x[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) x[k] = v[k];
    tri_prim[3 * (size_t)p + 0] = make_float4(x[0], x[1], x[2], __int_as_float(p));
    tri_prim[3 * (size_t)p + 1] = make_float4(x[3], x[4], x[5], 0.f);
    tri_prim[3 * (size_t)p + 2] = make_float4(x[6], x[7], x[8], 0.f);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float lo = fminf(x[a], fminf(x[3 + a], x[6 + a]));
      const float hi = fmaxf(x[a], fmaxf(x[3 + a], x[6 + a]));
      c[a] = 0.5f * (lo + hi);
    }
    if (cen) cen[p] = make_float4(c[0], c[1], c[2], 0.f);
  }
  if (!cen) return;
  // block reduction of the centroid bounds, then one atomic per block
  __shared__ int s_lo[3][kBlock / 32], s_hi[3][kBlock / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    int lo = ok ? f2o(c[a]) : 0x7FFFFFFF;
    int hi = ok ? f2o(c[a]) : (int)0x80000000;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo = min(lo, __shfl_xor_sync(0xFFFFFFFFu, lo, o));
      hi = max(hi, __shfl_xor_sync(0xFFFFFFFFu, hi, o));
    }
    if (lane == 0) {
      s_lo[a][warp] = lo;
      s_hi[a][warp] = hi;
    }
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    const int a = threadIdx.x;
    int lo = s_lo[a][0], hi = s_hi[a][0];
    for (int w = 1; w < kBlock / 32; ++w) {
      lo = min(lo, s_lo[a][w]);
      hi = max(hi, s_hi[a][w]);
    }
    atomicMin(&bounds[a], lo);
    atomicMax(&bounds[3 + a], hi);
  }
}

__global__ void k_morton(const float4* __restrict__ cen, const int* __restrict__ bounds, int P,
                         uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  const float4 c = cen[p];
  const float cc[3] = {c.x, c.y, c.z};
  uint32_t q[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float lo = o2f(bounds[a]), hi = o2f(bounds[3 + a]);
    const float ext = hi - lo;
    float u = ext > 0.f ? (cc[a] - lo) / ext : 0.5f;
    u = fminf(fmaxf(u * 1024.0f, 0.0f), 1023.0f);
    q[a] = (uint32_t)u;
  }
  keys[p] = (expand_bits(q[0]) << 2) | (expand_bits(q[1]) << 1) | expand_bits(q[2]);
  vals[p] = (uint32_t)p;
}

// ------------------------------------------------------------- radix sort
__global__ void k_sort_hist(const uint32_t* __restrict__ keys, int n, int shift, uint32_t* __restrict__ hist,
                            int tiles) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int base = blockIdx.x * kSortTile;
#pragma unroll 4
  for (int i = 0; i < kSortItems; ++i) {
    const int idx = base + i * kBlock + threadIdx.x;
    if (idx < n) atomicAdd(&h[(keys[idx] >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

// Exclusive scan of the histogram (digit-major: all tiles' counts of digit
// 0, then of digit 1, ...), giving each tile's first output position per
// digit. A 1024-thread block scans chunks of kScanChunk counters (8 a
// thread): one block walks them all for a small histogram; a large one is
// scanned as chunks in parallel, then the chunk totals, then each chunk gets
// its total's prefix added.
constexpr int kScanThreads = 1024, kScanPer = 8, kScanChunk = kScanThreads * kScanPer;

// Scans a[base, base + kScanChunk) (bounded by n) exclusively, starting from
// `carry`; returns carry + the chunk's total (to every thread).
__device__ __forceinline__ uint32_t scan_chunk(uint32_t* __restrict__ a, int n, int base, uint32_t carry) {
  __shared__ uint32_t warp_sum[32];
  __shared__ uint32_t total;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t v[kScanPer];
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    const int idx = base + threadIdx.x * kScanPer + k;
    v[k] = idx < n ? a[idx] : 0u;
    s += v[k];
  }
  uint32_t incl = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_sum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const uint32_t w = warp_sum[lane];
    uint32_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
      if (lane >= o) wi += y;
    }
    warp_sum[lane] = wi - w;  // exclusive prefix of warp totals
    if (lane == 31) total = wi;
  }
  __syncthreads();
  uint32_t run = carry + warp_sum[warp] + (incl - s);
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    const int idx = base + threadIdx.x * kScanPer + k;
    if (idx < n) a[idx] = run;
    run += v[k];
  }
  const uint32_t out = carry + total;
  __syncthreads();  // warp_sum and total are reused by the next chunk
  return out;
}

// One block over all of a[0, n).
__global__ void __launch_bounds__(kScanThreads) k_scan_excl(uint32_t* __restrict__ a, int n) {
  uint32_t carry = 0;
  for (int base = 0; base < n; base += kScanChunk) carry = scan_chunk(a, n, base, carry);
}

// Block b scans chunk b on its own and leaves the chunk's total in sums[b].
__global__ void __launch_bounds__(kScanThreads) k_scan_chunks(uint32_t* __restrict__ a, int n,
                                                              uint32_t* __restrict__ sums) {
  const uint32_t t = scan_chunk(a, n, blockIdx.x * kScanChunk, 0u);
  if (threadIdx.x == 0) sums[blockIdx.x] = t;
}

// Adds the exclusive prefix of the chunk totals (scanned sums) to chunk b.
__global__ void __launch_bounds__(kScanThreads) k_scan_add(uint32_t* __restrict__ a, int n,
                                                           const uint32_t* __restrict__ sums) {
  const uint32_t add = sums[blockIdx.x];
  const int base = blockIdx.x * kScanChunk;
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    const int idx = base + k * kScanThreads + threadIdx.x;
    if (idx < n) a[idx] += add;
  }
}

// Words of histogram storage for `tiles` sort tiles: 256 counters a tile and
// the chunk totals of the parallel scan.
size_t hist_words_for_tiles(size_t tiles) {
  const size_t n = 256 * tiles;
  return n + (n + kScanChunk - 1) / kScanChunk;
}

// Launches of one histogram scan.
int scan_launches(int tiles) { return 256 * tiles <= kScanChunk ? 1 : 3; }

// The exclusive scan of hist[0, 256 * tiles); the chunk totals go after it.
void scan_hist(uint32_t* hist, int tiles, cudaStream_t s) {
  const int n = 256 * tiles;
  if (n <= kScanChunk) {
    k_scan_excl<<<1, kScanThreads, 0, s>>>(hist, n);
    return;
  }
  const int chunks = (n + kScanChunk - 1) / kScanChunk;
  uint32_t* sums = hist + n;
  k_scan_chunks<<<chunks, kScanThreads, 0, s>>>(hist, n, sums);
  k_scan_excl<<<1, kScanThreads, 0, s>>>(sums, chunks);
  k_scan_add<<<chunks, kScanThreads, 0, s>>>(hist, n, sums);
}

// Stable scatter of one tile: keys are visited in index order (16 rounds of
// 256), ranked within each warp with __match_any_sync and across warps with a
// per-digit prefix in shared memory.
__global__ void k_sort_scatter(const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                               uint32_t* __restrict__ kout, uint32_t* __restrict__ vout, int n, int shift,
                               const uint32_t* __restrict__ offsets, int tiles) {
  __shared__ uint32_t run[256];
  __shared__ uint32_t wcnt[kBlock / 32][256];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  run[threadIdx.x] = offsets[threadIdx.x * tiles + blockIdx.x];
  const unsigned lt = (1u << lane) - 1u;
  const int base = blockIdx.x * kSortTile;
  for (int it = 0; it < kSortItems; ++it) {
    const int idx = base + it * kBlock + threadIdx.x;
    const bool valid = idx < n;
    const uint32_t k = valid ? kin[idx] : 0u;
    const uint32_t v = valid ? vin[idx] : 0u;
    const uint32_t digit = valid ? ((k >> shift) & 255u) : 256u;
    for (int j = lane; j < 256; j += 32) wcnt[warp][j] = 0u;
    __syncwarp();
    const unsigned peers = __match_any_sync(0xFFFFFFFFu, digit);
    const uint32_t rank = __popc(peers & lt);
    if (valid && rank == 0) wcnt[warp][digit] = __popc(peers);
    __syncthreads();
    {
      const int d = threadIdx.x;
      uint32_t acc = run[d];
#pragma unroll
      for (int w = 0; w < kBlock / 32; ++w) {
        const uint32_t c = wcnt[w][d];
        wcnt[w][d] = acc;
        acc += c;
      }
      run[d] = acc;
    }
    __syncthreads();
    if (valid) {
      const uint32_t pos = wcnt[warp][digit] + rank;
      kout[pos] = k;
      vout[pos] = v;
    }
    __syncthreads();
  }
}

__global__ void k_records(const uint32_t* __restrict__ order, const float4* __restrict__ tri_prim, int P,
                          float4* __restrict__ tri_sorted) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  const uint32_t p = order[i];
  tri_sorted[3 * (size_t)i + 0] = tri_prim[3 * (size_t)p + 0];  // w = primitive index
  tri_sorted[3 * (size_t)i + 1] = tri_prim[3 * (size_t)p + 1];
  tri_sorted[3 * (size_t)i + 2] = tri_prim[3 * (size_t)p + 2];
}

// ------------------------------------------------------------- hierarchy
__device__ __forceinline__ int delta(const uint32_t* __restrict__ keys, int P, int i, int j) {
  if (j < 0 || j >= P) return -1;
  const unsigned long long a = ((unsigned long long)keys[i] << 32) | (uint32_t)i;
  const unsigned long long b = ((unsigned long long)keys[j] << 32) | (uint32_t)j;
  return __clzll(a ^ b);
}

__global__ void k_karras(const uint32_t* __restrict__ keys, int P, BinNode* __restrict__ bn, int* __restrict__ bparent,
                         int* __restrict__ lparent) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P - 1) return;
  const int d = (delta(keys, P, i, i + 1) - delta(keys, P, i, i - 1)) >= 0 ? 1 : -1;
  const int dmin = delta(keys, P, i, i - d);
  int lmax = 2;
  while (delta(keys, P, i, i + lmax * d) > dmin) lmax <<= 1;
  int l = 0;
  for (int t = lmax >> 1; t >= 1; t >>= 1)
    if (delta(keys, P, i, i + (l + t) * d) > dmin) l += t;
  const int j = i + l * d;
  const int dnode = delta(keys, P, i, j);
  int s = 0, t = l;
  do {
    t = (t + 1) >> 1;
    if (delta(keys, P, i, i + (s + t) * d) > dnode) s += t;
  } while (t > 1);
  const int gamma = i + s * d + min(d, 0);
  const int first = min(i, j), last = max(i, j);
  const int left = (first == gamma) ? ~gamma : gamma;
  const int right = (last == gamma + 1) ? ~(gamma + 1) : gamma + 1;
  bn[i].left = left;
  bn[i].right = right;
  bn[i].first = first;
  bn[i].last = last;
  if (left >= 0) bparent[left] = i; else lparent[~left] = i;
  if (right >= 0) bparent[right] = i; else lparent[~right] = i;
  if (i == 0) bparent[0] = -1;
}

__device__ __forceinline__ void tri_box(const float4* __restrict__ tri, int pos, float4& lo, float4& hi) {
  const float4 a = tri[3 * (size_t)pos], b = tri[3 * (size_t)pos + 1], c = tri[3 * (size_t)pos + 2];
  lo = make_float4(fminf(a.x, fminf(b.x, c.x)), fminf(a.y, fminf(b.y, c.y)), fminf(a.z, fminf(b.z, c.z)), 0.f);
  hi = make_float4(fmaxf(a.x, fmaxf(b.x, c.x)), fmaxf(a.y, fmaxf(b.y, c.y)), fmaxf(a.z, fmaxf(b.z, c.z)), 0.f);
}

__device__ __forceinline__ void child_box(const BinNode* bn, const float4* tri, int ref, float4& lo, float4& hi) {
  if (ref >= 0) {
    lo = __ldcg(&bn[ref].lo);
    hi = __ldcg(&bn[ref].hi);
  } else {
    tri_box(tri, ~ref, lo, hi);
  }
}

__global__ void k_bottom_up(const float4* __restrict__ tri, int P, BinNode* bn, const int* __restrict__ bparent,
                            const int* __restrict__ lparent, int* flags) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P || P < 2) return;
  int node = lparent[p];
  while (node >= 0) {
    __threadfence();
    if (atomicAdd(&flags[node], 1) == 0) return;
    __threadfence();
    float4 l0, h0, l1, h1;
    const int left = __ldcg(&bn[node].left), right = __ldcg(&bn[node].right);
    child_box(bn, tri, left, l0, h0);
    child_box(bn, tri, right, l1, h1);
    const float4 lo = make_float4(fminf(l0.x, l1.x), fminf(l0.y, l1.y), fminf(l0.z, l1.z), 0.f);
    const float4 hi = make_float4(fmaxf(h0.x, h1.x), fmaxf(h0.y, h1.y), fmaxf(h0.z, h1.z), 0.f);
    __stcg(&bn[node].lo, lo);
    __stcg(&bn[node].hi, hi);
    node = bparent[node];
  }
}

// ------------------------------------------------------------- collapse
// counters: [0] wide nodes, [1] depth overflow flag, [2] level the collapse
// is at, [3] wide nodes in the levels above it, [4] blocks of the current
// k_collapse_big launch that finished
constexpr int kCtrLevel = 2, kCtrBase = 3, kCtrDone = 4, kNumCounters = 8;

__global__ void k_collapse_init(int P, int* levels, int* wbin, int* counters) {
  const int i = threadIdx.x;
  if (i < kMaxWideLevels + 1) levels[i] = (i == 0) ? 1 : 0;
  if (i < kNumCounters) counters[i] = 0;
  if (i == 0) wbin[0] = (P >= 2) ? 0 : ~0;  // root: binary node 0, or the single leaf
}

__device__ __forceinline__ float half_area(const BinNode* bn, int r) {
  const float4 lo = bn[r].lo, hi = bn[r].hi;
  const float x = hi.x - lo.x, y = hi.y - lo.y, z = hi.z - lo.z;
  return x * y + y * z + z * x;
}

// Wide node w of `level` (its binary source in wbin[w]): opens the child of
// largest surface area until 8 slots are filled, turns subtrees of at most
// kLeafMax triangles into leaves and appends the others to the next level
// (from index next_base on).
__device__ __forceinline__ void collapse_node(int w, int level, int next_base, const BinNode* __restrict__ bn,
                                              int* levels, int* wbin, int* __restrict__ wsrc,
                                              float4* __restrict__ wnodes) {
  const int b = wbin[w];
  int slot[kWide];
  int n;
  if (b < 0) {
    slot[0] = b;
    n = 1;
  } else {
    slot[0] = bn[b].left;
    slot[1] = bn[b].right;
    n = 2;
  }
  while (n < kWide) {
    int best = -1;
    float best_a = -1.f;
    for (int i = 0; i < n; ++i) {
      const int r = slot[i];
      if (r >= 0) {
        const float a = half_area(bn, r);
        if (a > best_a) {
          best_a = a;
          best = i;
        }
      }
    }
    if (best < 0) break;
    const int r = slot[best];
    slot[best] = bn[r].left;
    slot[n++] = bn[r].right;
  }
  uint32_t refs[kWide];
#pragma unroll
  for (int i = 0; i < kWide; ++i) {
    uint32_t ref = kEmptyRef;
    int src = (int)0x80000000;
    if (i < n) {
      const int r = slot[i];
      src = r;
      if (r < 0) {
        ref = leaf_ref((uint32_t)~r, 1u);
      } else {
        const int first = bn[r].first, size = bn[r].last - first + 1;
        if (size <= kLeafMax) {
          ref = leaf_ref((uint32_t)first, (uint32_t)size);
        } else {
          const int idx = next_base + atomicAdd(&levels[level + 1], 1);
          wbin[idx] = r;
          ref = (uint32_t)idx;
        }
      }
    }
    refs[i] = ref;
    wsrc[(size_t)w * kWide + i] = src;
  }
  float4* nd = wnodes + (size_t)w * kNodeF4;
  nd[12] = make_float4(__uint_as_float(refs[0]), __uint_as_float(refs[1]), __uint_as_float(refs[2]),
                       __uint_as_float(refs[3]));
  nd[13] = make_float4(__uint_as_float(refs[4]), __uint_as_float(refs[5]), __uint_as_float(refs[6]),
                       __uint_as_float(refs[7]));
}

// The top-down collapse runs level by level, and the host does not know the
// tree's depth without a synchronisation. So the levels go through a fixed,
// short sequence of launches that find their level on the device:
// k_collapse_small (one block) takes consecutive levels of at most `limit`
// nodes, with a block barrier between levels; each k_collapse_big (full
// grid) takes one level of any size and its last block to finish moves the
// level on; a final k_collapse_small with no limit takes whatever is left.
__global__ void __launch_bounds__(1024) k_collapse_small(const BinNode* __restrict__ bn, int* levels, int* wbin,
                                                         int* __restrict__ wsrc, float4* __restrict__ wnodes,
                                                         int* counters, int limit) {
  int level = counters[kCtrLevel], base = counters[kCtrBase];
  while (level < kMaxWideLevels) {
    const int cnt = *(volatile int*)&levels[level];
    if (cnt == 0 || cnt > limit) break;
    if (level == kMaxWideLevels - 1 && threadIdx.x == 0) counters[1] = 1;
    for (int k = threadIdx.x; k < cnt; k += blockDim.x)
      collapse_node(base + k, level, base + cnt, bn, levels, wbin, wsrc, wnodes);
    __syncthreads();  // the next level's count and sources are complete
    base += cnt;
    ++level;
  }
  if (threadIdx.x == 0) {
    counters[kCtrLevel] = level;
    counters[kCtrBase] = base;
  }
}

__global__ void k_collapse_big(const BinNode* __restrict__ bn, int* levels, int* wbin, int* __restrict__ wsrc,
                               float4* __restrict__ wnodes, int* counters) {
  // every block reads the level before any block can have finished: the
  // last block moves it on only after all blocks have counted themselves out
  const int level = *(volatile int*)&counters[kCtrLevel], base = *(volatile int*)&counters[kCtrBase];
  const int cnt = level < kMaxWideLevels ? *(volatile int*)&levels[level] : 0;
  if (level == kMaxWideLevels - 1 && cnt > 0 && blockIdx.x == 0 && threadIdx.x == 0) counters[1] = 1;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += gridDim.x * blockDim.x)
    collapse_node(base + k, level, base + cnt, bn, levels, wbin, wsrc, wnodes);
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const int done = atomicAdd(&counters[kCtrDone], 1);
    if (done == (int)gridDim.x - 1) {
      counters[kCtrDone] = 0;
      if (cnt > 0) {
        counters[kCtrLevel] = level + 1;
        counters[kCtrBase] = base + cnt;
      }
      __threadfence();
    }
  }
}

// Launches of k_collapse_big between the two k_collapse_small: the levels of
// more than kSmallLevel nodes of a large scene (a 3M-triangle LBVH has about
// 4), with room to spare; further ones fall to the final one-block pass.
constexpr int kSmallLevel = 4096;
__host__ __forceinline__ int collapse_big_launches(int P) { return P > 8 * kSmallLevel ? 8 : 0; }

__global__ void k_collapse_total(const int* levels, int* counters) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    int s = 0;
    for (int l = 0; l < kMaxWideLevels; ++l) s += levels[l];
    counters[0] = s;
  }
}

// (infinite planes of empty slots pass through unchanged)
__device__ __forceinline__ float pad_lo(float v) { return isinf(v) ? v : v - (fabsf(v) * 4e-6f + 1e-12f); }
__device__ __forceinline__ float pad_hi(float v) { return isinf(v) ? v : v + (fabsf(v) * 4e-6f + 1e-12f); }

// Child boxes of every wide node (SoA across the 8 slots); empty slots get
// inverted boxes (lo = +inf, hi = -inf), which no slab test accepts.
__global__ void k_wide_boxes(const int* __restrict__ wsrc, const BinNode* __restrict__ bn,
                             const float4* __restrict__ tri, const int* __restrict__ counters, int cap,
                             float4* __restrict__ wnodes) {
  const int total = counters[0];
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < total && w < cap; w += gridDim.x * blockDim.x) {
    float lo[3][kWide], hi[3][kWide];
#pragma unroll
    for (int i = 0; i < kWide; ++i) {
      const int r = wsrc[(size_t)w * kWide + i];
      float4 l, h;
      if (r == (int)0x80000000) {
        l = make_float4(INFINITY, INFINITY, INFINITY, 0.f);
        h = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.f);
      } else if (r >= 0) {
        l = bn[r].lo;
        h = bn[r].hi;
      } else {
        tri_box(tri, ~r, l, h);
      }
      // padded outward by a few ulps (relative) plus a tiny absolute margin, so
      // a slab test rounded in FP32 never culls a hit the triangle test reports
      lo[0][i] = pad_lo(l.x); lo[1][i] = pad_lo(l.y); lo[2][i] = pad_lo(l.z);
      hi[0][i] = pad_hi(h.x); hi[1][i] = pad_hi(h.y); hi[2][i] = pad_hi(h.z);
    }
    float4* nd = wnodes + (size_t)w * kNodeF4;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      nd[4 * a + 0] = make_float4(lo[a][0], lo[a][1], lo[a][2], lo[a][3]);
      nd[4 * a + 1] = make_float4(lo[a][4], lo[a][5], lo[a][6], lo[a][7]);
      nd[4 * a + 2] = make_float4(hi[a][0], hi[a][1], hi[a][2], hi[a][3]);
      nd[4 * a + 3] = make_float4(hi[a][4], hi[a][5], hi[a][6], hi[a][7]);
    }
  }
}

inline int blocks_for(long long n) { return (int)((n + kBlock - 1) / kBlock); }

cudaError_t launch_collapse(int P, const BinNode* bn, int* levels, int* wbin, int* wsrc, float4* wnodes,
                            int* counters, cudaStream_t s) {
  k_collapse_init<<<1, 128, 0, s>>>(P, levels, wbin, counters);
  k_collapse_small<<<1, 1024, 0, s>>>(bn, levels, wbin, wsrc, wnodes, counters, kSmallLevel);
  const int wcap = P > 1 ? P - 1 : 1;
  const int grid = blocks_for(wcap) < 148 * 4 ? blocks_for(wcap) : 148 * 4;
  for (int i = 0; i < collapse_big_launches(P); ++i)
    k_collapse_big<<<grid, kBlock, 0, s>>>(bn, levels, wbin, wsrc, wnodes, counters);
  k_collapse_small<<<1, 1024, 0, s>>>(bn, levels, wbin, wsrc, wnodes, counters, 0x7FFFFFFF);
  return cudaGetLastError();
}

}  // namespace

cudaError_t Bvh::reserve(int P) {
  if (P <= cap_) return cudaSuccess;
  const size_t n = (size_t)P;
  const size_t tiles = (n + kSortTile - 1) / kSortTile;
  const size_t wcap = n > 1 ? n - 1 : 1;
  cudaError_t e;
#define TT_RES(buf, bytes)            \
  if ((e = buf.reserve(bytes)) != cudaSuccess) return e;
  TT_RES(tri_prim_, n * 3 * sizeof(float4));
  TT_RES(tri_sorted_, n * 3 * sizeof(float4));
  TT_RES(centroid_, n * sizeof(float4));
  TT_RES(bounds_, 8 * sizeof(int));
  TT_RES(keys_, n * 4);
  TT_RES(vals_, n * 4);
  TT_RES(keys2_, n * 4);
  TT_RES(vals2_, n * 4);
  TT_RES(hist_, hist_words_for_tiles(tiles) * 4);
  TT_RES(bnode_, (n > 1 ? n - 1 : 1) * sizeof(BinNode));
  TT_RES(bparent_, (n > 1 ? n - 1 : 1) * 4);
  TT_RES(lparent_, n * 4);
  TT_RES(flags_, (n > 1 ? n - 1 : 1) * 4);
  TT_RES(wnodes_, wcap * kNodeF4 * sizeof(float4));
  TT_RES(wsrc_, wcap * kWide * 4);
  TT_RES(wbin_, wcap * 4);
  TT_RES(levels_, (kMaxWideLevels + 1) * 4);
  TT_RES(counters_, kNumCounters * 4);
#undef TT_RES
  cap_ = P;
  return cudaSuccess;
}

cudaError_t Bvh::prep(const float* verts, const int* cumsum, int P, bool with_centroids, cudaStream_t s) {
  if (with_centroids) {
    k_bounds_init<<<1, 32, 0, s>>>(bounds_.as<int>());
    ++launches_;
  }
  ++launches_;
  k_prep<<<blocks_for(P), kBlock, 0, s>>>(verts, cumsum, P, tri_prim_.as<float4>(),
                                          with_centroids ? centroid_.as<float4>() : nullptr, bounds_.as<int>());
  return cudaGetLastError();
}

cudaError_t Bvh::boxes(cudaStream_t s) {
  const int P = P_;
  cudaError_t e;
  if (P >= 2) {
    if ((e = cudaMemsetAsync(flags_.p, 0, (size_t)(P - 1) * 4, s)) != cudaSuccess) return e;
    k_bottom_up<<<blocks_for(P), kBlock, 0, s>>>(tri_sorted_.as<float4>(), P, bnode_.as<BinNode>(),
                                                 bparent_.as<int>(), lparent_.as<int>(), flags_.as<int>());
    ++launches_;
  }
  ++launches_;
  const int wcap = P > 1 ? P - 1 : 1;
  const int grid = blocks_for(wcap) < 148 * 8 ? blocks_for(wcap) : 148 * 8;
  k_wide_boxes<<<grid, kBlock, 0, s>>>(wsrc_.as<int>(), bnode_.as<BinNode>(), tri_sorted_.as<float4>(),
                                       counters_.as<int>(), wcap, wnodes_.as<float4>());
  return cudaGetLastError();
}

cudaError_t Bvh::build(const float* verts, const int* cumsum, int P, cudaStream_t s) {
  built_ = false;
  P_ = P;
  if (P <= 0) {
    built_ = true;
    return cudaSuccess;
  }
  cudaError_t e = reserve(P);
  if (e != cudaSuccess) return e;
  if ((e = prep(verts, cumsum, P, true, s)) != cudaSuccess) return e;
  // morton + 4 x (hist, scan, scatter) + records + karras + bottom-up + collapse init/levels/total + boxes
  const int tiles = (P + kSortTile - 1) / kSortTile;
  launches_ += 1 + 4 * (2 + scan_launches(tiles)) + 1 + (P >= 2 ? 2 : 0) + 1 + (2 + collapse_big_launches(P)) + 1 + 1;
  k_morton<<<blocks_for(P), kBlock, 0, s>>>(centroid_.as<float4>(), bounds_.as<int>(), P, keys_.as<uint32_t>(),
                                            vals_.as<uint32_t>());
  // 30-bit keys: four 8-bit passes, ending back in keys_/vals_
  uint32_t *ka = keys_.as<uint32_t>(), *va = vals_.as<uint32_t>();
  uint32_t *kb = keys2_.as<uint32_t>(), *vb = vals2_.as<uint32_t>();
  for (int pass = 0; pass < 4; ++pass) {
    const int shift = 8 * pass;
    k_sort_hist<<<tiles, kBlock, 0, s>>>(ka, P, shift, hist_.as<uint32_t>(), tiles);
    scan_hist(hist_.as<uint32_t>(), tiles, s);
    k_sort_scatter<<<tiles, kBlock, 0, s>>>(ka, va, kb, vb, P, shift, hist_.as<uint32_t>(), tiles);
    uint32_t* t;
    t = ka; ka = kb; kb = t;
    t = va; va = vb; vb = t;
  }
  // after an even number of passes the sorted data is back in keys_/vals_
  k_records<<<blocks_for(P), kBlock, 0, s>>>(vals_.as<uint32_t>(), tri_prim_.as<float4>(), P,
                                             tri_sorted_.as<float4>());
  if (P >= 2)
    k_karras<<<blocks_for(P - 1), kBlock, 0, s>>>(keys_.as<uint32_t>(), P, bnode_.as<BinNode>(), bparent_.as<int>(),
                                                  lparent_.as<int>());
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  // binary boxes are needed by the collapse's area heuristic
  if (P >= 2) {
    if ((e = cudaMemsetAsync(flags_.p, 0, (size_t)(P - 1) * 4, s)) != cudaSuccess) return e;
    k_bottom_up<<<blocks_for(P), kBlock, 0, s>>>(tri_sorted_.as<float4>(), P, bnode_.as<BinNode>(),
                                                 bparent_.as<int>(), lparent_.as<int>(), flags_.as<int>());
  }
  if ((e = launch_collapse(P, bnode_.as<BinNode>(), levels_.as<int>(), wbin_.as<int>(), wsrc_.as<int>(),
                           wnodes_.as<float4>(), counters_.as<int>(), s)) != cudaSuccess)
    return e;
  const int wcap = P > 1 ? P - 1 : 1;
  k_collapse_total<<<1, 32, 0, s>>>(levels_.as<int>(), counters_.as<int>());
  const int grid = blocks_for(wcap) < 148 * 8 ? blocks_for(wcap) : 148 * 8;
  k_wide_boxes<<<grid, kBlock, 0, s>>>(wsrc_.as<int>(), bnode_.as<BinNode>(), tri_sorted_.as<float4>(),
                                       counters_.as<int>(), wcap, wnodes_.as<float4>());
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  built_ = true;
  return cudaSuccess;
}

cudaError_t Bvh::refit(const float* verts, const int* cumsum, int P, cudaStream_t s) {
  if (!built_ || P != P_) return build(verts, cumsum, P, s);
  if (P <= 0) return cudaSuccess;
  cudaError_t e;
  if ((e = prep(verts, cumsum, P, false, s)) != cudaSuccess) return e;
  ++launches_;
  k_records<<<blocks_for(P), kBlock, 0, s>>>(vals_.as<uint32_t>(), tri_prim_.as<float4>(), P,
                                             tri_sorted_.as<float4>());
  return boxes(s);
}

// BVH blob: the topology only. Every box (binary nodes' lo/hi, the wide
// nodes' 12 child-box words) is recomputed by the refit that follows a load,
// so a blob holds the Morton permutation, the binary nodes' child/range
// fields, the parent links, the wide slots' binary sources and the wide
// nodes' child references: 28 bytes per triangle + 64 per wide node.
namespace {
struct BlobHeader {
  char magic[8];  // "TTBVH\0\0\2"
  int P, nw;      // triangles, wide nodes
  long long pad;
};
constexpr char kBlobMagic[8] = {'T', 'T', 'B', 'V', 'H', 0, 0, 2};
constexpr size_t kBinTopoOff = offsetof(BinNode, left), kBinTopoBytes = sizeof(BinNode) - kBinTopoOff;
constexpr size_t kWideRefOff = 12 * sizeof(float4), kWideRefBytes = (kNodeF4 - 12) * sizeof(float4);

size_t blob_bytes(int P, int nw) {
  const size_t p = (size_t)P, b = P > 1 ? (size_t)P - 1 : 1;
  return sizeof(BlobHeader) + p * 4 + b * kBinTopoBytes + b * 4 + p * 4 + (size_t)nw * kWide * 4 +
         (size_t)nw * kWideRefBytes;
}

// Host check of a blob's contents before anything reaches the device: every
// index in range, the Morton order a permutation, the binary hierarchy a
// tree rooted at node 0 whose parent links match its child links (the
// refit's bottom-up pass walks them), and every wide child reference
// pointing to a later wide node (so the wide hierarchy has no cycle).
bool blob_contents_valid(const char* in, int P, int nw) {
  const size_t p = (size_t)P, b = P > 1 ? (size_t)P - 1 : 1;
  const uint32_t* vals = reinterpret_cast<const uint32_t*>(in);
  const int* topo = reinterpret_cast<const int*>(in + p * 4);  // left, right, first, last per binary node
  const int* bparent = reinterpret_cast<const int*>(in + p * 4 + b * kBinTopoBytes);
  const int* lparent = bparent + b;
  const int* wsrc = lparent + p;
  const uint32_t* wref = reinterpret_cast<const uint32_t*>(wsrc + (size_t)nw * kWide);
  std::vector<char> seen(p, 0);
  for (size_t i = 0; i < p; ++i) {
    if (vals[i] >= (uint32_t)P || seen[vals[i]]) return false;
    seen[vals[i]] = 1;
  }
  if (P >= 2) {
    const int nb = P - 1;
    std::vector<char> leaf_seen(p, 0), node_seen(b, 0);
    std::vector<int> todo{0};
    if (bparent[0] != -1) return false;
    int nodes = 0, leaves = 0;
    while (!todo.empty()) {
      const int n = todo.back();
      todo.pop_back();
      if (node_seen[n]) return false;
      node_seen[n] = 1;
      ++nodes;
      const int* t = topo + 4 * (size_t)n;
      if (t[2] < 0 || t[3] >= P || t[2] >= t[3]) return false;
      for (int c = 0; c < 2; ++c) {
        const int ch = t[c];
        if (ch >= 0) {
          if (ch >= nb || bparent[ch] != n) return false;
          todo.push_back(ch);
        } else {
          const int l = ~ch;
          if (l >= P || leaf_seen[l] || lparent[l] != n) return false;
          leaf_seen[l] = 1;
          ++leaves;
        }
      }
    }
    if (nodes != nb || leaves != P) return false;
  }
  for (size_t i = 0; i < (size_t)nw * kWide; ++i) {
    const int v = wsrc[i];
    if (v != (int)0x80000000 && !(v >= 0 && v < (P > 1 ? P - 1 : 0)) && !(v < 0 && ~v < P)) return false;
  }
  for (size_t w = 0; w < (size_t)nw; ++w) {
    for (int i = 0; i < kWide; ++i) {
      const uint32_t r = wref[w * kWide + i];
      if (r == kEmptyRef) continue;
      if (ref_is_leaf(r)) {
        if (leaf_count(r) > (uint32_t)kLeafMax || leaf_first(r) + leaf_count(r) > (uint32_t)P) return false;
      } else if (r <= w || r >= (uint32_t)nw) {
        return false;
      }
    }
  }
  return true;
}
}  // namespace

cudaError_t Bvh::save(void* dst, size_t capacity, size_t* bytes, cudaStream_t s) {
  if (!built_ || P_ <= 0) {
    *bytes = 0;
    return cudaSuccess;
  }
  int cnt[4] = {0, 0, 0, 0};
  cudaError_t e = cudaMemcpyAsync(cnt, counters_.p, sizeof(cnt), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return e;
  const int nw = cnt[0];
  *bytes = blob_bytes(P_, nw);
  if (!dst) return cudaSuccess;
  if (capacity < *bytes) return cudaErrorInvalidValue;
  const size_t p = (size_t)P_, b = P_ > 1 ? (size_t)P_ - 1 : 1;
  char* o = static_cast<char*>(dst);
  BlobHeader hd;
  std::memcpy(hd.magic, kBlobMagic, 8);
  hd.P = P_;
  hd.nw = nw;
  hd.pad = 0;
  std::memcpy(o, &hd, sizeof(hd));
  o += sizeof(hd);
  auto d2h = [&](const DevBuf& buf, size_t n) {
    if (e == cudaSuccess) e = cudaMemcpyAsync(o, buf.p, n, cudaMemcpyDeviceToHost, s);
    o += n;
  };
  // rows of `width` bytes at `off` within records of `pitch` bytes: packed on
  // the device first (a strided copy into pageable host memory goes row by row)
  void* pack = nullptr;
  const size_t pack_bytes = std::max(b * kBinTopoBytes, (size_t)nw * kWideRefBytes);
  if ((e = cudaMallocAsync(&pack, pack_bytes, s)) != cudaSuccess) return e;
  auto d2h_rows = [&](const DevBuf& buf, size_t off, size_t width, size_t pitch, size_t rows) {
    if (e == cudaSuccess)
      e = cudaMemcpy2DAsync(pack, width, static_cast<const char*>(buf.p) + off, pitch, width, rows,
                            cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(o, pack, width * rows, cudaMemcpyDeviceToHost, s);
    o += width * rows;
  };
  d2h(vals_, p * 4);
  d2h_rows(bnode_, kBinTopoOff, kBinTopoBytes, sizeof(BinNode), b);
  d2h(bparent_, b * 4);
  d2h(lparent_, p * 4);
  d2h(wsrc_, (size_t)nw * kWide * 4);
  d2h_rows(wnodes_, kWideRefOff, kWideRefBytes, kNodeF4 * sizeof(float4), (size_t)nw);
  const cudaError_t ef = cudaFreeAsync(pack, s);
  if (e == cudaSuccess) e = ef;
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return e;
}

int Bvh::load(const void* src, size_t bytes, const float* verts, const int* cumsum, int P, cudaStream_t s,
              cudaError_t* err) {
  *err = cudaSuccess;
  BlobHeader hd;
  if (!src || bytes < sizeof(hd)) return 1;
  std::memcpy(&hd, src, sizeof(hd));
  if (std::memcmp(hd.magic, kBlobMagic, 8) != 0 || hd.P != P || P <= 0 || hd.nw < 1 ||
      hd.nw > (P > 1 ? P - 1 : 1) || bytes != blob_bytes(P, hd.nw))
    return 1;
  if (!blob_contents_valid(static_cast<const char*>(src) + sizeof(hd), P, hd.nw)) return 2;
  built_ = false;
  if ((*err = reserve(P)) != cudaSuccess) return 0;
  const size_t p = (size_t)P, b = P > 1 ? (size_t)P - 1 : 1;
  const char* in = static_cast<const char*>(src) + sizeof(hd);
  cudaError_t e = cudaSuccess;
  auto h2d = [&](DevBuf& buf, size_t n) {
    if (e == cudaSuccess) e = cudaMemcpyAsync(buf.p, in, n, cudaMemcpyHostToDevice, s);
    in += n;
  };
  // (uploads into strided destinations go straight from the host: measured
  // faster than staging them on the device, unlike the downloads of save)
  auto h2d_rows = [&](DevBuf& buf, size_t off, size_t width, size_t pitch, size_t rows) {
    if (e == cudaSuccess)
      e = cudaMemcpy2DAsync(static_cast<char*>(buf.p) + off, pitch, in, width, width, rows, cudaMemcpyHostToDevice,
                            s);
    in += width * rows;
  };
  h2d(vals_, p * 4);
  h2d_rows(bnode_, kBinTopoOff, kBinTopoBytes, sizeof(BinNode), b);
  h2d(bparent_, b * 4);
  h2d(lparent_, p * 4);
  h2d(wsrc_, (size_t)hd.nw * kWide * 4);
  h2d_rows(wnodes_, kWideRefOff, kWideRefBytes, kNodeF4 * sizeof(float4), (size_t)hd.nw);
  const int cnt[4] = {hd.nw, 0, 0, 0};
  if (e == cudaSuccess) e = cudaMemcpyAsync(counters_.p, cnt, sizeof(cnt), cudaMemcpyHostToDevice, s);
  // the host blob and cnt may go away on return
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    *err = e;
    return 0;
  }
  P_ = P;
  built_ = true;
  *err = refit(verts, cumsum, P, s);  // triangle records and boxes from the vertices
  return 0;
}

void Bvh::release() {
  DevBuf* all[] = {&tri_prim_, &tri_sorted_, &centroid_, &bounds_, &keys_,  &vals_,  &keys2_, &vals2_, &hist_,
                   &bnode_,    &bparent_,   &lparent_,  &flags_,  &wnodes_, &wsrc_, &wbin_,  &levels_, &counters_};
  for (DevBuf* b : all) b->release();
  cap_ = 0;
  built_ = false;
}

BvhView Bvh::view() const {
  BvhView v;
  v.nodes = wnodes_.as<float4>();
  v.tris = tri_sorted_.as<float4>();
  v.tri_prim = tri_prim_.as<float4>();
  v.P = P_;
  v.has_root = (built_ && P_ > 0) ? 1 : 0;
  v.wide_cap = P_ > 1 ? P_ - 1 : 1;
  return v;
}

// ------------------------------------------------------------- carved storage
namespace {

struct Carver {
  char* base;
  size_t off = 0;
  template <class T>
  T* take(size_t n) {
    off = (off + 255) & ~size_t(255);
    T* p = reinterpret_cast<T*>(base ? base + off : nullptr);
    off += n * sizeof(T);
    return p;
  }
};

BvhStorage carve(char* base, int P, size_t* total) {
  const size_t n = (size_t)(P > 0 ? P : 1);
  const size_t tiles = (n + kSortTile - 1) / kSortTile;
  const size_t inner = n > 1 ? n - 1 : 1;
  Carver c{base};
  BvhStorage st;
  st.tri_prim = c.take<float4>(3 * n);
  st.tri_sorted = c.take<float4>(3 * n);
  st.centroid = c.take<float4>(n);
  st.bounds = c.take<int>(8);
  st.keys = c.take<uint32_t>(n);
  st.vals = c.take<uint32_t>(n);
  st.keys2 = c.take<uint32_t>(n);
  st.vals2 = c.take<uint32_t>(n);
  st.hist = c.take<uint32_t>(hist_words_for_tiles(tiles));
  st.bnode = c.take<BinNode>(inner);
  st.bparent = c.take<int>(inner);
  st.lparent = c.take<int>(n);
  st.flags = c.take<int>(inner);
  st.wnodes = c.take<float4>(inner * kNodeF4);
  st.wsrc = c.take<int>(inner * kWide);
  st.wbin = c.take<int>(inner);
  st.levels = c.take<int>(kMaxWideLevels + 1);
  st.counters = c.take<int>(kNumCounters);
  if (total) *total = (c.off + 255) & ~size_t(255);
  return st;
}

}  // namespace

size_t bvh_storage_bytes(int P) {
  size_t total = 0;
  carve(nullptr, P, &total);
  return total;
}

BvhStorage bvh_storage_carve(void* base, int P) { return carve(static_cast<char*>(base), P, nullptr); }

cudaError_t bvh_build_into(const BvhStorage& st, const float* verts, const int* cumsum, int P, cudaStream_t s) {
  if (P <= 0) return cudaSuccess;
  BinNode* bn = static_cast<BinNode*>(st.bnode);
  k_bounds_init<<<1, 32, 0, s>>>(st.bounds);
  k_prep<<<blocks_for(P), kBlock, 0, s>>>(verts, cumsum, P, st.tri_prim, st.centroid, st.bounds);
  k_morton<<<blocks_for(P), kBlock, 0, s>>>(st.centroid, st.bounds, P, st.keys, st.vals);
  const int tiles = (P + kSortTile - 1) / kSortTile;
  uint32_t *ka = st.keys, *va = st.vals, *kb = st.keys2, *vb = st.vals2;
  for (int pass = 0; pass < 4; ++pass) {
    k_sort_hist<<<tiles, kBlock, 0, s>>>(ka, P, 8 * pass, st.hist, tiles);
    scan_hist(st.hist, tiles, s);
    k_sort_scatter<<<tiles, kBlock, 0, s>>>(ka, va, kb, vb, P, 8 * pass, st.hist, tiles);
    uint32_t* t;
    t = ka; ka = kb; kb = t;
    t = va; va = vb; vb = t;
  }
  k_records<<<blocks_for(P), kBlock, 0, s>>>(st.vals, st.tri_prim, P, st.tri_sorted);
  cudaError_t e;
  if (P >= 2) {
    k_karras<<<blocks_for(P - 1), kBlock, 0, s>>>(st.keys, P, bn, st.bparent, st.lparent);
    if ((e = cudaMemsetAsync(st.flags, 0, (size_t)(P - 1) * 4, s)) != cudaSuccess) return e;
    k_bottom_up<<<blocks_for(P), kBlock, 0, s>>>(st.tri_sorted, P, bn, st.bparent, st.lparent, st.flags);
  }
  if ((e = launch_collapse(P, bn, st.levels, st.wbin, st.wsrc, st.wnodes, st.counters, s)) != cudaSuccess) return e;
  const int wcap = P > 1 ? P - 1 : 1;
  const int grid = blocks_for(wcap) < 148 * 4 ? blocks_for(wcap) : 148 * 4;
  k_collapse_total<<<1, 32, 0, s>>>(st.levels, st.counters);
  k_wide_boxes<<<grid, kBlock, 0, s>>>(st.wsrc, bn, st.tri_sorted, st.counters, wcap, st.wnodes);
  return cudaGetLastError();
}

size_t sort_pairs_hist_words(int n) { return hist_words_for_tiles((size_t)((n + kSortTile - 1) / kSortTile)); }

int sort_pairs_launches(int n, int bits) {
  if (n <= 0) return 0;
  return ((bits + 7) / 8) * (2 + scan_launches((n + kSortTile - 1) / kSortTile));
}

cudaError_t sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t* keys2, uint32_t* vals2, uint32_t* hist, int n,
                       int bits, bool* in_second, cudaStream_t s) {
  *in_second = false;
  if (n <= 0) return cudaSuccess;
  const int tiles = (n + kSortTile - 1) / kSortTile;
  uint32_t *ka = keys, *va = vals, *kb = keys2, *vb = vals2;
  for (int shift = 0; shift < bits; shift += 8) {
    k_sort_hist<<<tiles, kBlock, 0, s>>>(ka, n, shift, hist, tiles);
    scan_hist(hist, tiles, s);
    k_sort_scatter<<<tiles, kBlock, 0, s>>>(ka, va, kb, vb, n, shift, hist, tiles);
    uint32_t* t;
    t = ka; ka = kb; kb = t;
    t = va; va = vb; vb = t;
    *in_second = !*in_second;
  }
  return cudaGetLastError();
}

BvhView bvh_storage_view(const BvhStorage& st, int P) {
  BvhView v;
  v.nodes = st.wnodes;
  v.tris = st.tri_sorted;
  v.tri_prim = st.tri_prim;
  v.P = P;
  v.has_root = P > 0 ? 1 : 0;
  v.wide_cap = P > 1 ? P - 1 : 1;
  return v;
}

}  // namespace tt
