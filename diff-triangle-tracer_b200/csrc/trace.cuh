// Launch interface of the trace kernels (trace.cu).
#pragma once
#include <cuda_runtime.h>

#include "tt_device.cuh"

struct tt_camera;  // include/tritracer.h

namespace tt {

// One camera image: its rays ([H][W][3]) and per-pixel outputs/inputs
// (channel-major [C][H][W]). Tiles are 8x4 pixels; tile_begin is the view's
// first tile in the launch's global tile numbering.
constexpr int kMaxViews = 32;
struct ViewDesc {
  const float* ray_o;
  const float* ray_d;
  float* out_color;
  float* out_others;
  const float* colors;   // adjoint: forward colour
  const float* others;   // adjoint: forward side outputs
  const float* dL_dpix;  // adjoint: upstream gradients
  const float* dL_doth;
  const float* interval;  // optional [2][H][W]: per-ray [t_near, t_far] clip of the traversal
  float* record;          // optional [3][H][W] (forward): t of the first / last hit visited, terminated
  int H, W, ntx, tile_begin;
  long long ray_begin;    // hit cache index of the view's pixel 0 (views laid out one after another)
};

// Hit cache: the k-closest queries of every ray as the forward found them,
// so the adjoint replays them instead of traversing again (a query's result
// depends only on the ray, the BVH and the key range, all unchanged). A
// 32-byte header; then the main part, k + 1 rows of `rays` 64-bit words with
// each ray's first query: rows 0..k-1 the sorted keys, row k the trusted
// bound t_drop (float bits, low half) and the pool entry of the ray's next
// query (high half, kNoEntry if none); then the pool, k + 2 rows of
// `pool_cap` words: later queries laid out the same way plus row k + 1, the
// query's lower key. The adjoint uses the cache only if the header's k, ray
// count, pool size and BVH generation are its own, and a pool entry only if
// its lower key is the one its own march asks for.
struct HitCacheHeader {
  uint32_t magic;
  uint32_t k;
  long long rays;
  unsigned long long gen;  // BVH builds + refits of the handle when the forward ran
  uint32_t pool_cap;       // pool entries
  uint32_t pool_used;      // entries handed out (may pass pool_cap: the rest were not stored)
};
constexpr uint32_t kHitCacheMagic = 0x43485454u;  // "TTHC"
constexpr uint32_t kNoEntry = 0xFFFFFFFFu;
__host__ __device__ inline size_t hit_cache_main_bytes(int k, long long rays) {
  return sizeof(HitCacheHeader) + (size_t)(k + 1) * 8 * (size_t)rays;
}
// The plain forward / adjoint's cache also holds each stored query's hit
// colours after the pool: per entry (main part, then pool) 3k float rows,
// the raw (unclamped) colour of the hit in slot i in rows 3i, 3i + 1, 3i + 2.
// The shading pass writes the colour of every hit it blends and the adjoint
// reads it instead of evaluating the hit's SH again. Header k carries
// kCacheColorsFlag when the colours were written.
constexpr uint32_t kCacheColorsFlag = 0x10000u;
__host__ __device__ inline size_t hit_cache_color_bytes(int k, long long entries) {
  return (size_t)12 * k * (size_t)entries;
}
// keys and colours of `rays` first queries and `pool` later ones
__host__ __device__ inline size_t hit_cache_bytes_pool(int k, long long rays, long long pool) {
  return hit_cache_main_bytes(k, rays) + (size_t)(k + 2) * 8 * (size_t)pool + hit_cache_color_bytes(k, rays + pool);
}
// default pool: later queries of a quarter of the rays
__host__ __device__ inline size_t hit_cache_bytes(int k, long long rays) {
  return hit_cache_bytes_pool(k, rays, (rays + 3) / 4);
}
// Cache modes: off; write (the forward stores its queries); read (the
// adjoint replays them); fill (the shading pass of the split forward replays
// what the collecting pass stored and stores the queries it traverses).
constexpr int kCacheOff = 0, kCacheWrite = 1, kCacheRead = 2, kCacheFill = 3;

// Secondary-ray passes: one record per ray of each pixel's ray tree
// (64 bytes). Level 0 holds the primary rays (record i = pixel i of view 0;
// their origin/direction fields are unused), level k + 1 the rays spawned by
// level k.
struct SecRecord {
  float o[3];
  int pixel;
  float d[3];
  float tau;   // product of the spawn weights along the path (the adjoint's scale)
  float L[3];  // radiance: without the spawn term after the trace, complete after the resolve
  float F;     // Fresnel share of the reflected child
  float w;     // blending weight of the spawning hit
  int child_r, child_t;  // records of the children in the next level, or -1
  uint32_t cache_link;   // hit cache: pool entry of the ray's first query (levels >= 1), or kNoEntry
};

constexpr int kMaxSecDepth = 2;

struct SecParams {
  const int* material;  // [P], 1 = dielectric interface
  const float* ior;     // [P]
  const float* env;     // [env_h][env_w][3] lat-long radiance
  int env_h, env_w, max_depth;
  SecRecord* rec;
  int level;                       // level traced / resolved by this launch
  int base[kMaxSecDepth + 1];      // first record of each level
  int cap[kMaxSecDepth + 1];       // records each level can hold
  int* count;                      // [kMaxSecDepth + 1] records per level, levels >= 1 (device)
  // Order in which k_sec_trace takes the records of the level it traces
  // (levels >= 1): item i is record base[level] + order[i]; nullptr = queue
  // order. The spawned rays sorted by direction and origin (Morton
  // code), so that the rays of a warp cross nearly the same BVH nodes.
  const uint32_t* order;
  // adjoint only, optional: gradients of the environment map and of the
  // per-triangle IOR (through the Fresnel share), or nullptr
  float* d_env;
  float* d_ior;
  // adjoint only: the order each spawned level was traced in (item i of
  // level l is record base[l] + bwd_order[l][i]), or nullptr for queue order
  const uint32_t* bwd_order[kMaxSecDepth + 1];
};

// Shading modes of the plain forward and adjoint (tt_config): the
// reference's semantics with the hit point from an FP64 plane solve
// (default); the exact adjoint; the reference's semantics in the reference's
// own FP32 arithmetic (hit point o + t d, window function on absolute
// coordinates), for comparison with the reference's code.
constexpr int kShadeRef = 0, kShadeExact = 1, kShadeRefArith = 2;

struct TraceParams {
  BvhView bvh;
  int nviews;
  int ntiles;  // tiles over all views
  ViewDesc views[kMaxViews];
  const float* verts;
  const int* cumsum;
  const int* num_points;
  const float* shs;
  int sh_degree, M;
  const float* cols;  // [P][3] precomputed colours in place of SH (shs NULL), or NULL
  float* d_cols;      // their gradient (adjoint)
  const float* opac;
  const float* sigma;
  const float* bg;
  // per-triangle forward outputs
  float* scaling;
  float* density;
  float* max_blending;
  // adjoint outputs
  float* d_tri;
  float* d_sigma;
  float* d_opac;
  float* d_sh;
  // variants (extra = [r, cx, cy, cz, samples])
  int variant;
  float sph_r, sph_cx, sph_cy, sph_cz;
  int samples;
  int tmin_inclusive;
  int mode;     // kShade*: how the plain forward / adjoint shade a hit
  int cfg;      // traversal configuration, kCfg*
  int collect_queries;  // collecting pass: queries stored per ray at most (0 = all the march makes)
  int count_work;       // count node visits and triangle tests (tt_stats), off by default
  int bwd_pair;         // adjoint launched as a replay-only / traversing pair: one of the two works
  int fwd_pair;         // shading pass of the split forward launched as such a pair
  int* work;    // tile counter, zero at launch
  int* status;  // kStatus* bits
  unsigned long long* stats;  // forward counters, kNumStats of them (add_stats in trace.cu)
  SecParams sec;              // secondary-ray passes only
  // hit cache (plain forward / adjoint only)
  void* hit_cache;
  int cache_mode;             // kCache*
  long long cache_rays;       // rays of all views of the launch
  unsigned long long cache_gen;
  uint32_t cache_pool_cap;    // pool entries the buffer holds
  float* cache_colors;        // plain forward / adjoint: the cache's colour rows (main part), or nullptr
};

struct HitStreamParams {
  BvhView bvh;
  int R;
  const float* ray_o;
  const float* ray_d;
  int max_hits;
  uint32_t* ids;
  float* ts;
  int* counts;
  int* status;
};

// counters: rays, evaluated hits, blended hits, node visits, triangle tests,
// queries, warp-packet node visits, interval continuations, interval
// re-traces (forward), hit cache replays (adjoint)
constexpr int kNumStats = 10;
constexpr int kStatReplays = 9;

constexpr int kTraceThreads = 128;
constexpr int kStackDepth = 32;
// traversal configurations (see trace.cu)
constexpr int kCfgLanes32 = 0;    // one ray per lane, 32-entry stack, 16 hits per query
constexpr int kCfgPackets16 = 1;  // warp packets of 8x4 pixels, 16 hits per query
constexpr int kCfgPackets32 = 2;  // warp packets, 32 hits per query
constexpr int kCfgLanes24 = 3;    // one ray per lane, 24-entry stack
constexpr int kNumCfgs = 4;

size_t trace_smem_bytes(int cfg);
// Resident blocks per SM of the forward / adjoint / variant kernels.
int trace_blocks_per_sm(int which /*0 forward, 1 adjoint, 2 variant, 3 collecting pass*/, int cfg);
// once per handle: kernel attributes (dynamic shared memory opt-ins)
cudaError_t trace_init();
// Traversal-only pass that fills the hit cache with every query of the march.
cudaError_t launch_collect(const TraceParams& p, int grid, cudaStream_t s);
cudaError_t launch_forward(const TraceParams& p, int grid, cudaStream_t s);
cudaError_t launch_backward(const TraceParams& p, int grid, cudaStream_t s);
cudaError_t launch_hit_stream(const HitStreamParams& p, cudaStream_t s);
// Secondary-ray passes (views[0] only): trace level p.sec.level, resolve it,
// or run the adjoint of every ray of every level.
int sec_blocks_per_sm(int which /*0 trace (levels >= 1), 1 adjoint, 2 primary level, 3 collecting pass*/);
cudaError_t launch_sec_trace(const TraceParams& p, int grid, cudaStream_t s);
cudaError_t launch_sec_primary(const TraceParams& p, int grid, cudaStream_t s);
// Traversal-only pass over a spawned level (fills the ray tree's hit cache).
cudaError_t launch_sec_collect(const TraceParams& p, int grid, cudaStream_t s);
cudaError_t launch_sec_resolve(const TraceParams& p, cudaStream_t s);
// Sort keys of the records of level p.sec.level (cap of them; the unused
// slots get 0xFFFFFFFF and sort last) and their indices, for sort_pairs.
cudaError_t launch_sec_sort_keys(const TraceParams& p, uint32_t* keys, uint32_t* vals, cudaStream_t s);
cudaError_t launch_sec_backward(const TraceParams& p, int grid, cudaStream_t s);
// camera.cu: primary rays of up to kMaxViews pinhole cameras (tt_camera_rays)
cudaError_t launch_camera_rays(const tt_camera* cams, int n, cudaStream_t s);

}  // namespace tt
