// C ABI (include/tritracer.h): the handle that replaces the reference's
// OptixTracer class (tritracer/tracer.h:67-126, tracer.cpp, pipeline.cpp).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>

#include <nvtx3/nvToolsExt.h>

#include "../../include/tritracer.h"
#include "bvh.cuh"
#include "proposal.cuh"
#include "trace.cuh"

struct tt_tracer {
  tt_config cfg;
  int device = 0;
  int num_sms = 148;
  int fwd_grid = 0, bwd_grid = 0, collect_grid = 0;
  bool split_forward = true;  // plain forward with a hit cache: collecting pass + shading pass
  int collect_queries = 2;    // queries a ray's collecting pass stores at most (0 = all)
  bool count_work = false;    // node visits and triangle tests counted into the stats
  bool sort_secondary = true; // secondary passes: spawned rays traced in sorted order
  tt::DevBuf sec_sort;        // their sort keys / indices (2 x 2 x 4R words) and the sort's histogram
  tt::DevBuf sec_order;       // each spawned level's trace order, kept for the adjoint
  bool sec_sorted = false;    // the last secondary forward sorted its spawned levels
  int cfg_id = tt::kCfgPackets16;
  std::string err;
  tt::Bvh bvh;
  tt::DevBuf scratch;  // int[0] tile counter, int[1] status word, u64 stats[kNumStats] from byte 16,
                       // int[3] secondary-ray queue counters from byte kSecCountOffset
  tt::DevBuf sec_rec;  // secondary-ray queue: R * (2^(depth+1) - 1) records
  tt::DevBuf sec_cache;        // hit cache of that ray tree (tt_forward_secondary writes, the adjoint replays)
  size_t sec_cache_bytes = 0;  // its size for the last tree
  int sec_R = 0, sec_depth = -1;  // the ray tree the last tt_forward_secondary left
  int sec_trace_grid = 0, sec_bwd_grid = 0, sec_primary_grid = 0, sec_collect_grid = 0, sec_collect0_grid = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev_mid = nullptr;
  float pass_ms[2] = {0.f, 0.f};  // last debug forward: collecting pass, shading pass (ms)
  unsigned long long trace_launches = 0;  // trace kernels enqueued
  unsigned long long launch_base = 0;     // launch count at the last stats reset
  unsigned long long bvh_gen = 0;         // BVH builds, refits and loads so far (hit cache validity)
  int k() const { return cfg_id == tt::kCfgPackets32 ? 32 : 16; }
  unsigned long long launches() const { return trace_launches + bvh.launches(); }
};

namespace {

constexpr int kSecCountOffset = 96;
static_assert(16 + tt::kNumStats * 8 <= kSecCountOffset, "stats overlap the secondary-ray counters");

int fail(tt_tracer* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

int cuda_fail(tt_tracer* h, cudaError_t e, const char* what) {
  const int code = (e == cudaErrorMemoryAllocation) ? TT_ERR_OOM : TT_ERR_CUDA;
  return fail(h, code, std::string("CUDA call (") + what + ") failed with error: '" + cudaGetErrorString(e) + "'");
}

#define TT_CUDA(h, call)                                   \
  do {                                                     \
    cudaError_t e_ = (call);                               \
    if (e_ != cudaSuccess) return cuda_fail(h, e_, #call); \
  } while (0)

#define TT_REQUIRE(h, cond, msg)                        \
  do {                                                  \
    if (!(cond)) return fail(h, TT_ERR_INVALID, (msg)); \
  } while (0)

cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

// NVTX range over an entry point, named after it: a profiler shows the
// launches the call enqueues under that name. Free when no tool is attached.
struct Range {
  explicit Range(const char* name) { nvtxRangePushA(name); }
  ~Range() { nvtxRangePop(); }
  Range(const Range&) = delete;
  Range& operator=(const Range&) = delete;
};
#define TT_RANGE() const Range tt_range_(__func__)

int accel_step(tt_tracer* h, const float* verts, int num_vertices, const int* cumsum, int P, int mode,
               cudaStream_t s) {
  TT_REQUIRE(h, mode == TT_BUILD || mode == TT_REFIT || mode == TT_KEEP, "rebuild_gas must be 0, 1 or 2");
  TT_REQUIRE(h, P >= 0, "number_of_points must be >= 0");
  if (mode == TT_KEEP) {
    if (!h->bvh.built()) return fail(h, TT_ERR_STATE, "rebuild_gas=2 before any acceleration structure was built");
    if (h->bvh.P() != P) return fail(h, TT_ERR_STATE, "rebuild_gas=2 with a different triangle count than the build");
    return TT_OK;
  }
  if (P > 0) {
    TT_REQUIRE(h, verts && cumsum, "vertices and cumsum must be device pointers");
    TT_REQUIRE(h, num_vertices >= 3, "need at least 3 vertices");
  }
  TT_REQUIRE(h, P < (1 << 27), "at most 2^27 triangles");
  ++h->bvh_gen;
  cudaError_t e = (mode == TT_BUILD) ? h->bvh.build(verts, cumsum, P, s) : h->bvh.refit(verts, cumsum, P, s);
  if (e != cudaSuccess) return cuda_fail(h, e, mode == TT_BUILD ? "bvh build" : "bvh refit");
  return TT_OK;
}

// Pool entries a hit cache of `bytes` holds after its main part (-1: too
// small for the main part).
long long cache_pool_cap(int k, long long rays, size_t bytes) {
  const size_t main = tt::hit_cache_main_bytes(k, rays);
  if (bytes < main) return -1;
  const unsigned long long cap = (bytes - main) / ((size_t)(k + 2) * 8);
  return (long long)(cap < 0xFFFFFFF0ull ? cap : 0xFFFFFFF0ull);
}

// The same for the plain forward / adjoint's cache, whose entries also hold
// their hits' colours (tt::hit_cache_bytes_pool).
long long cache_pool_cap_colors(int k, long long rays, size_t bytes) {
  const size_t main = tt::hit_cache_main_bytes(k, rays) + tt::hit_cache_color_bytes(k, rays);
  if (bytes < main) return -1;
  const unsigned long long cap = (bytes - main) / ((size_t)(k + 2) * 8 + (size_t)12 * k);
  return (long long)(cap < 0xFFFFFFF0ull ? cap : 0xFFFFFFF0ull);
}

// Colour rows of a plain cache with `cap` pool entries (after the pool's keys).
float* cache_colors_of(void* cache, int k, long long rays, long long cap) {
  return reinterpret_cast<float*>(static_cast<char*>(cache) + tt::hit_cache_main_bytes(k, rays) +
                                  (size_t)(k + 2) * 8 * (size_t)cap);
}

int check_sh(tt_tracer* h, const float* shs, int deg, int M, int P, const float* cols = nullptr) {
  if (cols && !shs) return TT_OK;  // precomputed colours in place of SH
  TT_REQUIRE(h, deg >= 0 && deg <= 3, "sh_degree must be in [0, 3]");
  // an empty scene reads no SH
  TT_REQUIRE(h, P == 0 || M >= (deg + 1) * (deg + 1), "shs has fewer coefficients per triangle than sh_degree needs");
  TT_REQUIRE(h, P == 0 || shs != nullptr, "shs is empty and no colors_precomp was given");
  return TT_OK;
}

}  // namespace

extern "C" {

int tt_create(const tt_config* cfg, tt_tracer** out) {
  if (!out) return TT_ERR_INVALID;
  *out = nullptr;
  tt_tracer* h = new (std::nothrow) tt_tracer();
  if (!h) return TT_ERR_OOM;
  tt_config def;
  std::memset(&def, 0, sizeof(def));
  def.variant = TT_VARIANT_PLAIN;
  def.tmin_inclusive = 1;
  h->cfg = cfg ? *cfg : def;
  if (h->cfg.variant < TT_VARIANT_PLAIN || h->cfg.variant > TT_VARIANT_ENVLIGHT ||
      (h->cfg.exact_adjoint != 0 && h->cfg.variant != TT_VARIANT_PLAIN) ||
      (h->cfg.reference_arithmetic != 0 && (h->cfg.variant != TT_VARIANT_PLAIN || h->cfg.exact_adjoint != 0))) {
    delete h;
    return TT_ERR_INVALID;
  }
  cudaError_t e;
  if ((e = cudaGetDevice(&h->device)) != cudaSuccess ||
      (e = cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device)) != cudaSuccess ||
      (e = h->scratch.reserve(128)) != cudaSuccess || (e = cudaMemset(h->scratch.p, 0, 128)) != cudaSuccess ||
      (e = cudaEventCreate(&h->ev0)) != cudaSuccess || (e = cudaEventCreate(&h->ev1)) != cudaSuccess ||
      (e = cudaEventCreate(&h->ev_mid)) != cudaSuccess ||
      (e = tt::trace_init()) != cudaSuccess) {
    delete h;
    return e == cudaErrorMemoryAllocation ? TT_ERR_OOM : TT_ERR_CUDA;
  }
  h->sec_trace_grid = h->num_sms * tt::sec_blocks_per_sm(0);
  h->sec_primary_grid = h->num_sms * tt::sec_blocks_per_sm(2);
  h->sec_bwd_grid = h->num_sms * tt::sec_blocks_per_sm(1);
  h->sec_collect_grid = h->num_sms * tt::sec_blocks_per_sm(3);
  h->sec_collect0_grid = h->num_sms * tt::trace_blocks_per_sm(3, tt::kCfgPackets16);
  if (tt_set_traversal(h, h->cfg.traversal, h->cfg.k, h->cfg.stack_depth) != TT_OK) {
    delete h;
    return TT_ERR_INVALID;
  }
  *out = h;
  return TT_OK;
}

int tt_set_traversal(tt_tracer* h, int traversal, int k, int stack_depth) {
  if (!h) return TT_ERR_INVALID;
  TT_REQUIRE(h, traversal >= TT_TRAVERSAL_AUTO && traversal <= TT_TRAVERSAL_LANES, "unknown traversal mode");
  TT_REQUIRE(h, k == 0 || k == 16 || k == 32, "k must be 16 or 32");
  TT_REQUIRE(h, stack_depth == 0 || stack_depth == 24 || stack_depth == 32, "stack_depth must be 24 or 32");
  // sphere variants bend rays incoherently: they always trace lane by lane
  const bool lanes = traversal == TT_TRAVERSAL_LANES || h->cfg.variant != TT_VARIANT_PLAIN;
  TT_REQUIRE(h, !(lanes && k == 32), "k = 32 needs packet traversal");
  TT_REQUIRE(h, lanes || stack_depth == 0 || stack_depth == 32, "stack_depth applies to lane traversal");
  int id;
  if (lanes)
    id = stack_depth == 24 ? tt::kCfgLanes24 : tt::kCfgLanes32;
  else
    id = k == 32 ? tt::kCfgPackets32 : tt::kCfgPackets16;
  h->cfg.traversal = traversal;
  h->cfg.k = k;
  h->cfg.stack_depth = stack_depth;
  h->cfg_id = id;
  const int which = h->cfg.variant != TT_VARIANT_PLAIN ? 2 : 0;
  h->fwd_grid = h->num_sms * tt::trace_blocks_per_sm(which, id);
  h->bwd_grid = h->num_sms * tt::trace_blocks_per_sm(1, id);
  h->collect_grid = h->num_sms * tt::trace_blocks_per_sm(3, id);
  return TT_OK;
}

int tt_set_option(tt_tracer* h, int option, int value) {
  if (!h) return TT_ERR_INVALID;
  switch (option) {
    case TT_OPT_SPLIT_FORWARD: h->split_forward = value != 0; return TT_OK;
    case TT_OPT_SORT_SECONDARY: h->sort_secondary = value != 0; return TT_OK;
    case TT_OPT_WORK_COUNTERS: h->count_work = value != 0; return TT_OK;
    case TT_OPT_COLLECT_QUERIES:
      TT_REQUIRE(h, value >= 0, "collect_queries must be >= 0");
      h->collect_queries = value;
      return TT_OK;
    default: return fail(h, TT_ERR_INVALID, "unknown option");
  }
}

size_t tt_hit_cache_bytes(const tt_tracer* h, long long rays) {
  if (!h || rays < 0) return 0;
  return tt::hit_cache_bytes(h->k(), rays);
}

size_t tt_hit_cache_bytes_pool(const tt_tracer* h, long long rays, long long pool_queries) {
  if (!h || rays < 0 || pool_queries < 0) return 0;
  return tt::hit_cache_bytes_pool(h->k(), rays, pool_queries);
}

int tt_camera_rays(tt_tracer* h, const tt_camera* cams, int n_cams, void* stream) {
  TT_RANGE();
  if (!h) return TT_ERR_INVALID;
  TT_REQUIRE(h, cams != nullptr && n_cams >= 1 && n_cams <= tt::kMaxViews, "1 to 32 cameras");
  for (int c = 0; c < n_cams; ++c) {
    TT_REQUIRE(h, cams[c].H > 0 && cams[c].W > 0, "camera H and W must be > 0");
    TT_REQUIRE(h, cams[c].ray_o != nullptr && cams[c].ray_d != nullptr, "camera ray_o / ray_d are null");
    TT_REQUIRE(h, (reinterpret_cast<uintptr_t>(cams[c].ray_o) & 3u) == 0 &&
                      (reinterpret_cast<uintptr_t>(cams[c].ray_d) & 3u) == 0,
               "camera ray_o / ray_d must be 4-byte aligned");
  }
  TT_CUDA(h, tt::launch_camera_rays(cams, n_cams, as_stream(stream)));
  return TT_OK;
}

int tt_hit_cache_usage(tt_tracer* h, const void* hit_cache, void* stream, int* k, long long* pool_cap,
                       long long* pool_used) {
  if (!h) return TT_ERR_INVALID;
  TT_REQUIRE(h, hit_cache != nullptr, "hit_cache is null");
  tt::HitCacheHeader hd;
  const cudaStream_t s = as_stream(stream);
  TT_CUDA(h, cudaMemcpyAsync(&hd, hit_cache, sizeof(hd), cudaMemcpyDeviceToHost, s));
  TT_CUDA(h, cudaStreamSynchronize(s));
  TT_REQUIRE(h, hd.magic == tt::kHitCacheMagic, "hit_cache was not written by a forward");
  if (k) *k = (int)(hd.k & ~tt::kCacheColorsFlag);
  if (pool_cap) *pool_cap = hd.pool_cap;
  if (pool_used) *pool_used = hd.pool_used;
  return TT_OK;
}

int tt_destroy(tt_tracer* h) {
  if (!h) return TT_ERR_INVALID;
  h->bvh.release();
  h->scratch.release();
  h->sec_rec.release();
  h->sec_cache.release();
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->ev_mid) cudaEventDestroy(h->ev_mid);
  delete h;
  return TT_OK;
}

const char* tt_last_error(const tt_tracer* h) { return h ? h->err.c_str() : "null tracer handle"; }

int tt_build(tt_tracer* h, const float* vertices, int num_vertices, const int* cumsum, int P, int mode,
             void* stream) {
  TT_RANGE();
  if (!h) return TT_ERR_INVALID;
  return accel_step(h, vertices, num_vertices, cumsum, P, mode, as_stream(stream));
}

static tt::TraceParams base_params(tt_tracer* h) {
  tt::TraceParams p;
  std::memset(&p, 0, sizeof(p));
  p.bvh = h->bvh.view();
  p.tmin_inclusive = h->cfg.tmin_inclusive;
  p.mode = h->cfg.exact_adjoint ? tt::kShadeExact : (h->cfg.reference_arithmetic ? tt::kShadeRefArith : tt::kShadeRef);
  p.variant = h->cfg.variant;
  p.cfg = h->cfg_id;
  p.count_work = h->count_work ? 1 : 0;
  p.work = h->scratch.as<int>();
  p.status = h->scratch.as<int>() + 1;
  p.stats = reinterpret_cast<unsigned long long*>(h->scratch.as<char>() + 16);
  return p;
}

// Appends a view to the launch: its tiles follow the previous views'.
static int add_view(tt_tracer* h, tt::TraceParams& p, const tt_view& v) {
  TT_REQUIRE(h, p.nviews < tt::kMaxViews, "at most 32 views per call");
  TT_REQUIRE(h, v.H > 0 && v.W > 0, "every view needs H, W > 0");
  TT_REQUIRE(h, (long long)v.H * v.W < (1ll << 31), "too many rays in a view");
  TT_REQUIRE(h, v.ray_o && v.ray_d, "null ray pointer in a view");
  tt::ViewDesc& d = p.views[p.nviews++];
  d.ray_o = v.ray_o;
  d.ray_d = v.ray_d;
  d.out_color = v.out_color;
  d.out_others = v.out_others;
  d.colors = v.colors;
  d.others = v.others;
  d.dL_dpix = v.dL_dpixels;
  d.dL_doth = v.dL_dothers;
  d.interval = v.interval;
  d.record = v.record;
  TT_REQUIRE(h, h->cfg.variant == TT_VARIANT_PLAIN || (!v.interval && !v.record),
             "proposed intervals and hit records are for the plain variant only");
  d.H = v.H;
  d.W = v.W;
  d.ntx = (v.W + 7) / 8;
  d.tile_begin = p.ntiles;
  d.ray_begin = p.cache_rays;
  p.cache_rays += (long long)v.H * v.W;
  const long long tiles = (long long)p.ntiles + (long long)d.ntx * ((v.H + 3) / 4);
  TT_REQUIRE(h, tiles < (1ll << 26), "too many tiles in one call");
  p.ntiles = (int)tiles;
  return TT_OK;
}

static int forward_impl(tt_tracer* h, const tt_fwd_args* a, const tt_view* views, int nviews, void* stream) {
  const cudaStream_t s = as_stream(stream);
  TT_REQUIRE(h, nviews >= 1, "need at least one view");
  for (int i = 0; i < nviews; ++i)
    TT_REQUIRE(h, views[i].out_color && views[i].out_others, "null output pointer in a view");
  TT_REQUIRE(h, a->P == 0 || (a->opacities && a->sigma && a->scaling && a->density_factor && a->max_blending &&
                              a->num_points),
             "null per-triangle pointer");
  TT_REQUIRE(h, a->bg, "null background");
  const float* cols = a->shs ? nullptr : a->colors_precomp;
  TT_REQUIRE(h, !cols || h->cfg.variant == TT_VARIANT_PLAIN, "colors_precomp needs the plain program");
  int rc = check_sh(h, a->shs, a->sh_degree, a->M, a->P, cols);
  if (rc != TT_OK) return rc;
  float ex[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
  if (h->cfg.variant != TT_VARIANT_PLAIN) {
    TT_REQUIRE(h, a->extra && a->extra_len >= (h->cfg.variant == TT_VARIANT_ENVLIGHT ? 5 : 4),
               "variant needs extra = [r, cx, cy, cz(, samples)]");
    // the sphere parameters are a few floats of a device tensor (extract_sphere, common.h:143-148)
    TT_CUDA(h, cudaMemcpyAsync(ex, a->extra, sizeof(float) * (a->extra_len >= 5 ? 5 : 4), cudaMemcpyDeviceToHost, s));
    TT_CUDA(h, cudaStreamSynchronize(s));
  }
  tt::TraceParams p = base_params(h);
  for (int i = 0; i < nviews; ++i) {
    rc = add_view(h, p, views[i]);
    if (rc != TT_OK) return rc;
  }
  rc = accel_step(h, a->vertices, a->num_vertices, a->cumsum, a->P, a->rebuild_gas, s);
  if (rc != TT_OK) return rc;
  if (a->hit_cache) {
    TT_REQUIRE(h, h->cfg.variant == TT_VARIANT_PLAIN, "the hit cache is for the plain program only");
    TT_REQUIRE(h, (reinterpret_cast<uintptr_t>(a->hit_cache) & 15u) == 0, "hit_cache must be 16-byte aligned");
    const long long cap = cache_pool_cap_colors(h->k(), p.cache_rays, a->hit_cache_bytes);
    TT_REQUIRE(h, cap >= 0, "hit_cache is too small for these rays (tt_hit_cache_bytes)");
    p.hit_cache = a->hit_cache;
    p.cache_mode = tt::kCacheWrite;
    p.cache_gen = h->bvh_gen;
    p.cache_pool_cap = (uint32_t)cap;
    p.cache_colors = cache_colors_of(a->hit_cache, h->k(), p.cache_rays, cap);
    TT_CUDA(h, cudaMemsetAsync(a->hit_cache, 0, sizeof(tt::HitCacheHeader), s));
  }
  p.bvh = h->bvh.view();
  p.verts = a->vertices;
  p.cumsum = a->cumsum;
  p.num_points = a->num_points;
  p.shs = a->shs;
  p.sh_degree = a->sh_degree;
  p.M = a->M;
  p.cols = cols;
  p.opac = a->opacities;
  p.sigma = a->sigma;
  p.bg = a->bg;
  p.scaling = a->scaling;
  p.density = a->density_factor;
  p.max_blending = a->max_blending;
  p.sph_r = ex[0];
  p.sph_cx = ex[1];
  p.sph_cy = ex[2];
  p.sph_cz = ex[3];
  p.samples = (int)ex[4];
  if (a->P > 0) TT_CUDA(h, cudaMemsetAsync(a->max_blending, 0, (size_t)a->P * sizeof(float), s));
  if (a->debug) TT_CUDA(h, cudaEventRecord(h->ev0, s));
  const bool split = p.hit_cache && h->split_forward;
  if (split) {
    // traversal-only pass: every query of the march into the cache; the
    // shading pass below replays them
    TT_CUDA(h, cudaMemsetAsync(p.work, 0, sizeof(int), s));
    p.collect_queries = h->collect_queries;
    TT_CUDA(h, tt::launch_collect(p, h->collect_grid, s));
    ++h->trace_launches;
    p.cache_mode = tt::kCacheFill;
    // When the first pass stores every query of every march (no cap, no
    // proposed interval stopping it early), the shading pass runs as a pair:
    // a replay-only build for a complete cache, the traversing one otherwise
    bool clipped = false;
    for (int i = 0; i < p.nviews; ++i) clipped = clipped || p.views[i].interval != nullptr;
    p.fwd_pair = h->collect_queries == 0 && !clipped &&
                         (p.cfg == tt::kCfgPackets16 || p.cfg == tt::kCfgPackets32) ? 1 : 0;
    if (p.fwd_pair) ++h->trace_launches;
  }
  if (a->debug) TT_CUDA(h, cudaEventRecord(h->ev_mid, s));
  TT_CUDA(h, cudaMemsetAsync(p.work, 0, sizeof(int), s));
  TT_CUDA(h, tt::launch_forward(p, h->fwd_grid, s));
  ++h->trace_launches;
  if (a->debug) {
    TT_CUDA(h, cudaEventRecord(h->ev1, s));
    TT_CUDA(h, cudaEventSynchronize(h->ev1));
    float ms = 0.f;
    TT_CUDA(h, cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    if (a->gpu_time_ms) *a->gpu_time_ms = ms;
    float m0 = 0.f, m1 = 0.f;
    TT_CUDA(h, cudaEventElapsedTime(&m0, h->ev0, h->ev_mid));
    TT_CUDA(h, cudaEventElapsedTime(&m1, h->ev_mid, h->ev1));
    h->pass_ms[0] = split ? m0 : 0.f;
    h->pass_ms[1] = m1;
  }
  return TT_OK;
}

int tt_forward_pass_times(tt_tracer* h, float* collect_ms, float* shade_ms) {
  if (!h) return TT_ERR_INVALID;
  if (collect_ms) *collect_ms = h->pass_ms[0];
  if (shade_ms) *shade_ms = h->pass_ms[1];
  return TT_OK;
}

int tt_forward(tt_tracer* h, const tt_fwd_args* a, void* stream) {
  TT_RANGE();
  if (!h) return TT_ERR_INVALID;
  if (!a) return fail(h, TT_ERR_INVALID, "null argument block");
  TT_REQUIRE(h, a->H > 0 && a->W > 0, "ray_o must be [H, W, 3] with H, W > 0");
  TT_REQUIRE(h, a->ray_o && a->ray_d && a->out_color && a->out_others, "null ray or output pointer");
  tt_view v;
  std::memset(&v, 0, sizeof(v));
  v.H = a->H;
  v.W = a->W;
  v.ray_o = a->ray_o;
  v.ray_d = a->ray_d;
  v.out_color = a->out_color;
  v.out_others = a->out_others;
  return forward_impl(h, a, &v, 1, stream);
}

int tt_forward_views(tt_tracer* h, const tt_fwd_args* a, const tt_view* views, int n_views, void* stream) {
  TT_RANGE();
  if (!h) return TT_ERR_INVALID;
  if (!a || !views) return fail(h, TT_ERR_INVALID, "null argument block or view list");
  return forward_impl(h, a, views, n_views, stream);
}

static int backward_impl(tt_tracer* h, const tt_bwd_args* a, const tt_view* views, int nviews, void* stream) {
  const cudaStream_t s = as_stream(stream);
  TT_REQUIRE(h, nviews >= 1, "need at least one view");
  for (int i = 0; i < nviews; ++i)
    TT_REQUIRE(h, views[i].colors && views[i].others && views[i].dL_dpixels && views[i].dL_dothers,
               "null forward-output or upstream-gradient pointer in a view");
  TT_REQUIRE(h, a->P == 0 || (a->opacities && a->sigma && a->cumsum && a->vertices), "null per-triangle pointer");
  const float* cols = a->shs ? nullptr : a->colors_precomp;
  TT_REQUIRE(h, a->P == 0 || (a->dL_dtriangle && a->dL_dsigma && a->dL_dopacity && (a->dL_dsh || cols)),
             "null gradient output");
  TT_REQUIRE(h, !cols || a->dL_dcolors, "colors_precomp needs a dL_dcolors output");
  int rc = check_sh(h, a->shs, a->sh_degree, a->M, a->P, cols);
  if (rc != TT_OK) return rc;
  if (!h->bvh.built()) return fail(h, TT_ERR_STATE, "backward before any forward/build");
  if (h->bvh.P() != a->P) return fail(h, TT_ERR_STATE, "backward with a different triangle count than the forward");
  tt::TraceParams p = base_params(h);
  for (int i = 0; i < nviews; ++i) {
    rc = add_view(h, p, views[i]);
    if (rc != TT_OK) return rc;
  }
  if (a->P > 0) {
    TT_CUDA(h, cudaMemsetAsync(a->dL_dtriangle, 0, (size_t)a->num_vertices * 3 * sizeof(float), s));
    TT_CUDA(h, cudaMemsetAsync(a->dL_dsigma, 0, (size_t)a->P * sizeof(float), s));
    TT_CUDA(h, cudaMemsetAsync(a->dL_dopacity, 0, (size_t)a->P * sizeof(float), s));
    if (a->dL_dsh && a->M > 0) TT_CUDA(h, cudaMemsetAsync(a->dL_dsh, 0, (size_t)a->P * a->M * 3 * sizeof(float), s));
    if (cols) TT_CUDA(h, cudaMemsetAsync(a->dL_dcolors, 0, (size_t)a->P * 3 * sizeof(float), s));
  }
  p.verts = a->vertices;
  p.cumsum = a->cumsum;
  p.num_points = a->num_points;
  p.shs = a->shs;
  p.sh_degree = a->sh_degree;
  p.M = a->M;
  p.cols = cols;
  p.d_cols = a->dL_dcolors;
  p.opac = a->opacities;
  p.sigma = a->sigma;
  p.bg = a->bg;
  p.d_tri = a->dL_dtriangle;
  p.d_sigma = a->dL_dsigma;
  p.d_opac = a->dL_dopacity;
  p.d_sh = a->dL_dsh;
  // a cache written for another k, ray count or pool size (or too small for
  // this k) fails the kernels' header check or is not passed at all: they re-trace
  const long long cap = a->hit_cache ? cache_pool_cap_colors(h->k(), p.cache_rays, a->hit_cache_bytes) : -1;
  if (cap >= 0) {
    TT_REQUIRE(h, (reinterpret_cast<uintptr_t>(a->hit_cache) & 15u) == 0, "hit_cache must be 16-byte aligned");
    p.hit_cache = const_cast<void*>(a->hit_cache);
    p.cache_mode = tt::kCacheRead;
    p.cache_gen = h->bvh_gen;
    p.cache_pool_cap = (uint32_t)cap;
    p.cache_colors = cache_colors_of(const_cast<void*>(a->hit_cache), h->k(), p.cache_rays, cap);
  }
  TT_CUDA(h, cudaMemsetAsync(p.work, 0, sizeof(int), s));
  if (a->debug) TT_CUDA(h, cudaEventRecord(h->ev0, s));
  // with a cache, the packet configurations run the adjoint as a pair: a
  // replay-only build (no traversal code, for a complete cache) and the
  // traversing one; each checks the cache on the device and one returns
  p.bwd_pair = p.hit_cache && (p.cfg == tt::kCfgPackets16 || p.cfg == tt::kCfgPackets32) ? 1 : 0;
  if (p.bwd_pair) ++h->trace_launches;
  TT_CUDA(h, tt::launch_backward(p, h->bwd_grid, s));
  ++h->trace_launches;
  if (a->debug) {
    TT_CUDA(h, cudaEventRecord(h->ev1, s));
    TT_CUDA(h, cudaEventSynchronize(h->ev1));
    float ms = 0.f;
    TT_CUDA(h, cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    if (a->gpu_time_ms) *a->gpu_time_ms = ms;
  }
  return TT_OK;
}

int tt_backward(tt_tracer* h, const tt_bwd_args* a, void* stream) {
  TT_RANGE();
  if (!h) return TT_ERR_INVALID;
  if (!a) return fail(h, TT_ERR_INVALID, "null argument block");
  TT_REQUIRE(h, a->H > 0 && a->W > 0, "ray_o must be [H, W, 3] with H, W > 0");
  TT_REQUIRE(h, a->ray_o && a->ray_d && a->colors && a->others && a->dL_dpixels && a->dL_dothers,
             "null ray, forward-output or upstream-gradient pointer");
  tt_view v;
  std::memset(&v, 0, sizeof(v));
  v.H = a->H;
  v.W = a->W;
  v.ray_o = a->ray_o;
  v.ray_d = a->ray_d;
  v.colors = a->colors;
  v.others = a->others;
  v.dL_dpixels = a->dL_dpixels;
  v.dL_dothers = a->dL_dothers;
  return backward_impl(h, a, &v, 1, stream);
}

int tt_backward_views(tt_tracer* h, const tt_bwd_args* a, const tt_view* views, int n_views, void* stream) {
  TT_RANGE();
  if (!h) return TT_ERR_INVALID;
  if (!a || !views) return fail(h, TT_ERR_INVALID, "null argument block or view list");
  return backward_impl(h, a, views, n_views, stream);
}

int tt_device_status(tt_tracer* h, void* stream) {
  if (!h) return TT_ERR_INVALID;
  const cudaStream_t s = as_stream(stream);
  int st = 0;
  TT_CUDA(h, cudaMemcpyAsync(&st, h->scratch.as<int>() + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
  TT_CUDA(h, cudaStreamSynchronize(s));
  TT_CUDA(h, cudaMemsetAsync(h->scratch.as<int>() + 1, 0, sizeof(int), s));
  if (st & tt::kStatusBounds) return fail(h, TT_ERR_BOUNDS, "a device index check failed (TT_BOUNDS_CHECK build)");
  if (st & tt::kStatusStack) return fail(h, TT_ERR_STACK, "traversal stack overflow made no progress on some ray");
  if (st & tt::kStatusTimeout) return fail(h, TT_ERR_TIMEOUT, "a bounded device loop gave up");
  if (st & tt::kStatusCacheMiss)
    return fail(h, TT_ERR_STATE, "the adjoint's hit cache lacked a query its forward had stored");
  return TT_OK;
}

int tt_get_stats(tt_tracer* h, tt_stats* out, void* stream) {
  if (!h) return TT_ERR_INVALID;
  if (!out) return fail(h, TT_ERR_INVALID, "null stats pointer");
  const cudaStream_t s = as_stream(stream);
  unsigned long long v[tt::kNumStats] = {};
  TT_CUDA(h, cudaMemcpyAsync(v, h->scratch.as<char>() + 16, sizeof(v), cudaMemcpyDeviceToHost, s));
  TT_CUDA(h, cudaStreamSynchronize(s));
  out->rays = v[0];
  out->evaluated_hits = v[1];
  out->blended_hits = v[2];
  out->kernel_launches = h->launches() - h->launch_base;
  out->node_visits = v[3];
  out->triangle_tests = v[4];
  out->queries = v[5];
  out->packet_node_visits = v[6];
  out->interval_continuations = v[7];
  out->interval_retraces = v[8];
  out->hit_cache_replays = v[tt::kStatReplays];
  return TT_OK;
}

int tt_reset_stats(tt_tracer* h, void* stream) {
  if (!h) return TT_ERR_INVALID;
  TT_CUDA(h, cudaMemsetAsync(h->scratch.as<char>() + 16, 0, tt::kNumStats * 8, as_stream(stream)));
  h->launch_base = h->launches();
  return TT_OK;
}

int tt_hit_stream(tt_tracer* h, const float* ray_o, const float* ray_d, int R, int max_hits, uint32_t* ids,
                  float* ts, int* counts, void* stream) {
  TT_RANGE();
  if (!h) return TT_ERR_INVALID;
  TT_REQUIRE(h, R >= 0 && max_hits >= 0, "R and max_hits must be >= 0");
  TT_REQUIRE(h, R == 0 || (ray_o && ray_d && counts && (max_hits == 0 || (ids && ts))), "null pointer");
  if (!h->bvh.built()) return fail(h, TT_ERR_STATE, "hit stream before any build");
  tt::HitStreamParams p;
  p.bvh = h->bvh.view();
  p.R = R;
  p.ray_o = ray_o;
  p.ray_d = ray_d;
  p.max_hits = max_hits;
  p.ids = ids;
  p.ts = ts;
  p.counts = counts;
  p.status = h->scratch.as<int>() + 1;
  TT_CUDA(h, tt::launch_hit_stream(p, as_stream(stream)));
  if (R > 0) ++h->trace_launches;
  return TT_OK;
}

// ---------------------------------------------------------------- proposal network
static int check_mlp(tt_tracer* h, const tt_mlp* net) {
  TT_REQUIRE(h, net != nullptr, "null network");
  TT_REQUIRE(h, net->weights && net->master, "network weights must be device pointers");
  TT_REQUIRE(h, (reinterpret_cast<uintptr_t>(net->weights) & 15u) == 0, "network weights must be 16-byte aligned");
  TT_REQUIRE(h, net->t_scale != 0.f, "t_scale must be nonzero");
  return TT_OK;
}

int tt_mlp_update(tt_tracer* h, const tt_mlp* net, void* stream) {
  TT_RANGE();
  if (!h) return TT_ERR_INVALID;
  int rc = check_mlp(h, net);
  if (rc != TT_OK) return rc;
  tt::mlp::AdamParams a;
  std::memset(&a, 0, sizeof(a));
  a.master = net->master;
  a.w = net->weights;
  a.adam = 0;
  TT_CUDA(h, tt::mlp::launch_adam(a, as_stream(stream)));
  ++h->trace_launches;
  return TT_OK;
}

int tt_mlp_train_step(tt_tracer* h, const tt_mlp* net, const tt_mlp_step* st, const float* rays,
                      const float* targets, int n, float* loss, void* stream) {
  TT_RANGE();
  if (!h) return TT_ERR_INVALID;
  int rc = check_mlp(h, net);
  if (rc != TT_OK) return rc;
  TT_REQUIRE(h, st != nullptr && st->step >= 1, "need a step description with step >= 1");
  TT_REQUIRE(h, n > 0 && rays && targets, "need n > 0 rays and targets");
  TT_REQUIRE(h, net->adam_m && net->adam_v && net->partial, "Adam state and partial buffer must be device pointers");
  const cudaStream_t s = as_stream(stream);
  const int ntiles = (n + tt::mlp::kTileRows - 1) / tt::mlp::kTileRows;
  const int per = (ntiles + h->num_sms - 1) / h->num_sms;
  const int grid = (ntiles + per - 1) / per;
  TT_REQUIRE(h, grid <= net->partial_ctas, "partial buffer too small for this batch");
  tt::mlp::TrainParams p;
  std::memset(&p, 0, sizeof(p));
  p.w = net->weights;
  p.rays = rays;
  p.targets = targets;
  p.n = n;
  p.ntiles = ntiles;
  p.tiles_per_cta = per;
  p.origin_scale = net->origin_scale;
  p.t_shift = net->t_shift;
  p.inv_t_scale = 1.0f / net->t_scale;
  p.cx = net->center[0];
  p.cy = net->center[1];
  p.cz = net->center[2];
  p.near_weight = st->near_weight;
  p.far_weight = st->far_weight;
  p.partial = net->partial;
  p.status = h->scratch.as<int>() + 1;
  TT_CUDA(h, tt::mlp::launch_train(p, grid, s));
  tt::mlp::AdamParams a;
  std::memset(&a, 0, sizeof(a));
  a.partial = net->partial;
  a.nparts = grid;
  a.grad_scale = 1.0f / (float)n;
  a.master = net->master;
  a.m = net->adam_m;
  a.v = net->adam_v;
  a.w = net->weights;
  a.lr = st->lr;
  a.beta1 = st->beta1;
  a.beta2 = st->beta2;
  a.eps = st->eps;
  a.c1 = (float)(1.0 / (1.0 - std::pow((double)st->beta1, st->step)));
  a.c2 = (float)(1.0 / (1.0 - std::pow((double)st->beta2, st->step)));
  a.loss = loss;
  a.adam = 1;
  TT_CUDA(h, tt::mlp::launch_adam(a, s));
  h->trace_launches += 2;
  return TT_OK;
}

static int mlp_infer(tt_tracer* h, const tt_mlp* net, tt::mlp::InferParams& p, float margin_near, float margin_far,
                     float far_cap, cudaStream_t s) {
  p.w = net->weights;
  p.origin_scale = net->origin_scale;
  p.t_shift = net->t_shift;
  p.t_scale = net->t_scale;
  p.cx = net->center[0];
  p.cy = net->center[1];
  p.cz = net->center[2];
  p.margin_near = margin_near;
  p.margin_far = margin_far;
  p.far_cap = far_cap;
  p.status = h->scratch.as<int>() + 1;
  if (p.ntiles == 0) return TT_OK;
  const int grid = std::min(p.ntiles, h->num_sms * tt::mlp::infer_blocks_per_sm());
  TT_CUDA(h, tt::mlp::launch_infer(p, grid, s));
  ++h->trace_launches;
  return TT_OK;
}

int tt_mlp_predict(tt_tracer* h, const tt_mlp* net, const float* rays, int n, float* out, void* stream) {
  TT_RANGE();
  if (!h) return TT_ERR_INVALID;
  int rc = check_mlp(h, net);
  if (rc != TT_OK) return rc;
  TT_REQUIRE(h, n >= 0 && (n == 0 || (rays && out)), "need rays and out for n > 0");
  tt::mlp::InferParams p;
  std::memset(&p, 0, sizeof(p));
  p.nsets = 1;
  tt::mlp::RaySet& r = p.sets[0];
  r.o = rays;
  r.d = rays + 3;
  r.stride = 6;
  r.out0 = out;
  r.out1 = out + 1;
  r.ostride = 2;
  r.n = n;
  r.tile_begin = 0;
  p.ntiles = (n + tt::mlp::kTileRows - 1) / tt::mlp::kTileRows;
  return mlp_infer(h, net, p, 0.f, 0.f, INFINITY, as_stream(stream));
}

int tt_mlp_intervals(tt_tracer* h, const tt_mlp* net, const tt_view* views, int n_views, float* const* intervals,
                     float margin_near, float margin_far, float far_cap, void* stream) {
  TT_RANGE();
  if (!h) return TT_ERR_INVALID;
  int rc = check_mlp(h, net);
  if (rc != TT_OK) return rc;
  TT_REQUIRE(h, views && intervals && n_views >= 1 && n_views <= tt::mlp::kMaxViews, "need 1..32 views");
  tt::mlp::InferParams p;
  std::memset(&p, 0, sizeof(p));
  long long tiles = 0;
  for (int i = 0; i < n_views; ++i) {
    const tt_view& v = views[i];
    TT_REQUIRE(h, v.H > 0 && v.W > 0 && v.ray_o && v.ray_d && intervals[i], "view needs H, W > 0, rays and an interval");
    TT_REQUIRE(h, (long long)v.H * v.W < (1ll << 31), "too many rays in a view");
    tt::mlp::RaySet& r = p.sets[i];
    r.n = v.H * v.W;
    r.o = v.ray_o;
    r.d = v.ray_d;
    r.stride = 3;
    r.out0 = intervals[i];
    r.out1 = intervals[i] + r.n;
    r.ostride = 1;
    r.tile_begin = (int)tiles;
    tiles += (r.n + tt::mlp::kTileRows - 1) / tt::mlp::kTileRows;
  }
  TT_REQUIRE(h, tiles < (1ll << 30), "too many rays");
  p.nsets = n_views;
  p.ntiles = (int)tiles;
  return mlp_infer(h, net, p, margin_near, margin_far, far_cap, as_stream(stream));
}

// ---------------------------------------------------------------- secondary rays
static int check_secondary(tt_tracer* h, const tt_secondary* sec, int P) {
  TT_REQUIRE(h, sec != nullptr, "null secondary-ray description");
  TT_REQUIRE(h, h->cfg.variant == TT_VARIANT_PLAIN, "secondary-ray passes need the plain program");
  TT_REQUIRE(h, sec->max_depth >= 0 && sec->max_depth <= TT_MAX_BOUNCES, "max_depth must be in [0, 2]");
  TT_REQUIRE(h, sec->env && sec->env_h > 0 && sec->env_w > 0, "need an environment map [env_h][env_w][3]");
  TT_REQUIRE(h, P == 0 || (sec->material && sec->ior), "need material and ior per triangle");
  return TT_OK;
}

static void sec_layout(tt::SecParams& sp, const tt_secondary* sec, tt::SecRecord* rec, int R, int* count) {
  sp.material = sec->material;
  sp.ior = sec->ior;
  sp.env = sec->env;
  sp.env_h = sec->env_h;
  sp.env_w = sec->env_w;
  sp.max_depth = sec->max_depth;
  sp.rec = rec;
  sp.count = count;
  sp.d_env = nullptr;  // the adjoint sets its optional material gradients itself
  sp.d_ior = nullptr;
  for (int l = 0; l <= tt::kMaxSecDepth; ++l) sp.bwd_order[l] = nullptr;
  for (int l = 0; l <= tt::kMaxSecDepth; ++l) {
    sp.base[l] = R * ((1 << l) - 1);
    sp.cap[l] = R << l;
  }
}

int tt_forward_secondary(tt_tracer* h, const tt_fwd_args* a, const tt_secondary* sec, void* stream) {
  TT_RANGE();
  if (!h) return TT_ERR_INVALID;
  if (!a) return fail(h, TT_ERR_INVALID, "null argument block");
  int rc = check_secondary(h, sec, a->P);
  if (rc != TT_OK) return rc;
  TT_REQUIRE(h, a->H > 0 && a->W > 0, "ray_o must be [H, W, 3] with H, W > 0");
  TT_REQUIRE(h, a->ray_o && a->ray_d && a->out_color && a->out_others, "null ray or output pointer");
  TT_REQUIRE(h, a->P == 0 || (a->opacities && a->sigma && a->scaling && a->density_factor && a->max_blending &&
                              a->num_points),
             "null per-triangle pointer");
  rc = check_sh(h, a->shs, a->sh_degree, a->M, a->P);
  if (rc != TT_OK) return rc;
  const long long R = (long long)a->H * a->W;
  const long long nrec = R * ((2ll << sec->max_depth) - 1);
  TT_REQUIRE(h, nrec < (1ll << 31), "too many rays for the secondary-ray queue");
  const cudaStream_t s = as_stream(stream);
  tt::TraceParams p = base_params(h);
  tt_view v;
  std::memset(&v, 0, sizeof(v));
  v.H = a->H;
  v.W = a->W;
  v.ray_o = a->ray_o;
  v.ray_d = a->ray_d;
  v.out_color = a->out_color;
  v.out_others = a->out_others;
  rc = add_view(h, p, v);
  if (rc != TT_OK) return rc;
  rc = accel_step(h, a->vertices, a->num_vertices, a->cumsum, a->P, a->rebuild_gas, s);
  if (rc != TT_OK) return rc;
  TT_CUDA(h, h->sec_rec.reserve((size_t)nrec * sizeof(tt::SecRecord)));
  // hit cache of the ray tree: each pixel's primary ray in the main part,
  // spawned rays and later queries in a pool of two entries per pixel
  const size_t cache_bytes =
      tt::hit_cache_main_bytes(tt::kChunk, R) + (size_t)(tt::kChunk + 2) * 8 * (size_t)(2 * R);
  h->sec_cache_bytes = 0;
  TT_CUDA(h, h->sec_cache.reserve(cache_bytes));
  h->sec_cache_bytes = cache_bytes;
  p.hit_cache = h->sec_cache.p;
  p.cache_mode = tt::kCacheWrite;
  p.cache_gen = h->bvh_gen;
  p.cache_pool_cap = (uint32_t)cache_pool_cap(tt::kChunk, R, cache_bytes);
  TT_CUDA(h, cudaMemsetAsync(h->sec_cache.p, 0, sizeof(tt::HitCacheHeader), s));
  p.bvh = h->bvh.view();
  p.verts = a->vertices;
  p.cumsum = a->cumsum;
  p.num_points = a->num_points;
  p.shs = a->shs;
  p.sh_degree = a->sh_degree;
  p.M = a->M;
  p.opac = a->opacities;
  p.sigma = a->sigma;
  p.bg = a->bg;
  p.scaling = a->scaling;
  p.density = a->density_factor;
  p.max_blending = a->max_blending;
  int* count = reinterpret_cast<int*>(h->scratch.as<char>() + kSecCountOffset);
  sec_layout(p.sec, sec, h->sec_rec.as<tt::SecRecord>(), (int)R, count);
  h->sec_depth = -1;  // no valid tree until this call's launches are enqueued
  if (a->P > 0) TT_CUDA(h, cudaMemsetAsync(a->max_blending, 0, (size_t)a->P * sizeof(float), s));
  TT_CUDA(h, cudaMemsetAsync(count, 0, (tt::kMaxSecDepth + 1) * sizeof(int), s));
  uint32_t *keys = nullptr, *vals = nullptr, *keys2 = nullptr, *vals2 = nullptr, *hist = nullptr;
  if (h->sort_secondary && sec->max_depth > 0) {
    const long long cap = R << sec->max_depth;  // the deepest level's capacity
    const size_t hw = tt::sort_pairs_hist_words((int)cap);
    TT_CUDA(h, h->sec_sort.reserve((size_t)(4 * cap) * 4 + hw * 4));
    TT_CUDA(h, h->sec_order.reserve((size_t)((2ll << sec->max_depth) - 2) * R * 4));  // levels 1..max_depth
    keys = h->sec_sort.as<uint32_t>();
    vals = keys + cap;
    keys2 = vals + cap;
    vals2 = keys2 + cap;
    hist = vals2 + cap;
  }
  if (a->debug) TT_CUDA(h, cudaEventRecord(h->ev0, s));
  for (int level = 0; level <= sec->max_depth; ++level) {
    p.sec.level = level;
    p.sec.order = nullptr;
    if (level > 0 && keys) {
      // trace the spawned rays in (direction bin, origin Morton code) order
      bool second = false;
      TT_CUDA(h, tt::launch_sec_sort_keys(p, keys, vals, s));
      TT_CUDA(h, tt::sort_pairs(keys, vals, keys2, vals2, hist, p.sec.cap[level], 32, &second, s));
      p.sec.order = second ? vals2 : vals;
      h->trace_launches += 1 + tt::sort_pairs_launches(p.sec.cap[level], 32);
      // the adjoint takes the level's rays in the same order
      TT_CUDA(h, cudaMemcpyAsync(h->sec_order.as<uint32_t>() + (size_t)(p.sec.base[level] - R), p.sec.order,
                                 (size_t)p.sec.cap[level] * 4, cudaMemcpyDeviceToDevice, s));
    }
    p.cache_mode = tt::kCacheWrite;
    if (h->split_forward) {
      // traversal-only pass over the level (the primary rays as warp
      // packets of 16-hit queries, like k_sec_primary; spawned rays lane by
      // lane), then the shading pass replays it
      TT_CUDA(h, cudaMemsetAsync(p.work, 0, sizeof(int), s));
      if (level == 0) {
        tt::TraceParams q = p;
        q.cfg = tt::kCfgPackets16;
        q.collect_queries = h->collect_queries;
        TT_CUDA(h, tt::launch_collect(q, h->sec_collect0_grid, s));
      } else {
        TT_CUDA(h, tt::launch_sec_collect(p, h->sec_collect_grid, s));
      }
      ++h->trace_launches;
      p.cache_mode = tt::kCacheFill;
    }
    TT_CUDA(h, cudaMemsetAsync(p.work, 0, sizeof(int), s));
    TT_CUDA(h, level == 0 ? tt::launch_sec_primary(p, h->sec_primary_grid, s)
                          : tt::launch_sec_trace(p, h->sec_trace_grid, s));
    ++h->trace_launches;
  }
  for (int level = sec->max_depth; level >= 0; --level) {
    p.sec.level = level;
    TT_CUDA(h, tt::launch_sec_resolve(p, s));
    ++h->trace_launches;
  }
  if (a->debug) {
    TT_CUDA(h, cudaEventRecord(h->ev1, s));
    TT_CUDA(h, cudaEventSynchronize(h->ev1));
    float ms = 0.f;
    TT_CUDA(h, cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    if (a->gpu_time_ms) *a->gpu_time_ms = ms;
  }
  h->sec_R = (int)R;
  h->sec_depth = sec->max_depth;
  h->sec_sorted = keys != nullptr;
  return TT_OK;
}

int tt_secondary_tree(tt_tracer* h, void* dst, unsigned long long dst_bytes, int* counts, void* stream) {
  if (!h) return TT_ERR_INVALID;
  TT_REQUIRE(h, counts != nullptr, "null counts");
  if (h->sec_depth < 0) return fail(h, TT_ERR_STATE, "no secondary-ray forward on this handle");
  const cudaStream_t s = as_stream(stream);
  int dev_counts[tt::kMaxSecDepth + 1] = {0, 0, 0};
  TT_CUDA(h, cudaMemcpyAsync(dev_counts, h->scratch.as<char>() + kSecCountOffset, sizeof(dev_counts),
                             cudaMemcpyDeviceToHost, s));
  const unsigned long long total =
      (unsigned long long)h->sec_R * ((2ull << h->sec_depth) - 1) * sizeof(tt::SecRecord);
  if (dst && dst_bytes)
    TT_CUDA(h, cudaMemcpyAsync(dst, h->sec_rec.p, dst_bytes < total ? dst_bytes : total, cudaMemcpyDeviceToDevice, s));
  TT_CUDA(h, cudaStreamSynchronize(s));
  counts[0] = h->sec_R;
  for (int l = 1; l <= tt::kMaxSecDepth; ++l) counts[l] = l <= h->sec_depth ? dev_counts[l] : 0;
  return TT_OK;
}

int tt_backward_secondary(tt_tracer* h, const tt_bwd_args* a, const tt_secondary* sec, void* stream) {
  TT_RANGE();
  if (!h) return TT_ERR_INVALID;
  if (!a) return fail(h, TT_ERR_INVALID, "null argument block");
  int rc = check_secondary(h, sec, a->P);
  if (rc != TT_OK) return rc;
  TT_REQUIRE(h, a->H > 0 && a->W > 0, "ray_o must be [H, W, 3] with H, W > 0");
  TT_REQUIRE(h, a->ray_o && a->ray_d && a->others && a->dL_dpixels && a->dL_dothers,
             "null ray, forward-output or upstream-gradient pointer");
  TT_REQUIRE(h, a->P == 0 || (a->opacities && a->sigma && a->cumsum && a->vertices), "null per-triangle pointer");
  TT_REQUIRE(h, a->P == 0 || (a->dL_dtriangle && a->dL_dsigma && a->dL_dopacity && a->dL_dsh),
             "null gradient output");
  rc = check_sh(h, a->shs, a->sh_degree, a->M, a->P);
  if (rc != TT_OK) return rc;
  if (!h->bvh.built() || h->bvh.P() != a->P) return fail(h, TT_ERR_STATE, "backward before a matching forward");
  if (h->sec_depth != sec->max_depth || h->sec_R != a->H * a->W)
    return fail(h, TT_ERR_STATE, "secondary backward without a matching tt_forward_secondary on this handle");
  const cudaStream_t s = as_stream(stream);
  tt::TraceParams p = base_params(h);
  tt_view v;
  std::memset(&v, 0, sizeof(v));
  v.H = a->H;
  v.W = a->W;
  v.ray_o = a->ray_o;
  v.ray_d = a->ray_d;
  v.colors = a->colors;
  v.others = a->others;
  v.dL_dpixels = a->dL_dpixels;
  v.dL_dothers = a->dL_dothers;
  rc = add_view(h, p, v);
  if (rc != TT_OK) return rc;
  if (a->P > 0) {
    TT_CUDA(h, cudaMemsetAsync(a->dL_dtriangle, 0, (size_t)a->num_vertices * 3 * sizeof(float), s));
    TT_CUDA(h, cudaMemsetAsync(a->dL_dsigma, 0, (size_t)a->P * sizeof(float), s));
    TT_CUDA(h, cudaMemsetAsync(a->dL_dopacity, 0, (size_t)a->P * sizeof(float), s));
    TT_CUDA(h, cudaMemsetAsync(a->dL_dsh, 0, (size_t)a->P * a->M * 3 * sizeof(float), s));
  }
  p.verts = a->vertices;
  p.cumsum = a->cumsum;
  p.num_points = a->num_points;
  p.shs = a->shs;
  p.sh_degree = a->sh_degree;
  p.M = a->M;
  p.opac = a->opacities;
  p.sigma = a->sigma;
  p.bg = a->bg;
  p.d_tri = a->dL_dtriangle;
  p.d_sigma = a->dL_dsigma;
  p.d_opac = a->dL_dopacity;
  p.d_sh = a->dL_dsh;
  int* count = reinterpret_cast<int*>(h->scratch.as<char>() + kSecCountOffset);
  sec_layout(p.sec, sec, h->sec_rec.as<tt::SecRecord>(), h->sec_R, count);
  if (h->sec_sorted)  // the spawned levels in the order the forward traced them
    for (int l = 1; l <= sec->max_depth; ++l)
      p.sec.bwd_order[l] = h->sec_order.as<uint32_t>() + (size_t)(p.sec.base[l] - h->sec_R);
  if (sec->dL_denv) {
    p.sec.d_env = sec->dL_denv;
    TT_CUDA(h, cudaMemsetAsync(sec->dL_denv, 0, (size_t)sec->env_h * sec->env_w * 3 * sizeof(float), s));
  }
  if (sec->dL_dior && a->P > 0) {
    p.sec.d_ior = sec->dL_dior;
    TT_CUDA(h, cudaMemsetAsync(sec->dL_dior, 0, (size_t)a->P * sizeof(float), s));
  }
  if (h->sec_cache_bytes > 0) {  // replayed where its header matches (same BVH generation)
    p.hit_cache = h->sec_cache.p;
    p.cache_mode = tt::kCacheRead;
    p.cache_gen = h->bvh_gen;
    p.cache_pool_cap = (uint32_t)cache_pool_cap(tt::kChunk, p.cache_rays, h->sec_cache_bytes);
  }
  TT_CUDA(h, cudaMemsetAsync(p.work, 0, sizeof(int), s));
  if (a->debug) TT_CUDA(h, cudaEventRecord(h->ev0, s));
  TT_CUDA(h, tt::launch_sec_backward(p, h->sec_bwd_grid, s));
  ++h->trace_launches;
  if (a->debug) {
    TT_CUDA(h, cudaEventRecord(h->ev1, s));
    TT_CUDA(h, cudaEventSynchronize(h->ev1));
    float ms = 0.f;
    TT_CUDA(h, cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    if (a->gpu_time_ms) *a->gpu_time_ms = ms;
  }
  return TT_OK;
}

// ---------------------------------------------------------------- BVH files
int tt_bvh_save(tt_tracer* h, void* dst, unsigned long long capacity, unsigned long long* bytes, void* stream) {
  TT_RANGE();
  if (!h) return TT_ERR_INVALID;
  TT_REQUIRE(h, bytes != nullptr, "null size pointer");
  if (!h->bvh.built() || h->bvh.P() <= 0) return fail(h, TT_ERR_STATE, "no acceleration structure to save");
  size_t n = 0;
  const cudaError_t e = h->bvh.save(dst, (size_t)capacity, &n, as_stream(stream));
  *bytes = n;
  if (e == cudaErrorInvalidValue) return fail(h, TT_ERR_INVALID, "destination buffer too small");
  if (e != cudaSuccess) return cuda_fail(h, e, "bvh save");
  return TT_OK;
}

int tt_bvh_load(tt_tracer* h, const void* src, unsigned long long bytes, const float* vertices, int num_vertices,
                const int* cumsum, int P, void* stream) {
  TT_RANGE();
  if (!h) return TT_ERR_INVALID;
  TT_REQUIRE(h, src && vertices && cumsum && P > 0 && num_vertices >= 3, "need a blob, vertices and cumsum");
  cudaError_t e = cudaSuccess;
  ++h->bvh_gen;
  const int bad = h->bvh.load(src, (size_t)bytes, vertices, cumsum, P, as_stream(stream), &e);
  if (bad == 1) return fail(h, TT_ERR_INVALID, "not a BVH blob for this triangle count");
  if (bad == 2) return fail(h, TT_ERR_INVALID, "corrupted BVH blob: an index or link is out of place");
  if (e != cudaSuccess) return cuda_fail(h, e, "bvh load");
  return TT_OK;
}

}  // extern "C"
