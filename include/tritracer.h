/*
 * tritracer.h - C ABI of the B200 differentiable k-closest-hit triangle tracer.
 *
 * Drop-in for the reference's host tracer class `OptixTracer`
 * (tritracer/tracer.h:67-126, bound to Python in ext.cpp:11-27). Every entry
 * point takes plain device pointers and sizes, never framework types, and
 * returns a status code (TT_OK = 0). Work is enqueued on the caller's CUDA
 * stream (`stream`, a cudaStream_t; NULL = legacy default stream) and nothing
 * synchronises unless stated.
 *
 * Data layout (the reference's per-triangle layout, tritracer/params.h:15-62):
 *   vertices   float[num_vertices][3]; triangle i uses vertices cumsum[i],
 *              cumsum[i]+1, cumsum[i]+2
 *   num_points int[P] (3 for every triangle), cumsum int[P] (exclusive prefix sum)
 *   shs        float[P][M][3], coefficient-major, RGB innermost
 *   opacities, sigma, scaling, density_factor, max_blending   float[P]
 *   rays       ray_o, ray_d float[H][W][3]
 *   out_color  float[3][H][W];  out_others float[7][H][W] with channels
 *              0 depth, 1 alpha = 1-T, 2..4 normal, 5 middepth, 6 distortion
 *              (tritracer/config.h:16-20)
 */
#ifndef TRITRACER_H
#define TRITRACER_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. The reference reports failures as C++ exceptions
 * (tritracer/exception.h:16-51); here each call returns one of these and
 * tt_last_error() holds the message. */
#define TT_OK 0
#define TT_ERR_INVALID 1 /* bad argument (shape, pointer, degree, size) */
#define TT_ERR_OOM 2     /* device allocation failed */
#define TT_ERR_TIMEOUT 3 /* a bounded device loop gave up (see tt_device_status) */
#define TT_ERR_STACK 4   /* traversal stack could not make progress */
#define TT_ERR_CUDA 5    /* CUDA runtime error */
#define TT_ERR_STATE 6   /* call order (e.g. trace before any BVH build) */
#define TT_ERR_TOO_LARGE 7 /* more triangles than tt_forward_noalloc's fixed capacity */
#define TT_ERR_BOUNDS 8  /* a device index check failed (library built with TT_BOUNDS_CHECK) */

/* Which raygen program the forward pass runs: the reference selects one by
 * the PTX file handed to OptixTracer (tritracer/pipeline.cpp:289-296). */
#define TT_VARIANT_PLAIN 0    /* forward.cu */
#define TT_VARIANT_REFLECT 1  /* reflect.cu: mirror sphere from extra[0..3] */
#define TT_VARIANT_REFRACT 2  /* refract.cu: glass sphere from extra[0..3] */
#define TT_VARIANT_ENVLIGHT 3 /* envlight.cu: extra[4] cosine samples off the sphere */

/* Acceleration-structure step taken by a forward call (`rebuild_gas` of
 * TracerSettings, diff_tritracer/__init__.py:42; tracer.cpp:56-69). */
#define TT_BUILD 0 /* full rebuild from the vertices */
#define TT_REFIT 1 /* keep the topology, refit boxes to moved vertices */
#define TT_KEEP 2  /* use the structure as is */

typedef struct tt_tracer tt_tracer;

/* How the rays of a warp traverse the BVH. */
#define TT_TRAVERSAL_AUTO 0    /* packets for camera-ordered rays (default) */
#define TT_TRAVERSAL_PACKETS 1 /* a warp traverses its 8x4-pixel tile as one packet */
#define TT_TRAVERSAL_LANES 2   /* every lane traverses its own ray */

typedef struct tt_config {
  int variant;        /* TT_VARIANT_* (default PLAIN) */
  int tmin_inclusive; /* 1 (default): each re-trace starts AT the last hit's t,
                         the closed interval of optixTrace; 0: strictly after */
  int traversal;      /* TT_TRAVERSAL_* */
  int k;              /* hits gathered per traversal: 16 (0 = default) or 32 (packets
                         only); compositing keeps the reference's 16-hit chunks */
  int stack_depth;    /* per-lane traversal stack: 32 (0 = default) or 24 (lanes only) */
  int exact_adjoint;  /* 0 (default): the reference's gradients (backward.cu), whose vertex
                         gradient leaves out how the incenter distance, the hit point and t
                         move; 1: the full chain rule, no gradient through a clamped alpha, and
                         the forward fills the channels the reference leaves at 0: depth
                         (sum w t), middepth (t of the hit after which T <= 0.5) and
                         distortion (sum over hit pairs i < j of w_i w_j (t_i - t_j)^2), all
                         differentiated by the adjoint. No reference counterpart; plain
                         program only (the secondary-ray passes take it for their adjoint
                         without the extra channels, see tt_forward_secondary) */
  int reference_arithmetic; /* 0 (default): each hit's point on its triangle comes from an
                         FP64 ray/plane solve and the window function is evaluated
                         relative to vertex A, which holds ~7 digits of the incircle; 1:
                         the reference's own FP32 arithmetic instead (hit point o + t d,
                         window function on absolute coordinates, every operation
                         rounded in the order of tritracer/common.h:57-114), whose edge
                         distances keep only ~3 digits on small triangles far from the
                         origin. Same semantics either way; 1 reproduces the reference's
                         numbers. Plain program only, not with exact_adjoint */
  int reserved[1];    /* zero */
} tt_config;

/* Arguments of the forward trace: OptixTracer::trace_fwd
 * (tritracer/tracer.h:78-95, tracer.cpp:16-142). All pointers are device
 * pointers except gpu_time_ms. */
typedef struct tt_fwd_args {
  int H, W;
  const float* ray_o;
  const float* ray_d;
  const float* vertices;
  int num_vertices;
  const int* num_points;
  const int* cumsum;
  int P; /* number_of_points: the triangle count (tracer.cpp:43) */
  const float* shs;
  int sh_degree; /* 0..3 */
  int M;         /* coefficients per triangle, >= (sh_degree+1)^2 */
  const float* colors_precomp; /* [P][3] RGB per triangle, used in place of SH when shs is NULL
                                  (the reference accepts it and never reads it, and reads a null
                                  SH pointer in that case); ignored when shs is given */
  const float* opacities;      /* already activated */
  const float* sigma;
  float* scaling;        /* in/out */
  float* density_factor; /* in/out */
  const float* bg;       /* [3] */
  const float* extra;    /* variant parameters [r, cx, cy, cz, samples] */
  int extra_len;         /* floats in extra */
  int rebuild_gas;       /* TT_BUILD / TT_REFIT / TT_KEEP */
  int debug;             /* 1: time the trace with events into *gpu_time_ms (syncs) */
  float* out_color;      /* [3,H,W], fully written */
  float* out_others;     /* [7,H,W], fully written */
  float* max_blending;   /* [P], zeroed then written */
  float* gpu_time_ms;    /* host pointer, may be NULL */
  /* Optional hit cache (plain program; NULL = none; no reference counterpart):
   * 16-byte aligned device memory, rays = H * W (the sum over the views of a
   * batched call). The forward stores every ray's k-closest queries in it:
   * the first ones in a main part, later ones in a pool while it lasts; each
   * stored query takes (k + 1) * 8 bytes of keys (k + 2 in the pool) and 12 * k
   * bytes for its hits' colours, which the warp-packet traversals store and
   * the adjoint reads instead of evaluating the SH again. The minimum size is
   * the main part, 32 + ((k + 1) * 8 + 12 * k) * rays bytes; the pool fills
   * the rest. tt_hit_cache_bytes(h, rays) sizes the pool for a quarter of the
   * rays. A tt_backward given the same cache replays the stored queries
   * instead of traversing the BVH again. tt_forward_noalloc ignores it. */
  void* hit_cache;
  size_t hit_cache_bytes;
} tt_fwd_args;

/* Arguments of the adjoint: OptixTracer::trace_bwd (tritracer/tracer.h:97-114,
 * tracer.cpp:144-228). Gradient outputs are zeroed, then accumulated. */
typedef struct tt_bwd_args {
  int H, W;
  const float* ray_o;
  const float* ray_d;
  const float* bg;
  const float* vertices;
  int num_vertices;
  const float* sigma;
  const int* num_points;
  const int* cumsum;
  const float* colors; /* forward out_color */
  const float* others; /* forward out_others */
  int P;
  const float* shs;
  int sh_degree;
  int M;
  const float* opacities;
  const float* dL_dpixels; /* [3,H,W] */
  const float* dL_dothers; /* [7,H,W]; channels 0 and 2..4 are read */
  const float* scaling;    /* unused by the adjoint, as in the reference */
  int debug;
  float* dL_dtriangle; /* [num_vertices,3] */
  float* dL_dsigma;    /* [P] */
  float* dL_dopacity;  /* [P] */
  float* dL_dsh;       /* [P,M,3] */
  float* gpu_time_ms;  /* host pointer, may be NULL */
  const float* colors_precomp; /* [P][3]: the forward's precomputed colours (shs NULL), or NULL */
  float* dL_dcolors;           /* [P][3] gradient of colors_precomp (zeroed, then accumulated) */
  /* Optional: the hit cache the forward of these rays filled (NULL = re-trace),
   * with the size it had there. It is only replayed if it was written with the
   * handle's current k and ray count, and no build, refit or load of the BVH
   * happened since; otherwise, and for queries the forward could not store,
   * the adjoint traverses as without it. The results are the same either way:
   * a replayed query is the one the adjoint would compute. */
  const void* hit_cache;
  size_t hit_cache_bytes;
} tt_bwd_args;

/* One camera image of a batched call: rays [H][W][3]; the forward writes
 * out_color [3][H][W] / out_others [7][H][W]; the adjoint reads colors /
 * others (forward outputs) and dL_dpixels / dL_dothers. Pointers a call does
 * not use may be NULL. */
typedef struct tt_view {
  int H, W;
  const float* ray_o;
  const float* ray_d;
  float* out_color;
  float* out_others;
  const float* colors;
  const float* others;
  const float* dL_dpixels;
  const float* dL_dothers;
  /* Proposed intervals (plain variant; NULL = none): [2][H][W], per ray the
   * [t_near, t_far] its traversal is clipped to. Hits before t_near are not
   * visited. A ray still unterminated when its hits up to t_far are used up
   * goes on beyond t_far (a continuation); a ray with no hit in its interval
   * is traced again without it. Forward and adjoint of the same rays must get
   * the same intervals. */
  const float* interval;
  /* Forward only (plain variant; NULL = none): [3][H][W], per ray the t of
   * the first and of the last hit the march visited (INFINITY if none) and
   * 1.0 if the ray ended on the transmittance cut-off, else 0.0: the
   * training targets of the proposal network. */
  float* record;
} tt_view;

/* OptixTracer::OptixTracer (tritracer/pipeline.cpp:267-302). `cfg` may be
 * NULL for the defaults. Uses the CUDA device current at the call. */
int tt_create(const tt_config* cfg, tt_tracer** out);

/* OptixTracer::~OptixTracer (tritracer/pipeline.cpp:322-326). */
int tt_destroy(tt_tracer* h);

/* OptixTracer::build_tri_accel (tritracer/pipeline.cpp:206-265) together with
 * the index-buffer set-up of tracer.cpp:53-69: mode TT_BUILD builds, TT_REFIT
 * refits the existing structure to moved vertices, TT_KEEP does nothing. */
int tt_build(tt_tracer* h, const float* vertices, int num_vertices, const int* cumsum, int P, int mode,
             void* stream);

/* OptixTracer::trace_fwd (tritracer/tracer.cpp:16-142). Runs the
 * acceleration-structure step `a->rebuild_gas` first. */
int tt_forward(tt_tracer* h, const tt_fwd_args* a, void* stream);

/* OptixTracer::trace_bwd (tritracer/tracer.cpp:144-228). Re-traces with the
 * structure of the last forward/build call. */
int tt_backward(tt_tracer* h, const tt_bwd_args* a, void* stream);

/* Batched forms of tt_forward / tt_backward, no reference counterpart (the
 * reference traces one [H, W] image per call): up to 32 views of uneven
 * resolution go through ONE persistent launch; the per-view fields of `a`
 * (H, W, ray and image pointers) are ignored, the per-triangle outputs
 * (scaling, density_factor, max_blending; gradients) accumulate over all
 * views. The view list travels in the kernel's parameters, so the call can be
 * captured in a CUDA graph (plain variant, debug = 0). */
int tt_forward_views(tt_tracer* h, const tt_fwd_args* a, const tt_view* views, int n_views, void* stream);
int tt_backward_views(tt_tracer* h, const tt_bwd_args* a, const tt_view* views, int n_views, void* stream);

/* Switches the traversal configuration of a live handle (the BVH is kept);
 * used by the autotuner. No reference counterpart. */
int tt_set_traversal(tt_tracer* h, int traversal, int k, int stack_depth);

/* Execution options of a handle (no reference counterpart); none changes a
 * result, only how the work is scheduled.
 * TT_OPT_SPLIT_FORWARD, 1 (default): a plain forward given a hit cache runs
 *   as two kernels, a traversal-only pass that makes every k-closest query
 *   of each ray's march and stores it in the cache, then a shading pass that
 *   replays them. The first needs far fewer registers, so more warps hide
 *   the latency of the node and triangle loads. 0: one fused kernel that
 *   traverses and shades.
 * TT_OPT_SORT_SECONDARY, 1 (default): the secondary-ray passes trace each
 *   level of spawned rays in order of direction (octahedral bins) and origin (Morton
 *   code), after a radix sort of the level, so the rays of a warp cross
 *   nearly the same BVH nodes. 0: in the order they were spawned.
 * TT_OPT_COLLECT_QUERIES, n >= 0 (default 2): the traversal-only pass of the
 *   split forward stores at most n k-closest queries per ray (0: every query
 *   of the march, also those past the point where the ray's transmittance
 *   would end it, which that pass cannot know); the shading pass traverses
 *   for the queries not stored. pool_used of tt_hit_cache_usage counts the
 *   pool entries both passes asked for: with a cap of 1 the later queries of
 *   the shading pass's march; otherwise also those the traversal-only pass
 *   made past a ray's cut-off, and a query it was refused counts again when
 *   the shading pass asks for it.
 * TT_OPT_WORK_COUNTERS, 0 (default): 1 makes the traversal kernels count
 *   their node visits and triangle tests into tt_stats (node_visits,
 *   triangle_tests, packet_node_visits; they stay 0 otherwise). The counts
 *   cost the packet traversal a shared-memory update per node visit, about
 *   4 % of its time, so they are off unless asked for. */
/* Device time of the two passes of the last forward on the handle that ran
 * with `debug` (events, as gpu_time_ms): the traversal-only pass (0 for a
 * fused forward) and the shading pass. No reference counterpart. */
int tt_forward_pass_times(tt_tracer* h, float* collect_ms, float* shade_ms);

#define TT_OPT_SPLIT_FORWARD 1
#define TT_OPT_SORT_SECONDARY 2
#define TT_OPT_COLLECT_QUERIES 3
#define TT_OPT_WORK_COUNTERS 4
int tt_set_option(tt_tracer* h, int option, int value);

/* Bytes of a hit cache (tt_fwd_args.hit_cache) for `rays` rays under the
 * handle's current traversal configuration, with a pool for later queries of
 * a quarter of the rays: tt_hit_cache_bytes_pool(h, rays, ceil(rays / 4)).
 * No reference counterpart. */
size_t tt_hit_cache_bytes(const tt_tracer* h, long long rays);

/* Bytes of a hit cache for `rays` rays whose pool holds `pool_queries` later
 * queries under the handle's current traversal configuration:
 * 32 + ((k + 1) * 8 + 12 * k) * rays + ((k + 2) * 8 + 12 * k) * pool_queries. No reference
 * counterpart. */
size_t tt_hit_cache_bytes_pool(const tt_tracer* h, long long rays, long long pool_queries);

/* Reads the header of a hit cache that a forward has filled, after
 * synchronising `stream`. It gives the hits per query `k` the cache was laid
 * out for, the pool's capacity, and the later queries the forward asked the
 * pool for. The last count can pass the capacity: those queries were not
 * stored and the adjoint traverses again for them. A ray stops asking after
 * its first refusal, so after an overflow the count is a lower bound.
 * Returns TT_ERR_INVALID if no forward wrote the cache. No reference
 * counterpart. */
int tt_hit_cache_usage(tt_tracer* h, const void* hit_cache, void* stream, int* k, long long* pool_cap,
                       long long* pool_used);

/* A pinhole camera whose rays tt_camera_rays writes. Pixel (x, y) of its
 * H x W image starts at `origin` and looks along normalize(forward + u right +
 * v up), u = (2 (x + 0.5) / W - 1) t (W / H), v = (1 - 2 (y + 0.5) / H) t,
 * t = tan_half_fov (half the vertical field of view), each step an FP64
 * operation in that order, the result rounded to FP32. ray_o / ray_d:
 * [H][W][3] float32 on the device. */
typedef struct tt_camera {
  double origin[3];
  double forward[3];
  double right[3];
  double up[3];
  double tan_half_fov;
  int H, W;
  float* ray_o;
  float* ray_d;
} tt_camera;

/* Writes the rays of 1 to 32 cameras in one launch on `stream`; capturable
 * in a CUDA graph. This is the caller's side of the path: the reference takes
 * ray tensors (tritracer/tracer.cpp:36-37) and leaves generating them to the
 * training code. No reference counterpart. */
int tt_camera_rays(tt_tracer* h, const tt_camera* cams, int n_cams, void* stream);

/* Message of the last failed call on this handle (never NULL). */
const char* tt_last_error(const tt_tracer* h);

/* Synchronises `stream` and returns the device-side status word of the
 * handle's kernels since the last call (TT_OK, TT_ERR_TIMEOUT, TT_ERR_STACK,
 * TT_ERR_STATE when an adjoint that found its hit cache complete still met a
 * query missing from it, or, in a TT_BOUNDS_CHECK build, TT_ERR_BOUNDS),
 * then clears it. No reference counterpart: the reference's
 * device code has no bounded loops to report on. */
int tt_device_status(tt_tracer* h, void* stream);

/* Counters of the handle's forward kernels since the last tt_reset_stats (no
 * reference counterpart; the reference reports only gpu_time). Evaluated hits
 * are hits at or beyond the near plane whose window function was computed;
 * blended hits are those composited; node visits (per ray), triangle tests and
 * queries (k-closest traversals) describe the traversal work (node visits and
 * triangle tests only with TT_OPT_WORK_COUNTERS on). kernel_launches counts
 * every kernel this handle enqueued (BVH steps included). */
typedef struct tt_stats {
  unsigned long long rays;
  unsigned long long evaluated_hits;
  unsigned long long blended_hits;
  unsigned long long kernel_launches;
  unsigned long long node_visits;
  unsigned long long triangle_tests;
  unsigned long long queries;
  unsigned long long packet_node_visits; /* node visits counted once per warp packet */
  unsigned long long interval_continuations; /* rays that went on beyond their proposed t_far */
  unsigned long long interval_retraces;      /* rays traced again: no hit in their interval */
  unsigned long long hit_cache_replays;      /* adjoint queries replayed from a hit cache */
} tt_stats;

/* Synchronises `stream`, then fills *out. */
int tt_get_stats(tt_tracer* h, tt_stats* out, void* stream);

/* Zeroes the counters (asynchronously on `stream`). */
int tt_reset_stats(tt_tracer* h, void* stream);

/* Serialised acceleration structure (no reference counterpart: OptiX's GAS
 * is rebuilt by every process). tt_bvh_save writes the handle's BVH
 * topology (Morton order, binary and 8-wide hierarchies; not the triangle
 * records or boxes) into the host buffer dst and its size into *bytes; with
 * dst == NULL it only reports the size. It synchronises `stream`.
 * tt_bvh_load restores such a blob into a handle and refits it to the given
 * vertices (the same triangles, moved or not): the result equals a build
 * followed by refits. A blob for another triangle count, or a damaged one,
 * gives TT_ERR_INVALID. */
int tt_bvh_save(tt_tracer* h, void* dst, unsigned long long capacity, unsigned long long* bytes, void* stream);
int tt_bvh_load(tt_tracer* h, const void* src, unsigned long long bytes, const float* vertices, int num_vertices,
                const int* cumsum, int P, void* stream);

/* Test hook, no reference counterpart: the first `max_hits` triangle hits of
 * each of R rays in [0, 1000], ordered by (t, primitive index), found by the
 * same chunked traversal the trace kernels use. ids/ts are [R][max_hits]
 * device arrays, counts [R] receives each ray's total hit count. */
int tt_hit_stream(tt_tracer* h, const float* ray_o, const float* ray_d, int R, int max_hits, uint32_t* ids,
                  float* ts, int* counts, void* stream);

/* ---------------------------------------------------------------------------
 * Proposal network (no reference counterpart). A small MLP maps each ray to
 * the interval [t_near, t_far] holding the hits its march visits; the trace
 * is clipped to it through tt_view.interval. The ray origin o is first
 * moved along the ray to the closest approach of the ray's line to `center`
 * (o' = o + s d, s = -(o - center).d / d.d), so the inputs depend on the line
 * only. Inputs (80): (o' - center) * origin_scale and the direction, sin and
 * cos of 2^k pi x over those 6 coordinates for k = 0..5, a constant 1 and a
 * zero. Layers: 80 -> 64 -> 64 -> 64 (ReLU, each output again followed by a
 * constant-1 input) -> 16, of which outputs 0 and 1 are
 * (t_near - s - t_shift) / t_scale and (t_far - s - t_shift) / t_scale.
 * Every layer runs on the tensor cores (BF16 operands, FP32 accumulation).
 *
 * The arrays are device memory owned by the caller:
 *   master, adam_m, adam_v  float[TT_MLP_PARAMS]: W1 [64][80], W2 [64][80],
 *       W3 [64][80], W4 [16][80] row-major, one after the other; the bias of
 *       each layer is the column fed by the constant 1 (column 78 of W1,
 *       column 64 of W2..W4). Columns fed by a zero and rows 2..15 of W4 are
 *       never updated and must start at 0.
 *   weights  uint16[TT_MLP_PARAMS]: the BF16 copy in the kernels' tensor-core
 *       layout, written by tt_mlp_update and by every training step.
 *   partial  float[partial_ctas][TT_MLP_PARTIAL]: training scratch; a step
 *       uses ceil(n / 128 / ceil(n / 128 / SMs)) CTAs (128 for n = 65536 on
 *       148 SMs).
 * Status: bounded device waits report through tt_device_status(h). */
#define TT_MLP_PARAMS 16640
#define TT_MLP_PARTIAL 16656
typedef struct tt_mlp {
  uint16_t* weights;
  float* master;
  float* adam_m;
  float* adam_v;
  float* partial;
  int partial_ctas;
  float origin_scale; /* closest-approach origins are multiplied by this before encoding */
  float t_shift;      /* t = output * t_scale + t_shift + s */
  float t_scale;
  float center[3];    /* scene centre */
} tt_mlp;

/* One Adam step on a batch. Loss per ray: w0 e0^2 + w1 e1^2 on the scaled
 * outputs, e = output - target, averaged over the batch; w0 = near_weight if
 * t_near is above its target (hits would be cut off), 1 below, 0 for a ray
 * whose t_near target is negative (no hit); w1 = far_weight if t_far is below
 * its target (the ray would need a continuation), else 1. */
typedef struct tt_mlp_step {
  float lr, beta1, beta2, eps;
  int step; /* 1-based, for Adam's bias correction */
  float near_weight;
  float far_weight;
} tt_mlp_step;

/* master -> weights (after initialising or loading master). */
int tt_mlp_update(tt_tracer* h, const tt_mlp* net, void* stream);
/* rays [n][6] (origin, direction), targets [n][2] (t_near, t_far; t_near < 0
 * for a ray without hits), device pointers; *loss (device float, may be
 * NULL) receives the batch's mean loss. */
int tt_mlp_train_step(tt_tracer* h, const tt_mlp* net, const tt_mlp_step* st, const float* rays,
                      const float* targets, int n, float* loss, void* stream);
/* Raw predictions: out [n][2] = (t_near, t_far) for rays [n][6]. */
int tt_mlp_predict(tt_tracer* h, const tt_mlp* net, const float* rays, int n, float* out, void* stream);
/* Proposed intervals for the rays of up to 32 views (ray_o / ray_d of each
 * view; other view fields ignored): intervals[i] is [2][H][W] of view i,
 * [t_near - margin_near, t_far + margin_far], with t_far = +inf when
 * t_far + margin_far - s >= far_cap (far_cap is measured from the ray's
 * closest approach to the centre). */
int tt_mlp_intervals(tt_tracer* h, const tt_mlp* net, const tt_view* views, int n_views, float* const* intervals,
                     float margin_near, float margin_far, float far_cap, void* stream);

/* ---------------------------------------------------------------------------
 * Secondary-ray passes (no reference counterpart: the reference bends rays
 * only at the analytic sphere of its reflect/refract/envlight programs).
 * Per pixel a tree of rays, traced level by level from a device ray queue
 * owned by the handle: the first blended hit of a ray of depth < max_depth on
 * a triangle with material[prim] == 1 (a dielectric interface with index of
 * refraction ior[prim]) spawns a reflected and, unless totally reflected, a
 * refracted ray from the exact hit point, and that hit's colour is
 * F L(reflected) + (1 - F) L(refracted) (Schlick's Fresnel term) instead of
 * its SH colour. Every other hit shades as in tt_forward. A ray's
 * transmittance left at the end sees the lat-long environment map env
 * (longitude atan2(d.z, d.x) over the columns, colatitude acos(d.y) over the
 * rows, bilinear) in place of bg. out_color = radiance of the primary ray;
 * out_others, density_factor, scaling and max_blending come from the primary
 * rays only. The adjoint differentiates every ray of the tree with the spawn
 * geometry (directions, F) held constant, and uses the ray tree of the last
 * tt_forward_secondary on the handle (same rays, scene and max_depth). With
 * tt_config.exact_adjoint it applies the full chain rule of the window
 * function and face normal (no gradient through a clamped alpha) to the
 * outputs the passes compute; depth, middepth and distortion stay 0 here,
 * so their upstream gradients are ignored. Only the spawning triangles'
 * vertex gradients then still hold the spawn geometry constant.
 * One view per call (H, W, rays and outputs of the argument block). */
#define TT_MAX_BOUNCES 2
typedef struct tt_secondary {
  const int* material; /* [P]: 1 = dielectric interface, 0 = plain */
  const float* ior;    /* [P] */
  const float* env;    /* [env_h][env_w][3] */
  int env_h, env_w;
  int max_depth;       /* 0..TT_MAX_BOUNCES */
  /* tt_backward_secondary only, optional (NULL: not computed; the forward
   * ignores both): dL/d(env) [env_h][env_w][3] and dL/d(ior) [P], overwritten.
   * The IOR gradient goes through Schlick's Fresnel share F of each spawning
   * hit; the bent directions are held constant, as for every other input. */
  float* dL_denv;
  float* dL_dior;
} tt_secondary;
int tt_forward_secondary(tt_tracer* h, const tt_fwd_args* a, const tt_secondary* s, void* stream);
int tt_backward_secondary(tt_tracer* h, const tt_bwd_args* a, const tt_secondary* s, void* stream);
/* Test hook: synchronises `stream`, writes the number of rays of each level
 * of the last tt_forward_secondary into counts[0..2] (host) and copies up to
 * dst_bytes of its 64-byte ray records (level 0 first, each level's records
 * at offset R * (2^level - 1)) into dst (device). */
int tt_secondary_tree(tt_tracer* h, void* dst, unsigned long long dst_bytes, int* counts, void* stream);

/* Forward trace that allocates nothing. No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc: an operator plugin that only
 * receives the input and output buffers of each call from its host framework
 * (a TensorRT plugin, an XLA custom call), or a frame loop held to a fixed
 * device-memory budget. It needs no handle: every call builds the BVH over
 * the given triangles and runs the plain forward trace using one fixed,
 * file-scope device array (4 MiB on every GPU that loads this library, for
 * the life of the process) instead of allocated memory. The caller passes the
 * inputs and outputs as in tt_forward (SH, or colors_precomp with shs NULL);
 * the results match tt_forward's.
 *
 * Limits: at most TT_NOALLOC_MAX_TRIANGLES triangles (else TT_ERR_TOO_LARGE,
 * nothing enqueued); plain variant only (cfg may be NULL for the defaults);
 * rebuild_gas is ignored (nothing persists between calls); debug timing is
 * not available (*gpu_time_ms is set to 0). All calls share the one array:
 * calls that overlap on the GPU race and must not be issued. The first call
 * on each device looks the array's address up once (host-side set-up, with
 * that device current); make it before any stream capture. That address
 * belongs to the device's primary context: do not use this entry point again
 * after cudaDeviceReset. With no handle there is no tt_last_error or
 * tt_device_status; an invalid argument returns TT_ERR_INVALID without a
 * message, and device-side failures are read with tt_noalloc_status. */
#define TT_NOALLOC_MAX_TRIANGLES 8192
int tt_forward_noalloc(const tt_config* cfg, const tt_fwd_args* a, void* stream);

/* Status of the last tt_forward_noalloc on the current device, for that
 * handle-free entry point what tt_device_status is for a handle: synchronises
 * `stream`, returns TT_OK, or TT_ERR_TIMEOUT / TT_ERR_STACK if a bounded
 * device loop of that call gave up (its rays were cut short), or
 * TT_ERR_BOUNDS from a TT_BOUNDS_CHECK build, and clears the word. Read it
 * after a call and before the next one, which clears it again. Allocates
 * nothing. No counterpart in the reference. */
int tt_noalloc_status(void* stream);

#ifdef __cplusplus
}
#endif

#endif /* TRITRACER_H */
