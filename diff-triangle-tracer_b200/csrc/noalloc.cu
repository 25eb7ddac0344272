// tt_forward_noalloc: the forward trace for callers that may not allocate
// device memory.
//
// Who needs it: code that only ever receives the buffers of one call and has
// no way to own memory across calls or to allocate inside the call, e.g. an
// operator plugin of an inference engine (TensorRT, an XLA custom call) whose
// framework hands over inputs, outputs and nothing else, or a renderer whose
// frame loop runs under a fixed device-memory budget. tt_create/tt_build
// allocate the BVH and the scheduler counters with cudaMalloc; this entry
// point instead builds the BVH and runs the persistent forward kernel entirely
// out of one file-scope device array of fixed size.
//
// Limits and behaviour (also stated in include/tritracer.h):
//  * at most TT_NOALLOC_MAX_TRIANGLES triangles; larger scenes are rejected
//    with TT_ERR_TOO_LARGE before anything is enqueued;
//  * the array (kScratchBytes, 4 MiB) exists on every GPU that loads the
//    library, for the life of the process;
//  * the BVH is rebuilt from the given vertices on every call (rebuild_gas is
//    ignored: nothing survives between calls);
//  * every call reuses the same array and it keeps the previous call's
//    contents; whatever must start at zero (counters, arrival flags) is
//    cleared by the call itself. Calls whose work overlaps on the GPU (on
//    different streams, or from several threads without ordering) race on the
//    array and must not be issued;
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (a host-side set-up, done once per device with that
//    device current); make that first call before any stream capture;
//  * `debug` timing is not available here (*gpu_time_ms is set to 0);
//  * with no handle there is no tt_device_status: tt_noalloc_status reads
//    (and clears) the status word the last call's kernels left in the array;
//  * the cached address belongs to the device's primary context: after
//    cudaDeviceReset (or anything else that destroys that context) the
//    address is stale, so this entry point must not be used again in that
//    process.
#include <cstring>
#include <mutex>

#include "../../include/tritracer.h"
#include "bvh.cuh"
#include "trace.cuh"

namespace {

constexpr int kMaxTriangles = TT_NOALLOC_MAX_TRIANGLES;
constexpr size_t kScratchBytes = size_t(4) << 20;
constexpr size_t kCounterBytes = 256;  // tile counter, status word, stats

// The only device memory this path uses besides the caller's buffers. In host
// code `g_noalloc_scratch` names a host-side stand-in, never the device
// array: its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct DeviceSetup {
  bool done = false;
  unsigned char* base = nullptr;  // device address of g_noalloc_scratch
  int grid = 0;
};
constexpr int kMaxDevices = 64;
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mutex;

int setup_current_device(DeviceSetup** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return TT_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  DeviceSetup& s = g_setup[dev];
  if (!s.done) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) return TT_ERR_CUDA;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return TT_ERR_CUDA;
    s.base = static_cast<unsigned char*>(p);
    s.grid = sms * tt::trace_blocks_per_sm(0, tt::kCfgPackets16);
    s.done = true;
  }
  *out = &s;
  return TT_OK;
}

}  // namespace

extern "C" int tt_forward_noalloc(const tt_config* cfg, const tt_fwd_args* a, void* stream) {
  if (!a) return TT_ERR_INVALID;
  const int variant = cfg ? cfg->variant : TT_VARIANT_PLAIN;
  const int tmin_inclusive = cfg ? cfg->tmin_inclusive : 1;
  if (variant != TT_VARIANT_PLAIN) return TT_ERR_INVALID;
  if (a->P < 0 || a->H <= 0 || a->W <= 0 || (long long)a->H * a->W >= (1ll << 31)) return TT_ERR_INVALID;
  if (a->P > kMaxTriangles) return TT_ERR_TOO_LARGE;
  if (tt::bvh_storage_bytes(kMaxTriangles) + kCounterBytes > kScratchBytes) return TT_ERR_TOO_LARGE;
  if (!a->ray_o || !a->ray_d || !a->out_color || !a->out_others || !a->bg) return TT_ERR_INVALID;
  // per-triangle colours in place of SH when shs is NULL, as tt_forward does
  const float* cols = a->shs ? nullptr : a->colors_precomp;
  if (a->P > 0 && (!a->vertices || !a->cumsum || !a->num_points || !a->opacities || !a->sigma || !a->scaling ||
                   !a->density_factor || !a->max_blending || !(a->shs || cols) || a->num_vertices < 3))
    return TT_ERR_INVALID;
  if (!cols && (a->sh_degree < 0 || a->sh_degree > 3 || a->M < (a->sh_degree + 1) * (a->sh_degree + 1)))
    return TT_ERR_INVALID;
  if (a->debug && a->gpu_time_ms) *a->gpu_time_ms = 0.0f;

  DeviceSetup* dev = nullptr;
  int rc = setup_current_device(&dev);
  if (rc != TT_OK) return rc;
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  unsigned char* counters = dev->base + (kScratchBytes - kCounterBytes);
  const tt::BvhStorage st = tt::bvh_storage_carve(dev->base, a->P);

  // counters start at zero; the build kernels initialise their own state
  if (cudaMemsetAsync(counters, 0, kCounterBytes, s) != cudaSuccess) return TT_ERR_CUDA;
  if (tt::bvh_build_into(st, a->vertices, a->cumsum, a->P, s) != cudaSuccess) return TT_ERR_CUDA;
  if (a->P > 0 && cudaMemsetAsync(a->max_blending, 0, (size_t)a->P * sizeof(float), s) != cudaSuccess)
    return TT_ERR_CUDA;

  tt::TraceParams p;
  std::memset(&p, 0, sizeof(p));
  p.bvh = tt::bvh_storage_view(st, a->P);
  p.nviews = 1;
  tt::ViewDesc& v = p.views[0];
  v.ray_o = a->ray_o;
  v.ray_d = a->ray_d;
  v.out_color = a->out_color;
  v.out_others = a->out_others;
  v.H = a->H;
  v.W = a->W;
  v.ntx = (a->W + 7) / 8;
  v.tile_begin = 0;
  p.ntiles = v.ntx * ((a->H + 3) / 4);
  p.verts = a->vertices;
  p.cumsum = a->cumsum;
  p.num_points = a->num_points;
  p.shs = a->shs;
  p.cols = cols;
  p.sh_degree = a->sh_degree;
  p.M = a->M;
  p.opac = a->opacities;
  p.sigma = a->sigma;
  p.bg = a->bg;
  p.scaling = a->scaling;
  p.density = a->density_factor;
  p.max_blending = a->max_blending;
  p.variant = TT_VARIANT_PLAIN;
  p.tmin_inclusive = tmin_inclusive;
  p.cfg = tt::kCfgPackets16;
  p.work = reinterpret_cast<int*>(counters);
  p.status = reinterpret_cast<int*>(counters) + 1;
  p.stats = reinterpret_cast<unsigned long long*>(counters + 16);
  if (tt::launch_forward(p, dev->grid, s) != cudaSuccess) return TT_ERR_CUDA;
  return TT_OK;
}

extern "C" int tt_noalloc_status(void* stream) {
  DeviceSetup* dev = nullptr;
  int rc = setup_current_device(&dev);
  if (rc != TT_OK) return rc;
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  int* word = reinterpret_cast<int*>(dev->base + (kScratchBytes - kCounterBytes)) + 1;
  int st = 0;
  if (cudaMemcpyAsync(&st, word, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) return TT_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return TT_ERR_CUDA;
  if (cudaMemsetAsync(word, 0, sizeof(int), s) != cudaSuccess) return TT_ERR_CUDA;
  if (st & tt::kStatusBounds) return TT_ERR_BOUNDS;
  if (st & tt::kStatusStack) return TT_ERR_STACK;
  if (st & tt::kStatusTimeout) return TT_ERR_TIMEOUT;
  return TT_OK;
}
