// Test infrastructure (oracle): runs the reference's own raygen/any-hit
// programs (tritracer/forward.cu, backward.cu, reflect.cu, refract.cu,
// envlight.cu, compiled for the host from the reference's files by
// ../Makefile) over every pixel, the way optixLaunch(W, H, 1) does in
// tritracer/tracer.cpp:119-120 and :219-220.
//
// optixTrace is implemented with the oracle's FP32 watertight intersector and
// CPU BVH (../accel.hpp): each candidate hit in [tmin, tmax] is handed to the
// module's any-hit program; a candidate it does not ignore shrinks tmax to
// its t, as OptiX does for an accepted hit.
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "../accel.hpp"
#include "../or_args.h"
#include "params.h"

// One raygen/any-hit pair and one launch-parameter block per module; the
// Makefile renames each module's `params`, `__raygen__rg` and `__anyhit__ah`.
#define TT_MODULE(m)                    \
  extern "C" Params ref_##m##_params;   \
  extern "C" void ref_##m##_raygen();   \
  extern "C" void ref_##m##_anyhit();
TT_MODULE(forward)
TT_MODULE(backward)
TT_MODULE(reflect)
TT_MODULE(refract)
TT_MODULE(envlight)
#undef TT_MODULE

namespace {

struct ShimThread {
  unsigned int* pl[32];
  unsigned int prim = 0;
  float t = 0.f;
  bool ignored = false;
  void (*anyhit)() = nullptr;
  uint3 idx, dim;
};
thread_local ShimThread g;
const tto::Scene* g_scene = nullptr;
bool g_tmin_inclusive = true;
const or_args* g_log = nullptr;  // forward calls that log their queries (or_args.chunk_*)

}  // namespace

#define TT_PAYLOAD(n)                                          \
  unsigned int optixGetPayload_##n() { return *g.pl[n]; }     \
  void optixSetPayload_##n(unsigned int v) { *g.pl[n] = v; }
TT_PAYLOAD(0) TT_PAYLOAD(1) TT_PAYLOAD(2) TT_PAYLOAD(3) TT_PAYLOAD(4) TT_PAYLOAD(5) TT_PAYLOAD(6) TT_PAYLOAD(7)
TT_PAYLOAD(8) TT_PAYLOAD(9) TT_PAYLOAD(10) TT_PAYLOAD(11) TT_PAYLOAD(12) TT_PAYLOAD(13) TT_PAYLOAD(14)
TT_PAYLOAD(15) TT_PAYLOAD(16) TT_PAYLOAD(17) TT_PAYLOAD(18) TT_PAYLOAD(19) TT_PAYLOAD(20) TT_PAYLOAD(21)
TT_PAYLOAD(22) TT_PAYLOAD(23) TT_PAYLOAD(24) TT_PAYLOAD(25) TT_PAYLOAD(26) TT_PAYLOAD(27) TT_PAYLOAD(28)
TT_PAYLOAD(29) TT_PAYLOAD(30) TT_PAYLOAD(31)
#undef TT_PAYLOAD

unsigned int optixGetPrimitiveIndex() { return g.prim; }
float optixGetRayTmax() { return g.t; }
void optixIgnoreIntersection() { g.ignored = true; }
uint3 optixGetLaunchIndex() { return g.idx; }
uint3 optixGetLaunchDimensions() { return g.dim; }

#define TT_U unsigned int&
void optixTrace(OptixTraversableHandle, float3 o, float3 d, float tmin, float tmax, float, OptixVisibilityMask,
                unsigned int, unsigned int, unsigned int, unsigned int, TT_U p0, TT_U p1, TT_U p2, TT_U p3, TT_U p4,
                TT_U p5, TT_U p6, TT_U p7, TT_U p8, TT_U p9, TT_U p10, TT_U p11, TT_U p12, TT_U p13, TT_U p14,
                TT_U p15, TT_U p16, TT_U p17, TT_U p18, TT_U p19, TT_U p20, TT_U p21, TT_U p22, TT_U p23,
                TT_U p24, TT_U p25, TT_U p26, TT_U p27, TT_U p28, TT_U p29, TT_U p30, TT_U p31) {
  unsigned int* pl[32] = {&p0,  &p1,  &p2,  &p3,  &p4,  &p5,  &p6,  &p7,  &p8,  &p9,  &p10,
                          &p11, &p12, &p13, &p14, &p15, &p16, &p17, &p18, &p19, &p20, &p21,
                          &p22, &p23, &p24, &p25, &p26, &p27, &p28, &p29, &p30, &p31};
  std::memcpy(g.pl, pl, sizeof(pl));
  const float of[3] = {o.x, o.y, o.z}, df[3] = {d.x, d.y, d.z};
  const tto::RayPre rp = tto::ray_pre(of, df);
  g_scene->for_each_hit(rp, tmin, tmax, g_tmin_inclusive, [&](int prim, float t, float tcur) -> float {
    g.prim = (unsigned int)prim;
    g.t = t;
    g.ignored = false;
    g.anyhit();
    return g.ignored ? tcur : t;
  });
  if (g_log && g_log->chunk_count) {
    // the payload after the trace: 16 (id, t) pairs, ids in the even words
    const size_t pix = (size_t)g.idx.y * g.dim.x + g.idx.x;
    const int c = g_log->chunk_count[pix]++;
    if (c < g_log->max_chunks) {
      const size_t q = pix * (size_t)g_log->max_chunks + (size_t)c;
      g_log->chunk_tmin[q] = tmin;
      for (int i = 0; i < 16; ++i) g_log->chunk_ids[q * 16 + i] = *g.pl[2 * i];
    }
  }
}
#undef TT_U

namespace {

void fill_common(Params& p, const or_args* a) {
  std::memset(&p, 0, sizeof(p));
  p.gas_handle = 1;
  p.width = (unsigned)a->W;
  p.height = (unsigned)a->H;
  p.ray_org = (float3*)a->ray_o;
  p.ray_dir = (float3*)a->ray_d;
  p.P = (unsigned)a->P;
  p.sh_degree = (unsigned)a->sh_degree;
  p.M = (unsigned)a->M;
  p.vertices = (float3*)a->verts;
  p.num_points_per_triangle = (int*)a->num_points;
  p.cumsum_of_points_per_triangle = (int*)a->cumsum;
  p.shs = (float*)a->shs;
  p.opacities = (float*)a->opacities;
  p.sigma = (float*)a->sigma;
  p.bg_color = (float*)a->bg;
  p.extra = (uint8_t*)a->extra;
  p.extra_len = (uint32_t)(a->extra_len * sizeof(float));
}

void launch(const or_args* a, void (*raygen)(), void (*anyhit)()) {
  const int r0 = a->row_begin > 0 ? a->row_begin : 0;
  const int r1 = a->row_end > 0 ? a->row_end : a->H;
  const int nt = a->nthreads > 1 ? a->nthreads : 1;
  auto rows = [&](int t) {
    g.anyhit = anyhit;
    g.dim = make_uint3((unsigned)a->W, (unsigned)a->H, 1u);
    for (int y = r0 + t; y < r1; y += nt)
      for (int x = 0; x < a->W; ++x) {
        g.idx = make_uint3((unsigned)x, (unsigned)y, 0u);
        raygen();
      }
  };
  if (nt == 1) {
    rows(0);
    return;
  }
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t) th.emplace_back(rows, t);
  for (auto& x : th) x.join();
}

}  // namespace

extern "C" {

void* ref_scene_new(const float* verts, const int* cumsum, int P) {
  tto::Scene* s = new tto::Scene();
  s->build(verts, cumsum, P);
  return s;
}

void ref_scene_free(void* s) { delete static_cast<tto::Scene*>(s); }

// trace_fwd's launch (tracer.cpp:16-142) minus the GAS build: `variant`
// selects the raygen module the way Tracer("forward.ptx" | "reflect.ptx" |
// "refract.ptx" | "envlight.ptx", ...) does. Output arrays must be zeroed by
// the caller, as torch::zeros does in the reference.
int ref_forward(void* scene, const or_args* a, float* scaling, float* density, float* color, float* others,
                float* maxb) {
  g_scene = static_cast<tto::Scene*>(scene);
  g_tmin_inclusive = a->tmin_inclusive != 0;
  Params* p = nullptr;
  void (*rg)() = nullptr;
  void (*ah)() = nullptr;
  switch (a->variant) {
    case 0: p = &ref_forward_params; rg = ref_forward_raygen; ah = ref_forward_anyhit; break;
    case 1: p = &ref_reflect_params; rg = ref_reflect_raygen; ah = ref_reflect_anyhit; break;
    case 2: p = &ref_refract_params; rg = ref_refract_raygen; ah = ref_refract_anyhit; break;
    case 3: p = &ref_envlight_params; rg = ref_envlight_raygen; ah = ref_envlight_anyhit; break;
    default: return 1;
  }
  fill_common(*p, a);
  p->scaling = scaling;
  p->density_factor = density;
  p->out_color = color;
  p->out_others = others;
  p->max_blending = maxb;
  g_log = (a->max_chunks > 0 && a->chunk_ids && a->chunk_tmin && a->chunk_count) ? a : nullptr;
  launch(a, rg, ah);
  g_log = nullptr;
  return 0;
}

// trace_bwd's launch (tracer.cpp:144-228); gradient arrays zeroed by the caller.
int ref_backward(void* scene, const or_args* a, float* dtri, float* dsigma, float* dopac, float* dsh) {
  g_scene = static_cast<tto::Scene*>(scene);
  g_tmin_inclusive = a->tmin_inclusive != 0;
  Params& p = ref_backward_params;
  fill_common(p, a);
  p.out_color = (float*)a->colors;
  p.out_others = (float*)a->others;
  p.dL_dpixels = (float*)a->dL_dpixels;
  p.dL_dothers = (float*)a->dL_dothers;
  p.out_dL_dtriangle = dtri;
  p.out_dL_dsigma = dsigma;
  p.out_dL_dopacity = dopac;
  p.out_dL_dsh = dsh;
  launch(a, ref_backward_raygen, ref_backward_anyhit);
  return 0;
}

}  // extern "C"
