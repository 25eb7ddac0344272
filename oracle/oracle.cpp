// Test infrastructure (oracle): C entry points over oracle.hpp, loaded with
// ctypes by the tests, the smoke check and the benchmark's CPU baseline leg.
// See oracle.hpp for what is restated from where, and its parity status.
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "or_args.h"
#include "oracle.hpp"

using namespace tto;



extern "C" void* or_scene_new(const float* verts, const int* cumsum, int P) {
  Scene* s = new Scene();
  s->build(verts, cumsum, P);
  return s;
}

extern "C" void or_scene_free(void* s) { delete static_cast<Scene*>(s); }

static Inputs to_inputs(const or_args* a) {
  Inputs in;
  in.H = a->H;
  in.W = a->W;
  in.ray_o = a->ray_o;
  in.ray_d = a->ray_d;
  in.verts = a->verts;
  in.num_points = a->num_points;
  in.cumsum = a->cumsum;
  in.P = a->P;
  in.shs = a->shs;
  in.sh_degree = a->sh_degree;
  in.M = a->M;
  in.opacities = a->opacities;
  in.sigma = a->sigma;
  in.bg = a->bg;
  in.extra = a->extra;
  in.extra_len = a->extra_len;
  in.interval = a->interval;
  in.colors = a->precomp;
  return in;
}

static Opts to_opts(const or_args* a, bool fp64) {
  Opts o;
  o.tmin_inclusive = a->tmin_inclusive != 0;
  o.canonical_ties = a->canonical_ties != 0;
  o.exact_geometry = fp64 && a->exact_geometry != 0;
  o.mt = a->nthreads > 1;
  o.exact_adjoint = fp64 && a->exact_adjoint != 0;
  return o;
}

template <class Fn>
static void parallel_rows(const or_args* a, Fn&& fn) {
  const int r0 = a->row_begin > 0 ? a->row_begin : 0;
  const int r1 = a->row_end > 0 ? a->row_end : a->H;
  const int nt = a->nthreads > 1 ? a->nthreads : 1;
  if (nt == 1) {
    for (int y = r0; y < r1; ++y)
      for (int x = 0; x < a->W; ++x) fn(y * a->W + x);
    return;
  }
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t) {
    th.emplace_back([&, t]() {
      for (int y = r0 + t; y < r1; y += nt)
        for (int x = 0; x < a->W; ++x) fn(y * a->W + x);
    });
  }
  for (auto& x : th) x.join();
}

template <class R>
static int forward_impl(void* scene, const or_args* a, R* scaling, R* density, R* color, R* others, R* maxb) {
  const Scene& sc = *static_cast<Scene*>(scene);
  const Inputs in = to_inputs(a);
  const Opts opt = to_opts(a, sizeof(R) == 8);
  FwdOut<R> out{scaling, density, color, others, maxb};
  parallel_rows(a, [&](int pix) {
    RayRecord rec;
    RayRecord* rp = nullptr;
    if (a->rec_count) {
      rec.max_rec = a->max_rec;
      rec.ids = a->rec_ids + (size_t)pix * a->max_rec;
      rp = &rec;
    }
    if (a->variant == kPlain)
      forward_ray(sc, in, pix, opt, out, rp);
    else
      variant_ray(sc, in, pix, a->variant, opt, out, rp);
    if (rp) {
      a->rec_count[pix] = rec.count;
      if (a->margin) a->margin[pix] = (float)rec.margin;
    }
  });
  return 0;
}

template <class R>
static int backward_impl(void* scene, const or_args* a, R* dtri, R* dsigma, R* dopac, R* dsh) {
  const Scene& sc = *static_cast<Scene*>(scene);
  const Inputs in = to_inputs(a);
  const Opts opt = to_opts(a, sizeof(R) == 8);
  BwdIn<R> bi{static_cast<const R*>(a->colors), static_cast<const R*>(a->others), a->dL_dpixels, a->dL_dothers};
  BwdOut<R> bo{dtri, dsigma, dopac, dsh, static_cast<R*>(a->dprecomp)};
  parallel_rows(a, [&](int pix) { backward_ray(sc, in, pix, opt, bi, bo); });
  return 0;
}

extern "C" int or_forward_f32(void* s, const or_args* a, float* scaling, float* density, float* color, float* others,
                   float* maxb) {
  return forward_impl<float>(s, a, scaling, density, color, others, maxb);
}
extern "C" int or_forward_f64(void* s, const or_args* a, double* scaling, double* density, double* color, double* others,
                   double* maxb) {
  return forward_impl<double>(s, a, scaling, density, color, others, maxb);
}
extern "C" int or_backward_f32(void* s, const or_args* a, float* dtri, float* dsigma, float* dopac, float* dsh) {
  return backward_impl<float>(s, a, dtri, dsigma, dopac, dsh);
}
extern "C" int or_backward_f64(void* s, const or_args* a, double* dtri, double* dsigma, double* dopac, double* dsh) {
  return backward_impl<double>(s, a, dtri, dsigma, dopac, dsh);
}

static SecInputs to_sec(const or_args* a) {
  SecInputs s;
  s.material = a->material;
  s.ior = a->ior;
  s.env = a->env;
  s.env_h = a->env_h;
  s.env_w = a->env_w;
  s.max_depth = a->max_depth;
  s.ior_fresnel = a->ior_fresnel;
  return s;
}

template <class R>
static int forward_sec_impl(void* scene, const or_args* a, R* scaling, R* density, R* color, R* others, R* maxb) {
  const Scene& sc = *static_cast<Scene*>(scene);
  const Inputs in = to_inputs(a);
  const SecInputs sec = to_sec(a);
  const Opts opt = to_opts(a, sizeof(R) == 8);
  FwdOut<R> out{scaling, density, color, others, maxb};
  parallel_rows(a, [&](int pix) {
    RayRecord rec;
    RayRecord* rp = nullptr;
    if (a->rec_count) {
      rec.max_rec = a->max_rec;
      rec.ids = a->rec_ids + (size_t)pix * a->max_rec;
      rp = &rec;
    }
    sec_radiance<R>(sc, in, sec, in.ray_o + 3 * (size_t)pix, in.ray_d + 3 * (size_t)pix, 0, opt, &out, pix, rp);
    if (rp) {
      a->rec_count[pix] = rec.count;
      if (a->margin) a->margin[pix] = (float)rec.margin;
    }
  });
  return 0;
}

template <class R>
static int backward_sec_impl(void* scene, const or_args* a, R* dtri, R* dsigma, R* dopac, R* dsh) {
  const Scene& sc = *static_cast<Scene*>(scene);
  const Inputs in = to_inputs(a);
  const SecInputs sec = to_sec(a);
  const Opts opt = to_opts(a, sizeof(R) == 8);
  const R* others = static_cast<const R*>(a->others);
  BwdOut<R> bo{dtri, dsigma, dopac, dsh};
  bo.denv = static_cast<R*>(a->denv);
  bo.dior = static_cast<R*>(a->dior);
  const int HW = a->H * a->W;
  parallel_rows(a, [&](int pix) {
    const R gL[3] = {(R)a->dL_dpixels[pix], (R)a->dL_dpixels[HW + pix], (R)a->dL_dpixels[2 * HW + pix]};
    const R go[4] = {(R)a->dL_dothers[kDepth * HW + pix], (R)a->dL_dothers[(kNormal + 0) * HW + pix],
                     (R)a->dL_dothers[(kNormal + 1) * HW + pix], (R)a->dL_dothers[(kNormal + 2) * HW + pix]};
    const R fo[4] = {others[kDepth * HW + pix], others[(kNormal + 0) * HW + pix], others[(kNormal + 1) * HW + pix],
                     others[(kNormal + 2) * HW + pix]};
    sec_backward<R>(sc, in, sec, in.ray_o + 3 * (size_t)pix, in.ray_d + 3 * (size_t)pix, 0, opt, gL, go, fo, bo);
  });
  return 0;
}

extern "C" int or_forward_secondary_f64(void* s, const or_args* a, double* scaling, double* density, double* color,
                                        double* others, double* maxb) {
  return forward_sec_impl<double>(s, a, scaling, density, color, others, maxb);
}
extern "C" int or_forward_secondary_f32(void* s, const or_args* a, float* scaling, float* density, float* color,
                                        float* others, float* maxb) {
  return forward_sec_impl<float>(s, a, scaling, density, color, others, maxb);
}
extern "C" int or_backward_secondary_f64(void* s, const or_args* a, double* dtri, double* dsigma, double* dopac,
                                         double* dsh) {
  return backward_sec_impl<double>(s, a, dtri, dsigma, dopac, dsh);
}
extern "C" int or_backward_secondary_f32(void* s, const or_args* a, float* dtri, float* dsigma, float* dopac,
                                         float* dsh) {
  return backward_sec_impl<float>(s, a, dtri, dsigma, dopac, dsh);
}

// Every triangle hit in [0, tmax] of each ray, ordered by (t, primitive id),
// truncated to max_hits: the stream the chunked k-closest query walks through.
extern "C" int or_hit_stream(void* scene, const float* ray_o, const float* ray_d, int R, float tmax, int max_hits,
                  uint32_t* ids, float* ts, int* counts, int nthreads) {
  const Scene& sc = *static_cast<Scene*>(scene);
  auto one = [&](int i) {
    const RayPre rp = ray_pre(ray_o + 3 * (size_t)i, ray_d + 3 * (size_t)i);
    std::vector<Hit> hits;
    sc.for_each_hit(rp, 0.0f, tmax, true, [&](int prim, float t, float tcur) -> float {
      hits.push_back(Hit{(uint32_t)prim, t});
      return tcur;
    });
    std::sort(hits.begin(), hits.end(), [](const Hit& a, const Hit& b) { return hit_less(a, b, true); });
    const int n = (int)hits.size();
    counts[i] = n;
    for (int k = 0; k < n && k < max_hits; ++k) {
      ids[(size_t)i * max_hits + k] = hits[k].id;
      ts[(size_t)i * max_hits + k] = hits[k].t;
    }
  };
  const int nt = nthreads > 1 ? nthreads : 1;
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t)
    th.emplace_back([&, t]() {
      for (int i = t; i < R; i += nt) one(i);
    });
  for (auto& x : th) x.join();
  return 0;
}

// The float watertight test on one ray/triangle pair (unit tests).
extern "C" int or_isect(const float* o, const float* d, const float* v0, const float* v1, const float* v2, float* t) {
  const RayPre rp = ray_pre(o, d);
  return isect_tri(rp, v0, v1, v2, t) ? 1 : 0;
}

