// Launch interface of the trace kernels (trace.cu).
#pragma once
#include <cuda_runtime.h>

#include "tt_device.cuh"

namespace tt {

struct TraceParams {
  BvhView bvh;
  int H, W;
  int ntx, ntiles;  // 8x4 pixel tiles
  const float* ray_o;
  const float* ray_d;
  const float* verts;
  const int* cumsum;
  const int* num_points;
  const float* shs;
  int sh_degree, M;
  const float* opac;
  const float* sigma;
  const float* bg;
  // forward outputs
  float* scaling;
  float* density;
  float* max_blending;
  float* out_color;
  float* out_others;
  // adjoint inputs/outputs
  const float* colors;
  const float* others;
  const float* dL_dpix;
  const float* dL_doth;
  float* d_tri;
  float* d_sigma;
  float* d_opac;
  float* d_sh;
  // variants (extra = [r, cx, cy, cz, samples])
  int variant;
  float sph_r, sph_cx, sph_cy, sph_cz;
  int samples;
  int tmin_inclusive;
  int packets;  // 1: warp packet traversal (coherent rays), 0: one independent ray per lane
  int* work;    // tile counter, zero at launch
  int* status;  // kStatus* bits
  unsigned long long* stats;  // forward: rays, evaluated hits, blended hits, node visits, triangle tests, queries
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

constexpr int kTraceThreads = 128;
constexpr int kStackDepth = 32;

size_t trace_smem_bytes(int packets);
// Resident blocks per SM of the forward / adjoint kernels (occupancy query).
int trace_blocks_per_sm(int which /*0 forward, 1 adjoint*/, int packets);
cudaError_t launch_forward(const TraceParams& p, int grid, cudaStream_t s);
cudaError_t launch_backward(const TraceParams& p, int grid, cudaStream_t s);
cudaError_t launch_hit_stream(const HitStreamParams& p, cudaStream_t s);

}  // namespace tt
