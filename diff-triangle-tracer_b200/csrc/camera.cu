// Pinhole camera -> primary rays on the device (tt_camera_rays). Each pixel's
// direction is evaluated in FP64 with explicitly rounded operations in the
// order of the package's host generator (diff_tritracer.scenes.camera_rays),
// so both give the same FP32 rays bit for bit.
#include "../../include/tritracer.h"
#include "trace.cuh"

namespace tt {
namespace {

struct CameraSet {
  tt_camera cam[kMaxViews];
  long long begin[kMaxViews + 1];  // first pixel of each camera in the launch's numbering
  int n;
};

__global__ void k_camera_rays(const __grid_constant__ CameraSet cs) {
  const long long total = cs.begin[cs.n];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    int c = 0;
    while (c + 1 < cs.n && cs.begin[c + 1] <= i) ++c;
    const tt_camera& k = cs.cam[c];
    const long long pix = i - cs.begin[c];
    const int y = (int)(pix / k.W), x = (int)(pix - (long long)y * k.W);
    const double W = (double)k.W, H = (double)k.H, t = k.tan_half_fov;
    const double u = __dmul_rn(__dmul_rn(__dsub_rn(__ddiv_rn(__dmul_rn(2.0, __dadd_rn((double)x, 0.5)), W), 1.0), t),
                               __ddiv_rn(W, H));
    const double v = __dmul_rn(__dsub_rn(1.0, __ddiv_rn(__dmul_rn(2.0, __dadd_rn((double)y, 0.5)), H)), t);
    double d[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) d[j] = __dadd_rn(__dadd_rn(k.forward[j], __dmul_rn(u, k.right[j])), __dmul_rn(v, k.up[j]));
    const double n = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(d[0], d[0]), __dmul_rn(d[1], d[1])), __dmul_rn(d[2], d[2])));
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      k.ray_o[3 * pix + j] = __double2float_rn(k.origin[j]);
      k.ray_d[3 * pix + j] = __double2float_rn(__ddiv_rn(d[j], n));
    }
  }
}

}  // namespace

cudaError_t launch_camera_rays(const tt_camera* cams, int n, cudaStream_t s) {
  CameraSet cs;
  cs.n = n;
  cs.begin[0] = 0;
  for (int c = 0; c < n; ++c) {
    cs.cam[c] = cams[c];
    cs.begin[c + 1] = cs.begin[c] + (long long)cams[c].H * cams[c].W;
  }
  const long long total = cs.begin[n];
  if (total == 0) return cudaSuccess;
  const int grid = (int)((total + 255) / 256 < 148 * 16 ? (total + 255) / 256 : 148 * 16);
  k_camera_rays<<<grid, 256, 0, s>>>(cs);
  return cudaGetLastError();
}

}  // namespace tt
