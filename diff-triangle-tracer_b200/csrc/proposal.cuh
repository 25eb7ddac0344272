// Launch interface of the proposal network kernels (proposal.cu).
//
// The network maps a ray (origin, direction) to the interval [t_near, t_far]
// of its hits. The origin is first moved along the ray to its closest
// approach to the scene centre (o' = o + s d, s = -(o - c).d / d.d), so the
// inputs depend on the ray's line only and rays of unseen cameras look like
// the training rays; the outputs are t - s. 80 encoded inputs: the 6
// coordinates (o' - c scaled, d), sin / cos of 2^k pi x for k = 0..5 over
// them, a constant 1 standing for the bias, one zero; three hidden layers of
// 64 ReLU units (each again followed by a constant-1 input) and a linear
// output layer of 16 rows of which the first two are used. Every contraction
// runs on the tensor cores (tcgen05.mma, BF16 operands, FP32 accumulators in
// tensor memory).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace tt {
namespace mlp {

constexpr int kIn = 80;      // encoded inputs per layer (incl. the bias input)
constexpr int kHid = 64;     // hidden units
constexpr int kOutRows = 16; // rows of the output layer (2 used)
constexpr int kLayerRows[4] = {kHid, kHid, kHid, kOutRows};
constexpr int kLayerOff[4] = {0, kHid * kIn, 2 * kHid * kIn, 3 * kHid * kIn};  // element offsets
constexpr int kParams = 3 * kHid * kIn + kOutRows * kIn;                       // 16640
constexpr int kPartial = kParams + 16;  // floats per CTA of the training reduction (+ loss)
constexpr int kMaxViews = 32;
constexpr int kTileRows = 128;  // rays per tile = MMA M

// Rays of one image or one packed batch: ray r has origin o[r*stride .. +3]
// and direction d[r*stride .. +3]; its two outputs go to out0[r*ostride] and
// out1[r*ostride].
struct RaySet {
  const float* o;
  const float* d;
  int stride;
  float* out0;
  float* out1;
  int ostride;
  int n;
  int tile_begin;
};

struct InferParams {
  const uint16_t* w;  // BF16 weights in the tensor-core layout (kParams)
  int nsets, ntiles;
  RaySet sets[kMaxViews];
  float origin_scale, t_shift, t_scale;
  float cx, cy, cz;  // scene centre
  // interval = [t0 - margin_near, t1 + margin_far]; t_far = +inf when
  // t1 + margin_far - s >= far_cap (measured from the closest approach)
  float margin_near, margin_far, far_cap;
  int* status;
};

struct TrainParams {
  const uint16_t* w;
  const float* rays;     // [n][6]: origin, direction
  const float* targets;  // [n][2]: t_near (< 0: no t_near target), t_far (t units)
  int n, ntiles, tiles_per_cta;
  float origin_scale, t_shift, inv_t_scale;
  float cx, cy, cz;
  float near_weight;  // loss weight of a t_near above its target (hits cut off)
  float far_weight;   // loss weight of a t_far below its target (a continuation)
  float* partial;  // [gridDim.x][kPartial]: dL/dW sums (unscaled) and the loss sum
  int* status;
};

struct AdamParams {
  const float* partial;
  int nparts;
  float grad_scale;  // 1 / batch
  float* master;     // FP32 weights [kParams], row-major per layer
  float* m;
  float* v;
  uint16_t* w;  // BF16 tensor-core layout
  float lr, beta1, beta2, eps, c1, c2;  // c1 = 1/(1-beta1^t), c2 = 1/(1-beta2^t)
  float* loss;  // optional: mean loss of the step
  int adam;     // 0: only convert master -> w (initialisation)
};

size_t infer_smem_bytes();
size_t train_smem_bytes();
cudaError_t launch_infer(const InferParams& p, int grid, cudaStream_t s);
cudaError_t launch_train(const TrainParams& p, int grid, cudaStream_t s);
cudaError_t launch_adam(const AdamParams& p, cudaStream_t s);
int infer_blocks_per_sm();

}  // namespace mlp
}  // namespace tt
