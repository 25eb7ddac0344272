// Test infrastructure: host stand-ins for the two CUDA fast-math intrinsics the
// reference's device code calls (__powf in common.h:111, __logf in
// backward.cu:320). Both the oracle restatement (oracle.hpp) and the host build
// of the reference's own sources (refshim/) call these same functions, so the
// FP32 restatement can be compared with the reference's code bit for bit.
//
// The GPU intrinsic __powf(x, y) is documented as exp2(y * log2(x)); for a
// negative base it is NaN whatever y is (log2 of a negative number), which the
// reference then clamps to 0 with fmaxf (common.h:111). std::pow would return a
// real value for integral y, so the negative base is handled explicitly. The
// value itself is the correctly rounded power (the hardware approximation is
// not reproduced; only its domain behaviour is).
#pragma once
#include <cmath>
#include <limits>

static inline float tt_host_powf(float x, float y) {
  if (!(x >= 0.0f)) return std::numeric_limits<float>::quiet_NaN();
  return (float)std::pow((double)x, (double)y);
}

static inline float tt_host_logf(float x) { return (float)std::log((double)x); }
