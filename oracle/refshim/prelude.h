// Test infrastructure (oracle): force-included ahead of each reference source
// when it is compiled as host C++. Supplies host versions of the CUDA device
// built-ins those sources use; __powf/__logf come from ../hostmath.h so the
// restatement and this build share them.
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>

#include "../hostmath.h"

static inline float __uint_as_float(unsigned int u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}
static inline unsigned int __float_as_uint(float f) {
  unsigned int u;
  std::memcpy(&u, &f, 4);
  return u;
}
static inline int __float_as_int(float f) {
  int u;
  std::memcpy(&u, &f, 4);
  return u;
}
inline float __powf(float x, float y) { return tt_host_powf(x, y); }
inline float __logf(float x) { return tt_host_logf(x); }

// Device min/max on float/double are fminf/fmaxf/fmin/fmax.
static inline float min(float a, float b) { return fminf(a, b); }
static inline float max(float a, float b) { return fmaxf(a, b); }
static inline double min(double a, double b) { return fmin(a, b); }
static inline double max(double a, double b) { return fmax(a, b); }

static inline float atomicAdd(float* p, float v) {
  float cur;
  __atomic_load(p, &cur, __ATOMIC_RELAXED);
  float nxt;
  do {
    nxt = cur + v;
  } while (!__atomic_compare_exchange(p, &cur, &nxt, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED));
  return cur;
}
static inline int atomicMax(int* p, int v) {
  int cur = __atomic_load_n(p, __ATOMIC_RELAXED);
  while (v > cur) {
    if (__atomic_compare_exchange_n(p, &cur, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) break;
  }
  return cur;
}
