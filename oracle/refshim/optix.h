// Test infrastructure (oracle): a stand-in for the OptiX 7.7 device API that
// lets the reference's own device sources (tritracer/*.cu) compile as host
// C++. It declares only what those sources call; ref_driver.cpp implements
// optixTrace with the oracle's FP32 intersector and CPU BVH (accel.hpp).
#pragma once
#include <cstdint>
#include <vector_types.h>

typedef unsigned long long OptixTraversableHandle;
typedef unsigned int OptixVisibilityMask;
enum { OPTIX_RAY_FLAG_NONE = 0u, OPTIX_RAY_FLAG_DISABLE_CLOSESTHIT = 1u << 3 };

#define TT_U unsigned int&
void optixTrace(OptixTraversableHandle, float3, float3, float, float, float, OptixVisibilityMask, unsigned int,
                unsigned int, unsigned int, unsigned int, TT_U, TT_U, TT_U, TT_U, TT_U, TT_U, TT_U, TT_U, TT_U,
                TT_U, TT_U, TT_U, TT_U, TT_U, TT_U, TT_U, TT_U, TT_U, TT_U, TT_U, TT_U, TT_U, TT_U, TT_U, TT_U,
                TT_U, TT_U, TT_U, TT_U, TT_U, TT_U, TT_U);
#undef TT_U

#define TT_PAYLOAD(n)                  \
  unsigned int optixGetPayload_##n(); \
  void optixSetPayload_##n(unsigned int);
TT_PAYLOAD(0) TT_PAYLOAD(1) TT_PAYLOAD(2) TT_PAYLOAD(3) TT_PAYLOAD(4) TT_PAYLOAD(5) TT_PAYLOAD(6) TT_PAYLOAD(7)
TT_PAYLOAD(8) TT_PAYLOAD(9) TT_PAYLOAD(10) TT_PAYLOAD(11) TT_PAYLOAD(12) TT_PAYLOAD(13) TT_PAYLOAD(14)
TT_PAYLOAD(15) TT_PAYLOAD(16) TT_PAYLOAD(17) TT_PAYLOAD(18) TT_PAYLOAD(19) TT_PAYLOAD(20) TT_PAYLOAD(21)
TT_PAYLOAD(22) TT_PAYLOAD(23) TT_PAYLOAD(24) TT_PAYLOAD(25) TT_PAYLOAD(26) TT_PAYLOAD(27) TT_PAYLOAD(28)
TT_PAYLOAD(29) TT_PAYLOAD(30) TT_PAYLOAD(31)
#undef TT_PAYLOAD

unsigned int optixGetPrimitiveIndex();
float optixGetRayTmax();
void optixIgnoreIntersection();
uint3 optixGetLaunchIndex();
uint3 optixGetLaunchDimensions();
