// fz_pair.cuh -- pair arithmetic shared by the stepping and adjoint kernels.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include "fz_device.cuh"

namespace fz {

// ------------------------------------------------------------------------------------------
// Pair arithmetic. A pair holds the same quantity for two variables (pressure and the velocity
// component normal to the sweep), so every WENO-Z and flux operation runs on both at once. In
// FP32 these are the sm_100 paired instructions (add/mul/fma .f32x2).
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ float2 pmk(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 pmk(double a, double b) { return make_double2(a, b); }
__device__ __forceinline__ float2 padd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 pmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 pfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 psub(float2 a, float2 b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;"
      : "=l"(r)
      : "l"(*reinterpret_cast<unsigned long long*>(&a)), "l"(*reinterpret_cast<unsigned long long*>(&b)));
  return *reinterpret_cast<float2*>(&r);
}
__device__ __forceinline__ float2 pabs(float2 a) { return make_float2(fabsf(a.x), fabsf(a.y)); }
__device__ __forceinline__ float frcp(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float2 prcp(float2 a) { return make_float2(frcp(a.x), frcp(a.y)); }
__device__ __forceinline__ float2 pswap(float2 a) { return make_float2(a.y, a.x); }

__device__ __forceinline__ double2 padd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 pmul(double2 a, double2 b) { return make_double2(a.x * b.x, a.y * b.y); }
__device__ __forceinline__ double2 pfma(double2 a, double2 b, double2 c) {
  return make_double2(fma(a.x, b.x, c.x), fma(a.y, b.y, c.y));
}
__device__ __forceinline__ double2 psub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 pabs(double2 a) { return make_double2(fabs(a.x), fabs(a.y)); }
__device__ __forceinline__ double2 prcp(double2 a) { return make_double2(1.0 / a.x, 1.0 / a.y); }
__device__ __forceinline__ double2 pswap(double2 a) { return make_double2(a.y, a.x); }

template <class R>
__device__ __forceinline__ typename Pair<R>::T psplat(R x) {
  return pmk(x, x);
}

}  // namespace fz
