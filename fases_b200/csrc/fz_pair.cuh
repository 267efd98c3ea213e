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

// ------------------------------------------------------------------------------------------
// WENO-Z reconstruction at one cell centre (Borges, Carmona, Costa & Don 2008, q = 1), the scheme
// of functions3D.cuh:763-1001 with the tables of main3D.cu:834-843 and eps = 1e-10 (main3D.cu:770).
//
// The reference evaluates V-(i+1/2) (idx = 1) and V+(i-1/2) (idx = 0) of a cell in two separate
// calls; both use the same three smoothness indicators and the same factors (1 + tau/(beta+eps)),
// and differ only in the linear weights d (mirrored) and the candidate rows. This evaluates them
// together, written on first differences a..d of the five-point stencil:
//   candidates:  u_i + delta_r,   V = u_i + sum_r w_r delta_r,   w_r = d_r q_r / sum d q
//   12/13 beta_r = (second difference)^2 + 3/13 (one-sided first-derivative term)^2
// (the 12/13 scaling is absorbed into eps).
// ------------------------------------------------------------------------------------------
// FACES selects the face values computed: WENO_BOTH, or only V- (WENO_LO) or V+ (WENO_HI) where a
// caller uses one of them (the tile's halo rows); the value computed is the same either way.
constexpr int WENO_LO = 1, WENO_HI = 2, WENO_BOTH = 3;
template <class R, int FACES = WENO_BOTH>
__device__ __forceinline__ void weno_core(typename Pair<R>::T a, typename Pair<R>::T b, typename Pair<R>::T c,
                                          typename Pair<R>::T d, typename Pair<R>::T D2, typename Pair<R>::T D1,
                                          typename Pair<R>::T D0, typename Pair<R>::T q0, typename Pair<R>::T& vm,
                                          typename Pair<R>::T& vp) {
  typedef typename Pair<R>::T P;
  const P E2 = pfma(b, psplat<R>(R(2)), D2);   // u_{i-2} - 4u_{i-1} + 3u_i
  const P E1 = padd(b, c);                     // -(u_{i-1} - u_{i+1})
  const P E0 = pfma(c, psplat<R>(R(-2)), D0);  // 3u_i - 4u_{i+1} + u_{i+2} (sign)
  // 12/13 (beta_r + eps) = D_r^2 + 3/13 E_r^2 + 12/13 eps
  const P k313 = psplat<R>(R(3.0 / 13.0));
  const P eps = psplat<R>(R(1e-10 * 12.0 / 13.0));
  const P B0 = pfma(D0, D0, pfma(pmul(E0, k313), E0, eps));
  const P B1 = pfma(D1, D1, pfma(pmul(E1, k313), E1, eps));
  const P B2 = pfma(D2, D2, pfma(pmul(E2, k313), E2, eps));
  const P tau = pabs(psub(B0, B2));
#if defined(FZ_V_FEWRCP)
  // w_r ~ d_r (1 + tau/B_r) = d_r (B_r + tau) / B_r: the normalised weights do not change when
  // every (1 + tau/B_r) is scaled by B0 B1 B2, which leaves (B_r + tau) times the other two B's
  const P B01 = pmul(B0, B1), B02 = pmul(B0, B2), B12 = pmul(B1, B2);
  const P B012 = pmul(B12, B0);
  const P q0w = pfma(tau, B12, B012);
  const P q1w = pfma(tau, B02, B012);
  const P q2w = pfma(tau, B01, B012);
#else
  const P one = psplat<R>(R(1));
  const P q0w = pfma(tau, prcp(B0), one);
  const P q1w = pfma(tau, prcp(B1), one);
  const P q2w = pfma(tau, prcp(B2), one);
#endif
  // normalisers: V- uses d = (3/10, 3/5, 1/10), V+ the mirrored (1/10, 3/5, 3/10)
  constexpr bool LO = (FACES & WENO_LO) != 0, HI = (FACES & WENO_HI) != 0;
  const P t1 = pmul(q1w, psplat<R>(R(0.6)));
  P Sm, Sp, em0, ep0, em1, ep1, em2, ep2;
  if constexpr (LO) Sm = pfma(q0w, psplat<R>(R(0.3)), pfma(q2w, psplat<R>(R(0.1)), t1));
  if constexpr (HI) Sp = pfma(q0w, psplat<R>(R(0.1)), pfma(q2w, psplat<R>(R(0.3)), t1));
  // d_r * delta_r for both faces, written on the first and second differences:
  //   em0 = 0.15 c - 0.05 D0      ep0 = -0.05 c + D0/30
  //   em1 = 0.15 E1 + 0.05 D1     ep1 = -0.15 E1 + 0.05 D1
  //   em2 = 0.05 b + D2/30        ep2 = -0.15 b - 0.05 D2
  const P h1 = pmul(D1, psplat<R>(R(0.05)));
  if constexpr (LO) em0 = pfma(c, psplat<R>(R(0.15)), pmul(D0, psplat<R>(R(-0.05))));
  if constexpr (HI) ep0 = pfma(c, psplat<R>(R(-0.05)), pmul(D0, psplat<R>(R(1.0 / 30.0))));
  if constexpr (LO) em1 = pfma(E1, psplat<R>(R(0.15)), h1);
  if constexpr (HI) ep1 = pfma(E1, psplat<R>(R(-0.15)), h1);
  if constexpr (LO) em2 = pfma(b, psplat<R>(R(0.05)), pmul(D2, psplat<R>(R(1.0 / 30.0))));
  if constexpr (HI) ep2 = pfma(b, psplat<R>(R(-0.15)), pmul(D2, psplat<R>(R(-0.05))));
  P Nm, Np;
  if constexpr (LO) Nm = pfma(q2w, em2, pfma(q1w, em1, pmul(q0w, em0)));
  if constexpr (HI) Np = pfma(q2w, ep2, pfma(q1w, ep1, pmul(q0w, ep0)));
  if constexpr (LO) vm = pfma(Nm, prcp(Sm), q0);
  if constexpr (HI) vp = pfma(Np, prcp(Sp), q0);
}

template <class R, int FACES = WENO_BOTH>
__device__ __forceinline__ void weno_center(typename Pair<R>::T qm2, typename Pair<R>::T qm1,
                                            typename Pair<R>::T q0, typename Pair<R>::T qp1,
                                            typename Pair<R>::T qp2, typename Pair<R>::T& vm,
                                            typename Pair<R>::T& vp) {
  typedef typename Pair<R>::T P;
  const P a = psub(qm1, qm2), b = psub(q0, qm1), c = psub(qp1, q0), d = psub(qp2, qp1);
  weno_core<R, FACES>(a, b, c, d, psub(b, a), psub(c, b), psub(d, c), q0, vm, vp);
}

// Godunov (exact Riemann) flux of linear acoustics for a (pressure, normal velocity) pair
// (functions3D.cuh:56-78):  F_p = 1/2 (rho c^2 (q+ + q-) - c (p+ - p-)),
//                           F_q = 1/2 ((p+ + p-)/rho - c (q+ - q-)).
template <class R>
__device__ __forceinline__ typename Pair<R>::T godunov(typename Pair<R>::T vm, typename Pair<R>::T vp,
                                                       typename Pair<R>::T kA, typename Pair<R>::T kC) {
  const typename Pair<R>::T sum = padd(vm, vp), dif = psub(vp, vm);
#if defined(FZ_V_SCALARFLUX)
  return pmk(fma(dif.x, kC.x, sum.y * kA.x), fma(dif.y, kC.y, sum.x * kA.y));
#else
  return pfma(dif, kC, pmul(pswap(sum), kA));
#endif
}

// Difference of the Godunov fluxes through the low and the high face of a cell, F(lo) - F(hi),
// from the face states (left state of a face = V- of the centre below it, right state = V+ of the
// centre above): the flux is linear in the states, so the difference is taken on the sums and
// differences first and swapped and scaled once.
template <class R>
__device__ __forceinline__ typename Pair<R>::T godunov_diff(typename Pair<R>::T vm_lo, typename Pair<R>::T vp_lo,
                                                            typename Pair<R>::T vm_hi, typename Pair<R>::T vp_hi,
                                                            typename Pair<R>::T kA, typename Pair<R>::T kC) {
  const typename Pair<R>::T S = psub(padd(vm_lo, vp_lo), padd(vm_hi, vp_hi));
  const typename Pair<R>::T D = psub(psub(vp_lo, vm_lo), psub(vp_hi, vm_hi));
#if defined(FZ_V_SCALARFLUX)
  // the swapped product in scalar form: the same arithmetic without moving the pair's halves
  return pmk(fma(D.x, kC.x, S.y * kA.x), fma(D.y, kC.y, S.x * kA.y));
#else
  return pfma(D, kC, pmul(pswap(S), kA));
#endif
}

}  // namespace fz
