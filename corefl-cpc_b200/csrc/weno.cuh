// Nonlinear WENO reconstruction of one interface value from point values.
//
// weno5: Jiang-Shu weights a_r = d_r/(eps+beta_r)^2 (src/WENO.cu:3033-3088).
// weno7: Z-type weights a_r = d_r (1 + tau7/(eps+beta_r)^2), tau7 = (b0+3b1-3b2-b3)^2
//        (src/WENO.cu:3090-3196).
// Both fall back to the linear (optimal) weights when `shock` is false.
//
// The "plus" side reconstructs the left-biased value at i+1/2 from v[i-r+1 .. i+r-1]
// (r = 3 or 4, v[r-1] is node i); the "minus" side reconstructs the right-biased value
// from v[i-r+2 .. i+r] (v[r-2] is node i).  The interface value is plus + minus.
#pragma once
#include "common.cuh"

namespace cb2 {

template <typename T>
__device__ __forceinline__ T sq(T x) { return x * x; }

// ---- WENO5 -------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T weno5_plus(const T *v, T eps, bool shock) {
  const T k6 = T(1.0 / 6);
  // candidate stencils S2={i,i+1,i+2}, S1={i-1,i,i+1}, S0={i-2,i-1,i}
  const T q2 = k6 * (2 * v[2] + 5 * v[3] - v[4]);
  const T q1 = k6 * (-v[1] + 5 * v[2] + 2 * v[3]);
  const T q0 = k6 * (2 * v[0] - 7 * v[1] + 11 * v[2]);
  if (!shock) return T(0.3) * q2 + T(0.6) * q1 + T(0.1) * q0;
  const T k13 = T(13.0 / 12);
  const T b2 = k13 * sq(v[2] + v[4] - 2 * v[3]) + T(0.25) * sq(3 * v[2] - 4 * v[3] + v[4]);
  const T b1 = k13 * sq(v[1] + v[3] - 2 * v[2]) + T(0.25) * sq(v[1] - v[3]);
  const T b0 = k13 * sq(v[0] + v[2] - 2 * v[1]) + T(0.25) * sq(v[0] - 4 * v[1] + 3 * v[2]);
  const T a2 = T(0.3) / sq(eps + b2);
  const T a1 = T(0.6) / sq(eps + b1);
  const T a0 = T(0.1) / sq(eps + b0);
  return (a2 * q2 + a1 * q1 + a0 * q0) / (a2 + a1 + a0);
}

template <typename T>
__device__ __forceinline__ T weno5_minus(const T *v, T eps, bool shock) {
  const T k6 = T(1.0 / 6);
  const T q0 = k6 * (11 * v[2] - 7 * v[3] + 2 * v[4]);
  const T q1 = k6 * (2 * v[1] + 5 * v[2] - v[3]);
  const T q2 = k6 * (-v[0] + 5 * v[1] + 2 * v[2]);
  if (!shock) return T(0.1) * q0 + T(0.6) * q1 + T(0.3) * q2;
  const T k13 = T(13.0 / 12);
  const T b0 = k13 * sq(v[2] + v[4] - 2 * v[3]) + T(0.25) * sq(3 * v[2] - 4 * v[3] + v[4]);
  const T b1 = k13 * sq(v[1] + v[3] - 2 * v[2]) + T(0.25) * sq(v[1] - v[3]);
  const T b2 = k13 * sq(v[0] + v[2] - 2 * v[1]) + T(0.25) * sq(v[0] - 4 * v[1] + 3 * v[2]);
  const T a0 = T(0.1) / sq(eps + b0);
  const T a1 = T(0.6) / sq(eps + b1);
  const T a2 = T(0.3) / sq(eps + b2);
  return (a0 * q0 + a1 * q1 + a2 * q2) / (a0 + a1 + a2);
}

// ---- WENO7 -------------------------------------------------------------------------
// Smoothness indicator of one 4-point sub-stencil written with its first, second and
// third undivided differences d1, d2, d3: beta = d1^2 + 13/12 d2^2 + 1043/960 d3^2 + d1 d3/12.
template <typename T>
__device__ __forceinline__ T beta7(T d1, T d2, T d3) {
  return d1 * d1 + T(13.0 / 12.0) * d2 * d2 + T(1043.0 / 960) * d3 * d3 + T(1.0 / 12) * d1 * d3;
}

// Plus side on u[0..6] (u[3] = node i).  The minus side is the same function applied to
// the mirrored stencil (u[k] = v[6-k]) of the right-biased values.
template <typename T>
__device__ __forceinline__ T weno7_side(T u0, T u1, T u2, T u3, T u4, T u5, T u6, T eps, bool shock) {
  const T c0 = T(1.0 / 35), c1 = T(12.0 / 35), c2 = T(18.0 / 35), c3 = T(4.0 / 35);
  const T q0 = -3 * u0 + 13 * u1 - 23 * u2 + 25 * u3;
  const T q1 = u1 - 5 * u2 + 13 * u3 + 3 * u4;
  const T q2 = -u2 + 7 * u3 + 7 * u4 - u5;
  const T q3 = 3 * u3 + 13 * u4 - 5 * u5 + u6;
  if (!shock) return T(1.0 / 12) * (c0 * q0 + c1 * q1 + c2 * q2 + c3 * q3);
  const T k6 = T(1.0 / 6);
  const T b0 = beta7(k6 * (-2 * u0 + 9 * u1 - 18 * u2 + 11 * u3), -u0 + 4 * u1 - 5 * u2 + 2 * u3,
                     -u0 + 3 * u1 - 3 * u2 + u3);
  const T d2m = u2 - 2 * u3 + u4;  // shared second difference of sub-stencils 1 and 2
  const T b1 = beta7(k6 * (u1 - 6 * u2 + 3 * u3 + 2 * u4), d2m, -u1 + 3 * u2 - 3 * u3 + u4);
  const T b2 = beta7(k6 * (-2 * u2 - 3 * u3 + 6 * u4 - u5), d2m, -u2 + 3 * u3 - 3 * u4 + u5);
  const T b3 = beta7(k6 * (-11 * u3 + 18 * u4 - 9 * u5 + 2 * u6), 2 * u3 - 5 * u4 + 4 * u5 - u6,
                     -u3 + 3 * u4 - 3 * u5 + u6);
  const T tau = sq(b0 + 3 * b1 - 3 * b2 - b3);
  const T a0 = c0 + c0 * tau / sq(eps + b0);
  const T a1 = c1 + c1 * tau / sq(eps + b1);
  const T a2 = c2 + c2 * tau / sq(eps + b2);
  const T a3 = c3 + c3 * tau / sq(eps + b3);
  return T(1.0 / 12) * (a0 * q0 + a1 * q1 + a2 * q2 + a3 * q3) / (a0 + a1 + a2 + a3);
}

template <typename T>
__device__ __forceinline__ T weno7_plus(const T *v, T eps, bool shock) {
  return weno7_side(v[0], v[1], v[2], v[3], v[4], v[5], v[6], eps, shock);
}
template <typename T>
__device__ __forceinline__ T weno7_minus(const T *v, T eps, bool shock) {
  return weno7_side(v[6], v[5], v[4], v[3], v[2], v[1], v[0], eps, shock);
}

template <int ORDER, typename T>
__device__ __forceinline__ T weno_pm(const T *vp, const T *vm, T eps, bool shock) {
  if constexpr (ORDER == 5) return weno5_plus(vp, eps, shock) + weno5_minus(vm, eps, shock);
  else return weno7_plus(vp, eps, shock) + weno7_minus(vm, eps, shock);
}

}  // namespace cb2
