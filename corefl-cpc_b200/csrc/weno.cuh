// Nonlinear WENO reconstruction of one interface value from point values.
//
// weno5: Jiang-Shu weights a_r = d_r/(eps+beta_r)^2 (src/WENO.cu:3033-3088).
// weno7: Z-type weights a_r = d_r (1 + tau7/(eps+beta_r)^2), tau7 = (b0+3b1-3b2-b3)^2
//        (src/WENO.cu:3090-3196).
// Both fall back to the linear (optimal) weights when `shock` is false.
// The normalised weights are evaluated with one division per side: every a_r is multiplied
// by the product of all (eps+beta)^2 terms, which leaves sum(a_r q_r)/sum(a_r) unchanged
// (the reference divides once per sub-stencil, src/WENO.cu:3051-3053, 3127-3130).
//
// The "plus" side reconstructs the left-biased value at i+1/2 from v[i-r+1 .. i+r-1]
// (r = 3 or 4, v[r-1] is node i); the "minus" side reconstructs the right-biased value
// from v[i-r+2 .. i+r] (v[r-2] is node i).  The interface value is plus + minus.
#pragma once
#include "common.cuh"

namespace cb2 {

template <typename T>
__device__ __forceinline__ T sq(T x) { return x * x; }

// Exact power of two s with x*s in [1, 2) for a positive normal x (the reciprocal of x's
// binade).  The nonlinear weights below are products of three or four (eps + beta)^2 terms;
// scaling every term by the same s keeps the normalised weights unchanged, changes no
// rounding, and keeps the products far from FP underflow and overflow.
__device__ __forceinline__ double binade_inv(double x) {
  return __hiloint2double(0x7FE00000 - (__double2hiint(x) & 0x7FF00000), 0);
}
__device__ __forceinline__ float binade_inv(float x) {
  return __int_as_float(0x7F000000 - (__float_as_int(x) & 0x7F800000));
}

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
  // a_r = d_r / D_r with D_r = (eps + beta_r)^2; multiplying every a_r by D0 D1 D2 leaves
  // the normalised weights unchanged and needs one division instead of four
  T D0 = sq(eps + b0), D1 = sq(eps + b1), D2 = sq(eps + b2);
  const T sc = binade_inv(fmax(fmax(D0, D1), D2));
  D0 *= sc; D1 *= sc; D2 *= sc;
  const T w2 = T(0.3) * (D0 * D1), w1 = T(0.6) * (D0 * D2), w0 = T(0.1) * (D1 * D2);
  return (w2 * q2 + w1 * q1 + w0 * q0) / (w2 + w1 + w0);
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
  T D0 = sq(eps + b0), D1 = sq(eps + b1), D2 = sq(eps + b2);
  const T sc = binade_inv(fmax(fmax(D0, D1), D2));
  D0 *= sc; D1 *= sc; D2 *= sc;
  const T w0 = T(0.1) * (D1 * D2), w1 = T(0.6) * (D0 * D2), w2 = T(0.3) * (D0 * D1);
  return (w0 * q0 + w1 * q1 + w2 * q2) / (w0 + w1 + w2);
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
  T tau = sq(b0 + 3 * b1 - 3 * b2 - b3);
  // a_r = c_r (1 + tau/D_r) = c_r (D_r + tau)/D_r, D_r = (eps + beta_r)^2; scaled by
  // D0 D1 D2 D3 the normalised weights need a single division.  D_r and tau are first
  // brought to the binade of the largest D_r, so the triple products cannot underflow.
  T D0 = sq(eps + b0), D1 = sq(eps + b1), D2 = sq(eps + b2), D3 = sq(eps + b3);
  const T sc = binade_inv(fmax(fmax(D0, D1), fmax(D2, D3)));
  D0 *= sc; D1 *= sc; D2 *= sc; D3 *= sc; tau *= sc;
  const T D01 = D0 * D1, D23 = D2 * D3;
  const T w0 = c0 * (D0 + tau) * (D1 * D23);
  const T w1 = c1 * (D1 + tau) * (D0 * D23);
  const T w2 = c2 * (D2 + tau) * (D01 * D3);
  const T w3 = c3 * (D3 + tau) * (D01 * D2);
  return T(1.0 / 12) * (w0 * q0 + w1 * q1 + w2 * q2 + w3 * q3) / (w0 + w1 + w2 + w3);
}

template <typename T>
__device__ __forceinline__ T weno7_plus(const T *v, T eps, bool shock) {
  return weno7_side(v[0], v[1], v[2], v[3], v[4], v[5], v[6], eps, shock);
}
template <typename T>
__device__ __forceinline__ T weno7_minus(const T *v, T eps, bool shock) {
  return weno7_side(v[6], v[5], v[4], v[3], v[2], v[1], v[0], eps, shock);
}

// FP32 weights.  The single-division product form needs the product of three or four
// (eps + beta)^2 terms, which FP32 cannot hold across the dynamic range of a discontinuity.  The
// FP32 path normalises by the smallest term instead: with r_s = D_min / D_s in (0, 1],
//   WENO-JS  alpha_s ~ c_s r_s,   WENO-Z  alpha_s ~ c_s (D_min + tau r_s),
// the same weights up to a common factor, every term bounded by c_s (D_min + tau).
__device__ __forceinline__ float rcp32(float x) { return __frcp_rn(x); }

// ---- node-centred pair ---------------------------------------------------------------
// Both one-sided values that the stencil centred on node n produces: the left-biased value at
// n+1/2 (`lp`, the plus side) and the right-biased value at n-1/2 (`rm`, the minus side).
// The two sides integrate over the same cell n with the same sub-stencils, so they share the
// smoothness indicators: beta of minus sub-stencil r equals beta of plus sub-stencil
// (last - r).  The pair costs one set of indicators instead of two.
//   WENO5: v[0..4], v[2] = node n.   WENO7: v[0..6], v[3] = node n.
template <typename T>
__device__ __forceinline__ void weno5_node(const T *v, T eps, T &lp, T &rm) {
  const T k6 = T(1.0 / 6);
  const T q2 = k6 * (2 * v[2] + 5 * v[3] - v[4]);
  const T q1 = k6 * (-v[1] + 5 * v[2] + 2 * v[3]);
  const T q0 = k6 * (2 * v[0] - 7 * v[1] + 11 * v[2]);
  const T m0 = k6 * (11 * v[2] - 7 * v[3] + 2 * v[4]);  // minus side, sub-stencil {n, n+1, n+2}
  const T m1 = k6 * (2 * v[1] + 5 * v[2] - v[3]);
  const T m2 = k6 * (-v[0] + 5 * v[1] + 2 * v[2]);
  const T k13 = T(13.0 / 12);
  const T b2 = k13 * sq(v[2] + v[4] - 2 * v[3]) + T(0.25) * sq(3 * v[2] - 4 * v[3] + v[4]);
  const T b1 = k13 * sq(v[1] + v[3] - 2 * v[2]) + T(0.25) * sq(v[1] - v[3]);
  const T b0 = k13 * sq(v[0] + v[2] - 2 * v[1]) + T(0.25) * sq(v[0] - 4 * v[1] + 3 * v[2]);
  T D0 = sq(eps + b0), D1 = sq(eps + b1), D2 = sq(eps + b2);
  T E0, E1, E2;  // weights of the sub-stencils up to a common factor
  if constexpr (sizeof(T) == 4) {
    const T Dm = fmin(fmin(D0, D1), D2);
    E0 = Dm * rcp32(D0); E1 = Dm * rcp32(D1); E2 = Dm * rcp32(D2);
  } else {
    const T sc = binade_inv(fmax(fmax(D0, D1), D2));
    D0 *= sc; D1 *= sc; D2 *= sc;
    E2 = D0 * D1; E1 = D0 * D2; E0 = D1 * D2;  // prod of D over the other sub-stencils
  }
  const T w2 = T(0.3) * E2, w1 = T(0.6) * E1, w0 = T(0.1) * E0;
  lp = (w2 * q2 + w1 * q1 + w0 * q0) / (w2 + w1 + w0);
  const T u0 = T(0.1) * E2, u1 = T(0.6) * E1, u2 = T(0.3) * E0;
  rm = (u0 * m0 + u1 * m1 + u2 * m2) / (u0 + u1 + u2);
}

template <typename T>
__device__ __forceinline__ void weno7_node(const T *u, T eps, T &lp, T &rm) {
  const T c0 = T(1.0 / 35), c1 = T(12.0 / 35), c2 = T(18.0 / 35), c3 = T(4.0 / 35);
  const T q0 = -3 * u[0] + 13 * u[1] - 23 * u[2] + 25 * u[3];
  const T q1 = u[1] - 5 * u[2] + 13 * u[3] + 3 * u[4];
  const T q2 = -u[2] + 7 * u[3] + 7 * u[4] - u[5];
  const T q3 = 3 * u[3] + 13 * u[4] - 5 * u[5] + u[6];
  // minus side (the plus formulas on the mirrored stencil); m_r lives on plus sub-stencil 3-r
  const T m0 = -3 * u[6] + 13 * u[5] - 23 * u[4] + 25 * u[3];
  const T m1 = u[5] - 5 * u[4] + 13 * u[3] + 3 * u[2];
  const T m2 = -u[4] + 7 * u[3] + 7 * u[2] - u[1];
  const T m3 = 3 * u[3] + 13 * u[2] - 5 * u[1] + u[0];
  const T k6 = T(1.0 / 6);
  const T b0 = beta7(k6 * (-2 * u[0] + 9 * u[1] - 18 * u[2] + 11 * u[3]), -u[0] + 4 * u[1] - 5 * u[2] + 2 * u[3],
                     -u[0] + 3 * u[1] - 3 * u[2] + u[3]);
  const T d2m = u[2] - 2 * u[3] + u[4];
  const T b1 = beta7(k6 * (u[1] - 6 * u[2] + 3 * u[3] + 2 * u[4]), d2m, -u[1] + 3 * u[2] - 3 * u[3] + u[4]);
  const T b2 = beta7(k6 * (-2 * u[2] - 3 * u[3] + 6 * u[4] - u[5]), d2m, -u[2] + 3 * u[3] - 3 * u[4] + u[5]);
  const T b3 = beta7(k6 * (-11 * u[3] + 18 * u[4] - 9 * u[5] + 2 * u[6]), 2 * u[3] - 5 * u[4] + 4 * u[5] - u[6],
                     -u[3] + 3 * u[4] - 3 * u[5] + u[6]);
  T tau = sq(b0 + 3 * b1 - 3 * b2 - b3);  // unchanged by the mirroring
  T D0 = sq(eps + b0), D1 = sq(eps + b1), D2 = sq(eps + b2), D3 = sq(eps + b3);
  T E0, E1, E2, E3;  // Z weights of the sub-stencils up to a common factor
  if constexpr (sizeof(T) == 4) {
    const T Dm = fmin(fmin(D0, D1), fmin(D2, D3));
    E0 = Dm + tau * (Dm * rcp32(D0)); E1 = Dm + tau * (Dm * rcp32(D1));
    E2 = Dm + tau * (Dm * rcp32(D2)); E3 = Dm + tau * (Dm * rcp32(D3));
  } else {
    const T sc = binade_inv(fmax(fmax(D0, D1), fmax(D2, D3)));
    D0 *= sc; D1 *= sc; D2 *= sc; D3 *= sc; tau *= sc;
    const T D01 = D0 * D1, D23 = D2 * D3;
    E0 = (D0 + tau) * (D1 * D23); E1 = (D1 + tau) * (D0 * D23);
    E2 = (D2 + tau) * (D01 * D3); E3 = (D3 + tau) * (D01 * D2);
  }
  const T w0 = c0 * E0, w1 = c1 * E1, w2 = c2 * E2, w3 = c3 * E3;
  lp = T(1.0 / 12) * (w0 * q0 + w1 * q1 + w2 * q2 + w3 * q3) / (w0 + w1 + w2 + w3);
  const T v0 = c0 * E3, v1 = c1 * E2, v2 = c2 * E1, v3 = c3 * E0;
  rm = T(1.0 / 12) * (v0 * m0 + v1 * m1 + v2 * m2 + v3 * m3) / (v0 + v1 + v2 + v3);
}

template <int ORDER, typename T>
__device__ __forceinline__ T weno_pm(const T *vp, const T *vm, T eps, bool shock) {
  if constexpr (ORDER == 5) return weno5_plus(vp, eps, shock) + weno5_minus(vm, eps, shock);
  else return weno7_plus(vp, eps, shock) + weno7_minus(vm, eps, shock);
}

}  // namespace cb2
