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
// FP32 path normalises by the smallest term instead, and takes every ratio before squaring so
// that nothing underflows: with A_s = eps + beta_s (D_s = A_s^2), q_s = (A_min / A_s)^2 in (0, 1],
// T = |b0 + 3 b1 - 3 b2 - b3| (tau = T^2) and t = 1 / (1 + (A_min / T)^2) = tau / (D_min + tau),
//   WENO-JS  alpha_s ~ c_s q_s,   WENO-Z  alpha_s ~ c_s ((1 - t) + t q_s),
// the same weights up to a common factor, every term bounded by c_s.  (The square of a small A_s,
// e.g. eps + 0 for a uniform density of 0.3, is below the smallest normal FP32 number, and the
// paired FP32 instructions flush such results to zero.)
// The reciprocal is the hardware approximation (rcp.approx, within 1 ulp): 1/0 = inf and
// 1/inf = 0 as the formulas above require.
__device__ __forceinline__ float rcp32(float x) { return __fdividef(1.0f, x); }

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
    const T A0 = eps + b0, A1 = eps + b1, A2 = eps + b2;
    const T Am = fmin(fmin(A0, A1), A2);
    E0 = sq(Am * rcp32(A0)); E1 = sq(Am * rcp32(A1)); E2 = sq(Am * rcp32(A2));
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
    const T A0 = eps + b0, A1 = eps + b1, A2 = eps + b2, A3 = eps + b3;
    const T Am = fmin(fmin(A0, A1), fmin(A2, A3));
    const T rz = Am * rcp32(fabs(b0 + 3 * b1 - 3 * b2 - b3));
    const T t = rcp32(1 + rz * rz), u = 1 - t;
    E0 = u + t * sq(Am * rcp32(A0)); E1 = u + t * sq(Am * rcp32(A1));
    E2 = u + t * sq(Am * rcp32(A2)); E3 = u + t * sq(Am * rcp32(A3));
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

// ---- packed FP32 node-centred pair ------------------------------------------------------
// The minus side is the plus formula applied to the mirrored stencil, so both sides run as one
// stream of float2 values through the sm_100 paired FP32 instructions (FFMA2, FADD2, FMUL2):
// lane x is the plus side on u[k], lane y the minus side on u[last - k].  Mirroring maps the
// plus sub-stencil r onto sub-stencil last - r, so the packed indicators of the first half of
// the sub-stencils carry the others in lane y.  Per lane the arithmetic is the FP32 node form
// above (D_min normalisation), with the final division done as a reciprocal and a product.
__device__ __forceinline__ float2 p2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 swap2(float2 a) { return make_float2(a.y, a.x); }
__device__ __forceinline__ float2 rcp2(float2 a) { return make_float2(rcp32(a.x), rcp32(a.y)); }
// c0 a + c1 b + c2 c (+ c3 d) with scalar coefficients
__device__ __forceinline__ float2 lin3(float c0, float2 a, float c1, float2 b, float c2, float2 c) {
  return fma2(p2(c2), c, fma2(p2(c1), b, mul2(p2(c0), a)));
}
__device__ __forceinline__ float2 lin4(float c0, float2 a, float c1, float2 b, float c2, float2 c, float c3,
                                       float2 d) {
  return fma2(p2(c3), d, lin3(c0, a, c1, b, c2, c));
}
__device__ __forceinline__ float2 beta7_x2(float2 d1, float2 d2, float2 d3) {
  // d1^2 + 13/12 d2^2 + 1043/960 d3^2 + d1 d3/12; invariant under (d1, d3) -> (-d1, -d3), the
  // sign change that mirroring gives the first and third differences
  const float2 t = fma2(p2(1.0f / 12), d3, d1);
  return fma2(p2(1043.0f / 960), mul2(d3, d3), fma2(p2(13.0f / 12), mul2(d2, d2), mul2(d1, t)));
}

__device__ __forceinline__ void weno5_node_x2(const float *v, float eps, float &lp, float &rm) {
  const float2 U0 = make_float2(v[0], v[4]), U1 = make_float2(v[1], v[3]), U2 = p2(v[2]);
  const float2 U3 = make_float2(v[3], v[1]), U4 = make_float2(v[4], v[0]);
  const float k6 = 1.0f / 6;
  const float2 Q0 = lin3(2 * k6, U0, -7 * k6, U1, 11 * k6, U2);  // (q0, m0)
  const float2 Q1 = lin3(-k6, U1, 5 * k6, U2, 2 * k6, U3);       // (q1, m1)
  const float2 Q2 = lin3(2 * k6, U2, 5 * k6, U3, -k6, U4);       // (q2, m2)
  const float2 e0 = lin3(1, U0, -2, U1, 1, U2), f0 = lin3(1, U0, -4, U1, 3, U2);
  const float2 B0 = fma2(p2(13.0f / 12), mul2(e0, e0), mul2(p2(0.25f), mul2(f0, f0)));  // (b0, b2)
  const float e1 = v[1] + v[3] - 2 * v[2], f1 = v[1] - v[3];
  const float b1 = 13.0f / 12 * (e1 * e1) + 0.25f * (f1 * f1);
  const float2 AA = add2(p2(eps), B0);  // (A0, A2)
  const float A1 = eps + b1;
  const float Am = fminf(fminf(AA.x, AA.y), A1);
  const float2 RA = mul2(p2(Am), rcp2(AA));
  const float2 EA = mul2(RA, RA);  // (E0, E2)
  const float R1 = Am * rcp32(A1), E1 = R1 * R1;
  const float2 W0 = mul2(p2(0.1f), EA), W1 = p2(0.6f * E1), W2 = mul2(p2(0.3f), swap2(EA));
  const float2 num = fma2(W2, Q2, fma2(W1, Q1, mul2(W0, Q0)));
  const float2 den = add2(add2(W0, W1), W2);
  const float2 r = mul2(num, rcp2(den));
  lp = r.x;
  rm = r.y;
}

__device__ __forceinline__ void weno7_node_x2(const float *u, float eps, float &lp, float &rm) {
  float2 U[7];
#pragma unroll
  for (int k = 0; k < 7; ++k) U[k] = make_float2(u[k], u[6 - k]);
  const float2 Q0 = lin4(-3, U[0], 13, U[1], -23, U[2], 25, U[3]);  // (q0, m0)
  const float2 Q1 = lin4(1, U[1], -5, U[2], 13, U[3], 3, U[4]);
  const float2 Q2 = lin4(-1, U[2], 7, U[3], 7, U[4], -1, U[5]);
  const float2 Q3 = lin4(3, U[3], 13, U[4], -5, U[5], 1, U[6]);
  const float k6 = 1.0f / 6;
  const float2 B0 = beta7_x2(lin4(-2 * k6, U[0], 9 * k6, U[1], -18 * k6, U[2], 11 * k6, U[3]),
                             lin4(-1, U[0], 4, U[1], -5, U[2], 2, U[3]), lin4(-1, U[0], 3, U[1], -3, U[2], 1, U[3]));
  const float2 B1 = beta7_x2(lin4(k6, U[1], -6 * k6, U[2], 3 * k6, U[3], 2 * k6, U[4]), lin3(1, U[2], -2, U[3], 1, U[4]),
                             lin4(-1, U[1], 3, U[2], -3, U[3], 1, U[4]));
  // plus side: b0 = B0.x, b1 = B1.x, b2 = B1.y, b3 = B0.y
  const float2 A0 = add2(p2(eps), B0), A1 = add2(p2(eps), B1);  // (A0, A3), (A1, A2)
  const float Am = fminf(fminf(A0.x, A0.y), fminf(A1.x, A1.y));
  const float2 R0 = mul2(p2(Am), rcp2(A0)), R1 = mul2(p2(Am), rcp2(A1));
  // t = tau / (D_min + tau), tau unchanged by the mirroring; T = 0 gives rz = inf and t = 0
  const float rz = Am * rcp32(fabsf((B0.x - B0.y) + 3 * (B1.x - B1.y)));
  const float t = rcp32(1.0f + rz * rz);
  const float2 EA = fma2(p2(t), mul2(R0, R0), p2(1.0f - t));  // (E0, E3)
  const float2 EB = fma2(p2(t), mul2(R1, R1), p2(1.0f - t));  // (E1, E2)
  const float2 W0 = mul2(p2(1.0f / 35), EA), W1 = mul2(p2(12.0f / 35), EB);
  const float2 W2 = mul2(p2(18.0f / 35), swap2(EB)), W3 = mul2(p2(4.0f / 35), swap2(EA));
  const float2 num = fma2(W3, Q3, fma2(W2, Q2, fma2(W1, Q1, mul2(W0, Q0))));
  const float2 den = add2(add2(W0, W1), add2(W2, W3));
  const float2 r = mul2(mul2(num, p2(1.0f / 12)), rcp2(den));
  lp = r.x;
  rm = r.y;
}

template <int ORDER, typename T>
__device__ __forceinline__ T weno_pm(const T *vp, const T *vm, T eps, bool shock) {
  if constexpr (ORDER == 5) return weno5_plus(vp, eps, shock) + weno5_minus(vm, eps, shock);
  else return weno7_plus(vp, eps, shock) + weno7_minus(vm, eps, shock);
}

}  // namespace cb2
