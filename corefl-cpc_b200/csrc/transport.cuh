// Mixture-averaged transport properties (compute_transport_property, src/Transport.cu:43-150;
// compute_Omega_D, src/Transport.cu:182-184):
//  * species viscosity from the Lennard-Jones collision integral fit,
//  * Wilke mixing rule for mu,
//  * species conductivity with the Warnatz rotational/vibrational correction for linear and
//    non-linear molecules, mixed with the 1.065/0.065 denominator of the reference,
//  * mixture-averaged rho*D_k from binary diffusivities (the pressure cancels, so it is not
//    needed).
#pragma once
#include "common.cuh"

namespace cb2 {

__device__ __forceinline__ double omega_d(double t_red) {
  return 1.0548 * pow(t_red, -0.15504) + pow(t_red + 0.55909, -2.1705);
}

// Omega_D at the reduced temperature t_red = T k, given ln t_red = ln T + ln k: the first power
// as one exponential, the shifted one as exp(a ln(t_red + c)) -- the same values as pow to a few
// ulp, at about a third of the cost.
__device__ __forceinline__ double omega_d_ln(double t_red, double ln_t_red) {
  return 1.0548 * exp(-0.15504 * ln_t_red) + exp(-2.1705 * log(t_red + 0.55909));
}

template <int NS>
__device__ __forceinline__ void transport_properties(double t, double /*p*/, double mw_total, const double *y,
                                                     const double *cp, const Mech &m, double &mu, double &kappa,
                                                     double *rhoD) {
  constexpr double pi = 3.141592653589793;
  double X[NS], vs[NS];
  double st = sqrt(t);
  const bool use_ln = m.transport_ln != 0;
  const double lnt = use_ln ? log(t) : 0.0;
  auto omega = [&](double t_red, int pair) {
    return use_ln ? omega_d_ln(t_red, lnt + __ldg(m.ln_kbe + pair)) : omega_d(t_red);
  };
#pragma unroll
  for (int l = 0; l < NS; ++l) {
    X[l] = y[l] * mw_total / __ldg(m.mw + l);
    const double tdl = t * __ldg(m.lj_inv + l);
    const double q = tdl + 0.5;
    const double a = use_ln ? exp(-0.145 * (lnt + __ldg(m.ln_lj_inv + l))) : pow(tdl, -0.145);
    vs[l] = __ldg(m.vis_coeff + l) * st / (1.147 * a + 1.0 / (q * q));
  }
  const double t32 = t * st;
  double visc = 0, cond = 0;
#pragma unroll
  for (int a = 0; a < NS; ++a) {
    const double Ra = __ldg(m.gas_const + a);
    double lambda = 15 * 0.25 * vs[a] * Ra;
    const double geom = __ldg(m.geometry + a);
    if (geom == 1 || geom == 2) {
      const double t_red = t * __ldg(m.kbe + a * NS + a);
      const double tri = 1 / t_red;
      const double tmp = sqrt(tri * pi) * pi;
      const double FT = 1 + 0.5 * tmp + (2 + 0.25 * pi * pi) * tri + tmp * tri;
      const double rd = __ldg(m.bdc + a * NS + a) * t32 / (omega(t_red, a * NS + a) * Ra * t);
      if (geom == 1) {
        const double adpb = (2.5 * vs[a] - rd) / ((pi * __ldg(m.zrot + a) / FT * vs[a] + 10.0 / 3 * vs[a] + 2.0 * rd));
        lambda += -5 * adpb * vs[a] * Ra + rd * cp[a] + rd * (2 * adpb - 2.5) * Ra;
      } else {
        const double adpb = (2.5 * vs[a] - rd) / ((pi * __ldg(m.zrot + a) / FT * vs[a] + 5 * vs[a] + 2.0 * rd));
        lambda += -7.5 * adpb * vs[a] * Ra + rd * cp[a] + rd * (3 * adpb - 2.5) * Ra;
      }
    }
    double den = 0;
    const double sva = sqrt(vs[a]);
#pragma unroll
    for (int b = 0; b < NS; ++b) {
      double phi = 1.0;
      if (a != b) {
        const double num = 1.0 + rsqrt(vs[b]) * (sva * __ldg(m.wjwi14 + a * NS + b));
        phi = num * num * __ldg(m.sqwiwj8 + a * NS + b);
      }
      den += phi * X[b];
    }
    visc += vs[a] * X[a] / den;
    cond += lambda * X[a] / (1.065 * den - 0.065 * X[a]);
  }
  mu = visc;
  kappa = cond;
  // mixture-averaged diffusivity
  constexpr double eps = 1e-12;
  double num[NS], dsum[NS], sum = 0;
#pragma unroll
  for (int l = 0; l < NS; ++l) {
    num[l] = (X[l] + eps) * __ldg(m.mw + l);
    sum += num[l];
    dsum[l] = 0;
  }
#pragma unroll
  for (int l = 0; l < NS; ++l) num[l] = sum - num[l];
#pragma unroll
  for (int l = 0; l < NS; ++l)
#pragma unroll
    for (int n = l + 1; n < NS; ++n) {
      const double inv = omega(t * __ldg(m.kbe + l * NS + n), l * NS + n) / (__ldg(m.bdc + l * NS + n) * t32);
      dsum[l] += (X[n] + eps) * inv;
      dsum[n] += (X[l] + eps) * inv;
    }
  const double tinv = 1.0 / (t * kRu);
#pragma unroll
  for (int l = 0; l < NS; ++l) rhoD[l] = num[l] * tinv / dsum[l];
}

// The same mixture-averaged transport in FP32 for the mixed form (transport is not among the
// quantities that form keeps in FP64: the temperature inversions, the Arrhenius and Gibbs
// exponentials, the point-implicit solve and the state).  Inputs and outputs stay FP64; the powers
// are FP32 expf / logf (a few ulp), the rest FP32 arithmetic in the order of the FP64 version.
__device__ __forceinline__ float omega_d_f32(float t_red, float ln_t_red) {
  return 1.0548f * expf(-0.15504f * ln_t_red) + expf(-2.1705f * logf(t_red + 0.55909f));
}

template <int NS>
__device__ __forceinline__ void transport_properties_f32(double t64, double mw_total, const double *y,
                                                         const double *cp, const Mech &m, double &mu,
                                                         double &kappa, double *rhoD) {
  constexpr float pi = 3.14159265358979f;
  const float t = float(t64);
  float X[NS], vs[NS];
  const float st = sqrtf(t);
  // ln of the reduced temperatures: ln T + ln k from the tables, or ln(T k)
  const bool use_ln = m.transport_ln != 0;
  const float lnt = logf(t);
  auto ln_red = [&](float t_red, int pair) { return use_ln ? lnt + float(__ldg(m.ln_kbe + pair)) : logf(t_red); };
#pragma unroll
  for (int l = 0; l < NS; ++l) {
    X[l] = float(y[l] * mw_total / __ldg(m.mw + l));
    const float tdl = t * float(__ldg(m.lj_inv + l));
    const float q = tdl + 0.5f;
    const float lnd = use_ln ? lnt + float(__ldg(m.ln_lj_inv + l)) : logf(tdl);
    vs[l] = float(__ldg(m.vis_coeff + l)) * st / (1.147f * expf(-0.145f * lnd) + 1.0f / (q * q));
  }
  const float t32 = t * st;
  float visc = 0, cond = 0;
#pragma unroll
  for (int a = 0; a < NS; ++a) {
    const float Ra = float(__ldg(m.gas_const + a));
    float lambda = 15 * 0.25f * vs[a] * Ra;
    const double geom = __ldg(m.geometry + a);
    if (geom == 1 || geom == 2) {
      const float t_red = t * float(__ldg(m.kbe + a * NS + a));
      const float tri = 1 / t_red;
      const float tmp = sqrtf(tri * pi) * pi;
      const float FT = 1 + 0.5f * tmp + (2 + 0.25f * pi * pi) * tri + tmp * tri;
      const float rd = float(__ldg(m.bdc + a * NS + a)) * t32 / (omega_d_f32(t_red, ln_red(t_red, a * NS + a)) * Ra * t);
      const float zr = float(__ldg(m.zrot + a));
      if (geom == 1) {
        const float adpb = (2.5f * vs[a] - rd) / ((pi * zr / FT * vs[a] + 10.0f / 3 * vs[a] + 2.0f * rd));
        lambda += -5 * adpb * vs[a] * Ra + rd * float(cp[a]) + rd * (2 * adpb - 2.5f) * Ra;
      } else {
        const float adpb = (2.5f * vs[a] - rd) / ((pi * zr / FT * vs[a] + 5 * vs[a] + 2.0f * rd));
        lambda += -7.5f * adpb * vs[a] * Ra + rd * float(cp[a]) + rd * (3 * adpb - 2.5f) * Ra;
      }
    }
    float den = 0;
    const float sva = sqrtf(vs[a]);
#pragma unroll
    for (int b = 0; b < NS; ++b) {
      float phi = 1.0f;
      if (a != b) {
        const float num = 1.0f + rsqrtf(vs[b]) * (sva * float(__ldg(m.wjwi14 + a * NS + b)));
        phi = num * num * float(__ldg(m.sqwiwj8 + a * NS + b));
      }
      den += phi * X[b];
    }
    visc += vs[a] * X[a] / den;
    cond += lambda * X[a] / (1.065f * den - 0.065f * X[a]);
  }
  mu = visc;
  kappa = cond;
  constexpr float eps = 1e-12f;
  float num[NS], dsum[NS], sum = 0;
#pragma unroll
  for (int l = 0; l < NS; ++l) {
    num[l] = (X[l] + eps) * float(__ldg(m.mw + l));
    sum += num[l];
    dsum[l] = 0;
  }
#pragma unroll
  for (int l = 0; l < NS; ++l) num[l] = sum - num[l];
#pragma unroll
  for (int l = 0; l < NS; ++l)
#pragma unroll
    for (int n = l + 1; n < NS; ++n) {
      const float t_red = t * float(__ldg(m.kbe + l * NS + n));
      const float inv = omega_d_f32(t_red, ln_red(t_red, l * NS + n)) / (float(__ldg(m.bdc + l * NS + n)) * t32);
      dsum[l] += (X[n] + eps) * inv;
      dsum[n] += (X[l] + eps) * inv;
    }
  const float tinv = 1.0f / (t * float(kRu));
#pragma unroll
  for (int l = 0; l < NS; ++l) rhoD[l] = num[l] * tinv / dsum[l];
}

}  // namespace cb2
