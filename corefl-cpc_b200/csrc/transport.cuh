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

template <int NS>
__device__ __forceinline__ void transport_properties(double t, double /*p*/, double mw_total, const double *y,
                                                     const double *cp, const Mech &m, double &mu, double &kappa,
                                                     double *rhoD) {
  constexpr double pi = 3.141592653589793;
  double X[NS], vs[NS];
  double st = sqrt(t);
#pragma unroll
  for (int l = 0; l < NS; ++l) {
    X[l] = y[l] * mw_total / __ldg(m.mw + l);
    const double tdl = t * __ldg(m.lj_inv + l);
    vs[l] = __ldg(m.vis_coeff + l) * st / (1.147 * pow(tdl, -0.145) + pow(tdl + 0.5, -2));
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
      const double rd = __ldg(m.bdc + a * NS + a) * t32 / (omega_d(t_red) * Ra * t);
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
      const double inv = omega_d(t * __ldg(m.kbe + l * NS + n)) / (__ldg(m.bdc + l * NS + n) * t32);
      dsum[l] += (X[n] + eps) * inv;
      dsum[n] += (X[l] + eps) * inv;
    }
  const double tinv = 1.0 / (t * kRu);
#pragma unroll
  for (int l = 0; l < NS; ++l) rhoD[l] = num[l] * tinv / dsum[l];
}

}  // namespace cb2
