// Species thermodynamics of a thermally perfect mixture: NASA7 two-range polynomials (the
// Combustion2Part branch of src/Thermo.cu:386-632) or NASA9 multi-range polynomials (the
// HighTempMultiPart branch with therm_nasa_7_9 = 9, src/Thermo.cu:76-112, 201-238, 288-320,
// 352-384), chosen by the mechanism; and the Roe-state "characteristic thermo" helper
// (src/Thermo.cuh:49-110).  Coefficients are read from the device copy of the mechanism;
// outside the fitted range the enthalpy is extended linearly with the edge cp and cp is held
// constant, as the reference does.
#pragma once
#include "common.cuh"

namespace cb2 {

// NASA9: the range of species s that holds t, or the edge range and its boundary outside.
__device__ __forceinline__ const double *nasa9_range(const Mech &m, int s, double t, double &tt, bool &outside) {
  const double *cut = m.t_cut + s * (m.max_range + 1);
  const int n = __ldg(m.n_range + s);
  const double *a = m.poly9 + s * m.max_range * 9;
  outside = true;
  if (t < __ldg(cut)) { tt = __ldg(cut); return a; }
  if (t > __ldg(cut + n)) { tt = __ldg(cut + n); return a + (n - 1) * 9; }
  outside = false;
  tt = t;
  int j = n - 1;
  for (int r = 0; r < n; ++r)
    if (__ldg(cut + r) <= t && t <= __ldg(cut + r + 1)) { j = r; break; }
  return a + j * 9;
}

// NASA9 h/R at tt (1/tt and ln tt given) and cp/R at tt (1/tt^2 and 1/tt given)
__device__ __forceinline__ double nasa9_h(const double *a, double tt, double itt, double lntt) {
  const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt5 = tt4 * tt;
  return -__ldg(a + 0) * itt + __ldg(a + 1) * lntt + __ldg(a + 2) * tt + 0.5 * __ldg(a + 3) * tt2 +
         __ldg(a + 4) * tt3 / 3 + 0.25 * __ldg(a + 5) * tt4 + 0.2 * __ldg(a + 6) * tt5 + __ldg(a + 7);
}
__device__ __forceinline__ double nasa9_cp(const double *a, double tt, double itt2, double itt) {
  const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt;
  return __ldg(a + 0) * itt2 + __ldg(a + 1) * itt + __ldg(a + 2) + __ldg(a + 3) * tt + __ldg(a + 4) * tt2 +
         __ldg(a + 5) * tt3 + __ldg(a + 6) * tt4;
}

// NASA9 h_k and cp_k (compute_enthalpy_and_cp, src/Thermo.cu:201-238)
template <int NS>
__device__ __forceinline__ void nasa9_h_cp(double t, const Mech &m, double *h, double *cp) {
  const double it = 1.0 / t, lnt = log(t), it2 = it * it;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    double tt;
    bool outside;
    const double *a = nasa9_range(m, s, t, tt, outside);
    double hs, cps;
    if (outside) {
      const double tt2 = tt * tt, itt2 = 1.0 / tt2, itt = 1.0 / tt;
      cps = nasa9_cp(a, tt, itt2, itt);
      hs = nasa9_h(a, tt, itt, log(tt)) + cps * (t - tt);
    } else {
      hs = nasa9_h(a, t, it, lnt);
      cps = nasa9_cp(a, t, it2, it);
    }
    cp[s] = cps * __ldg(m.gas_const + s);
    h[s] = hs * __ldg(m.gas_const + s);
  }
}

// NASA9 g_k/(R_k T) (compute_gibbs_div_rt, src/Thermo.cu:352-384)
template <int NS>
__device__ __forceinline__ void nasa9_gibbs_rt(double t, const Mech &m, double *g) {
  const double it = 1.0 / t, lnt = log(t), it2 = it * it;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    double tt;
    bool outside;
    const double *a = nasa9_range(m, s, t, tt, outside);
    double itt = it, lntt = lnt, itt2 = it2;
    if (outside) {
      itt = 1 / tt;
      lntt = log(tt);
      itt2 = itt * itt;
    }
    const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt;
    g[s] = -0.5 * __ldg(a + 0) * itt2 + __ldg(a + 1) * itt * (lntt + 1) + __ldg(a + 2) * (1.0 - lntt) -
           0.5 * __ldg(a + 3) * tt - __ldg(a + 4) * tt2 / 6.0 - __ldg(a + 5) * tt3 / 12.0 -
           __ldg(a + 6) * tt4 * 0.05 + __ldg(a + 7) * itt - __ldg(a + 8);
  }
}

// h_k [J/kg] and cp_k [J/(kg K)] of every species at temperature t
// (compute_enthalpy_and_cp, src/Thermo.cu:453-523).
template <int NS>
__device__ __forceinline__ void species_h_cp(double t, const Mech &m, double *h, double *cp) {
  if (m.nasa9) {
    nasa9_h_cp<NS>(t, m, h, cp);
    return;
  }
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const double tl = __ldg(m.t_low + s), th = __ldg(m.t_high + s);
    if (t < tl || t > th) {
      const double tt = t < tl ? tl : th;
      const double *c = (t < tl ? m.lo : m.hi) + s * 7;
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt5 = tt4 * tt;
      double hs = __ldg(c + 0) * tt + 0.5 * __ldg(c + 1) * tt2 + __ldg(c + 2) * tt3 / 3 + 0.25 * __ldg(c + 3) * tt4 +
                  0.2 * __ldg(c + 4) * tt5 + __ldg(c + 5);
      const double cps = __ldg(c + 0) + __ldg(c + 1) * tt + __ldg(c + 2) * tt2 + __ldg(c + 3) * tt3 + __ldg(c + 4) * tt4;
      hs += cps * (t - tt);
      h[s] = hs * __ldg(m.gas_const + s);
      cp[s] = cps * __ldg(m.gas_const + s);
    } else {
      const double *c = (t < __ldg(m.t_mid + s) ? m.lo : m.hi) + s * 7;
      const double hs = __ldg(c + 0) * t + 0.5 * __ldg(c + 1) * t2 + __ldg(c + 2) * t3 / 3 + 0.25 * __ldg(c + 3) * t4 +
                        0.2 * __ldg(c + 4) * t5 + __ldg(c + 5);
      const double cps = __ldg(c + 0) + __ldg(c + 1) * t + __ldg(c + 2) * t2 + __ldg(c + 3) * t3 + __ldg(c + 4) * t4;
      h[s] = hs * __ldg(m.gas_const + s);
      cp[s] = cps * __ldg(m.gas_const + s);
    }
  }
}

// h_k only (compute_enthalpy, src/Thermo.cu:386-451).
template <int NS>
__device__ __forceinline__ void species_h(double t, const Mech &m, double *h) {
  if (m.nasa9) {
    double cp[NS];
    nasa9_h_cp<NS>(t, m, h, cp);
    return;
  }
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const double tl = __ldg(m.t_low + s), th = __ldg(m.t_high + s);
    double hs;
    if (t < tl || t > th) {
      const double tt = t < tl ? tl : th;
      const double *c = (t < tl ? m.lo : m.hi) + s * 7;
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt5 = tt4 * tt;
      hs = __ldg(c + 0) * tt + 0.5 * __ldg(c + 1) * tt2 + __ldg(c + 2) * tt3 / 3 + 0.25 * __ldg(c + 3) * tt4 +
           0.2 * __ldg(c + 4) * tt5 + __ldg(c + 5);
      const double cps = __ldg(c + 0) + __ldg(c + 1) * tt + __ldg(c + 2) * tt2 + __ldg(c + 3) * tt3 + __ldg(c + 4) * tt4;
      hs += cps * (t - tt);
    } else {
      const double *c = (t < __ldg(m.t_mid + s) ? m.lo : m.hi) + s * 7;
      hs = __ldg(c + 0) * t + 0.5 * __ldg(c + 1) * t2 + __ldg(c + 2) * t3 / 3 + 0.25 * __ldg(c + 3) * t4 +
           0.2 * __ldg(c + 4) * t5 + __ldg(c + 5);
    }
    h[s] = hs * __ldg(m.gas_const + s);
  }
}

// cp_k only (compute_cp, src/Thermo.cu:525-574).
template <int NS>
__device__ __forceinline__ void species_cp(double t, const Mech &m, double *cp) {
  if (m.nasa9) {
    double h[NS];
    nasa9_h_cp<NS>(t, m, h, cp);
    return;
  }
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const double tl = __ldg(m.t_low + s), th = __ldg(m.t_high + s);
    double tt = t;
    const double *c;
    if (t < tl) { tt = tl; c = m.lo + s * 7; }
    else if (t > th) { tt = th; c = m.hi + s * 7; }
    else c = (t < __ldg(m.t_mid + s) ? m.lo : m.hi) + s * 7;
    double cps;
    if (tt == t) cps = __ldg(c + 0) + __ldg(c + 1) * t + __ldg(c + 2) * t2 + __ldg(c + 3) * t3 + __ldg(c + 4) * t4;
    else {
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt;
      cps = __ldg(c + 0) + __ldg(c + 1) * tt + __ldg(c + 2) * tt2 + __ldg(c + 3) * tt3 + __ldg(c + 4) * tt4;
    }
    cp[s] = cps * __ldg(m.gas_const + s);
  }
}

// g_k/(R_k T) of every species (compute_gibbs_div_rt, src/Thermo.cu:576-632, NASA7 branch);
// outside [t_low, t_high] the polynomial is evaluated at the range edge.
template <int NS>
__device__ __forceinline__ void species_gibbs_rt(double t, const Mech &m, double *g) {
  if (m.nasa9) {
    nasa9_gibbs_rt<NS>(t, m, g);
    return;
  }
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t_inv = 1 / t, log_t = log(t);
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const double tl = __ldg(m.t_low + s), th = __ldg(m.t_high + s);
    if (t < tl || t > th) {
      const double tt = t < tl ? tl : th;
      const double *c = (t < tl ? m.lo : m.hi) + s * 7;
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt_inv = 1 / tt, log_tt = log(tt);
      g[s] = __ldg(c + 0) * (1.0 - log_tt) - 0.5 * __ldg(c + 1) * tt - __ldg(c + 2) * tt2 / 6.0 -
             __ldg(c + 3) * tt3 / 12.0 - __ldg(c + 4) * tt4 * 0.05 + __ldg(c + 5) * tt_inv - __ldg(c + 6);
    } else {
      const double *c = (t < __ldg(m.t_mid + s) ? m.lo : m.hi) + s * 7;
      g[s] = __ldg(c + 0) * (1.0 - log_t) - 0.5 * __ldg(c + 1) * t - __ldg(c + 2) * t2 / 6.0 -
             __ldg(c + 3) * t3 / 12.0 - __ldg(c + 4) * t4 * 0.05 + __ldg(c + 5) * t_inv - __ldg(c + 6);
    }
  }
}

// Mixture gamma and sound speed at the Roe state, plus the scalar rows of the left
// eigenvectors (alpha_s) and the energy coefficients of the right eigenvectors
// (src/Thermo.cuh:49-110 with two_temperature off: e_ve = 0).
template <int NS>
__device__ __forceinline__ void characteristic_thermo(double t, const double *y, const Mech &m, double &gamma,
                                                      double &c, double *alpha, double *ecoef, double *e_tr_out) {
  const double te = fmax(t, 1.0);
  double h[NS], cp[NS];
  species_h_cp<NS>(te, m, h, cp);
  double e_tr = 0, r = 0, cpm = 0, cvm = 0;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const double rs = __ldg(m.gas_const + s);
    e_tr += y[s] * (h[s] - rs * te);
    r += y[s] * rs;
    cpm += y[s] * cp[s];
    cvm += y[s] * (cp[s] - rs);
  }
  gamma = cpm / fmax(cvm, 1e-8);
  c = sqrt(fmax(gamma * r * te, 1e-12));
  if (e_tr_out) *e_tr_out = e_tr;
  if (alpha) {
    const double gm1 = gamma - 1.0;
    const double c2 = fmax(c * c, 1e-30);
    const double inv_gm1 = 1.0 / fmax(gm1, 1e-12);
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const double a = (gamma * __ldg(m.gas_const + s) * te - gm1 * h[s]) / c2;
      alpha[s] = a;
      ecoef[s] = -a * c2 * inv_gm1;
    }
  }
}

// FP32 twins of species_h_cp and characteristic_thermo for the NASA7 tables (the mixed form's
// reconstructed and Roe states; its temperature inversions stay FP64).  Same formulas and branch
// structure, coefficients rounded to FP32.
template <int NS>
__device__ __forceinline__ void species_h_cp_f32(float t, const Mech &m, float *h, float *cp) {
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const float tl = float(__ldg(m.t_low + s)), th = float(__ldg(m.t_high + s));
    const bool out = t < tl || t > th;
    const float tt = out ? (t < tl ? tl : th) : t;
    const double *c = (out ? (t < tl) : (t < float(__ldg(m.t_mid + s)))) ? m.lo + s * 7 : m.hi + s * 7;
    const float c0 = float(__ldg(c + 0)), c1 = float(__ldg(c + 1)), c2 = float(__ldg(c + 2)), c3 = float(__ldg(c + 3));
    const float c4 = float(__ldg(c + 4)), c5 = float(__ldg(c + 5));
    // Horner forms of h/R = a0 T + a1 T^2/2 + a2 T^3/3 + a3 T^4/4 + a4 T^5/5 + a5 and cp/R
    float hs = tt * (c0 + tt * (0.5f * c1 + tt * (c2 * (1.0f / 3) + tt * (0.25f * c3 + tt * (0.2f * c4))))) + c5;
    const float cps = c0 + tt * (c1 + tt * (c2 + tt * (c3 + tt * c4)));
    if (out) hs += cps * (t - tt);
    const float r = float(__ldg(m.gas_const + s));
    h[s] = hs * r;
    cp[s] = cps * r;
  }
}

template <int NS>
__device__ __forceinline__ void characteristic_thermo_f32(float t, const float *y, const Mech &m, float &gamma,
                                                          float &c, float *alpha, float *ecoef, float *e_tr_out) {
  const float te = fmaxf(t, 1.0f);
  float h[NS], cp[NS];
  species_h_cp_f32<NS>(te, m, h, cp);
  float e_tr = 0, r = 0, cpm = 0, cvm = 0;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const float rs = float(__ldg(m.gas_const + s));
    e_tr += y[s] * (h[s] - rs * te);
    r += y[s] * rs;
    cpm += y[s] * cp[s];
    cvm += y[s] * (cp[s] - rs);
  }
  gamma = cpm / fmaxf(cvm, 1e-8f);
  c = sqrtf(fmaxf(gamma * r * te, 1e-12f));
  if (e_tr_out) *e_tr_out = e_tr;
  if (alpha) {
    const float gm1 = gamma - 1.0f;
    const float c2 = fmaxf(c * c, 1e-30f);
    const float inv_gm1 = 1.0f / fmaxf(gm1, 1e-12f);
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const float a = (gamma * float(__ldg(m.gas_const + s)) * te - gm1 * h[s]) / c2;
      alpha[s] = a;
      ecoef[s] = -a * c2 * inv_gm1;
    }
  }
}

}  // namespace cb2
