// FP64 host oracle (see oracle.hpp).  TEST INFRASTRUCTURE ONLY.
#include "oracle.hpp"
#include <array>
#include <cmath>
#include <cstring>
#include <cstdio>

namespace oracle {

namespace {

inline double sqr(double x) { return x * x; }

// ---------------------------------------------------------------------------------------
// Thermodynamics, NASA9 multi-range (the HighTempMultiPart build with therm_nasa_7_9 = 9:
// compute_enthalpy src/Thermo.cu:76-112, compute_enthalpy_and_cp :201-238, compute_cp
// :288-320, compute_gibbs_div_rt :352-384).  Outside the first / last boundary the polynomial
// is evaluated at the boundary; h is then extended linearly with that cp.
// ---------------------------------------------------------------------------------------
struct Range9 {
  const double *a;  // a0..a6, b1, b2 of the range used
  double tt;        // evaluation temperature (t, or the boundary outside)
  bool outside;
};

Range9 range9(const Mechanism &m, int s, double t) {
  const double *cut = m.t_cut.data() + s * (m.max_range + 1);
  const int n = m.n_range[s];
  const double *a = m.poly9.data() + (size_t)s * m.max_range * 9;
  if (t < cut[0]) return {a, cut[0], true};
  if (t > cut[n]) return {a + (n - 1) * 9, cut[n], true};
  int j = n - 1;
  for (int r = 0; r < n; ++r)
    if (cut[r] <= t && t <= cut[r + 1]) {
      j = r;
      break;
    }
  return {a + j * 9, t, false};
}

// h/R at tt with 1/tt and ln tt given
double h9(const double *a, double tt, double itt, double lntt) {
  const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt5 = tt4 * tt;
  return -a[0] * itt + a[1] * lntt + a[2] * tt + 0.5 * a[3] * tt2 + a[4] * tt3 / 3 + 0.25 * a[5] * tt4 +
         0.2 * a[6] * tt5 + a[7];
}
// cp/R at tt with 1/tt^2 and 1/tt given
double cp9(const double *a, double tt, double itt2, double itt) {
  const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt;
  return a[0] * itt2 + a[1] * itt + a[2] + a[3] * tt + a[4] * tt2 + a[5] * tt3 + a[6] * tt4;
}

void nasa9_h_cp(double t, const Mechanism &m, double *h, double *cp) {
  const double it = 1.0 / t, lnt = std::log(t), it2 = it * it;
  for (int i = 0; i < m.n_spec; ++i) {
    const Range9 r = range9(m, i, t);
    if (r.outside) {
      const double tt2 = r.tt * r.tt, itt2 = 1.0 / tt2, itt = 1.0 / r.tt;
      const double c = cp9(r.a, r.tt, itt2, itt);
      h[i] = h9(r.a, r.tt, itt, std::log(r.tt)) + c * (t - r.tt);
      cp[i] = c;
    } else {
      h[i] = h9(r.a, t, it, lnt);
      cp[i] = cp9(r.a, t, it2, it);
    }
    cp[i] *= m.gas_const[i];
    h[i] *= m.gas_const[i];
  }
}

void nasa9_gibbs_rt(double t, const Mechanism &m, double *g) {
  const double it = 1.0 / t, lnt = std::log(t), it2 = it * it;
  for (int i = 0; i < m.n_spec; ++i) {
    const Range9 r = range9(m, i, t);
    double itt = it, lntt = lnt, itt2 = it2;
    if (r.outside) {
      itt = 1 / r.tt;
      lntt = std::log(r.tt);
      itt2 = itt * itt;
    }
    const double tt = r.tt, tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt;
    const double *a = r.a;
    g[i] = -0.5 * a[0] * itt2 + a[1] * itt * (lntt + 1) + a[2] * (1.0 - lntt) - 0.5 * a[3] * tt - a[4] * tt2 / 6.0 -
           a[5] * tt3 / 12.0 - a[6] * tt4 * 0.05 + a[7] * itt - a[8];
  }
}

// ---------------------------------------------------------------------------------------
// Thermodynamics, NASA7 two-range (src/Thermo.cu:386-574, Combustion2Part branch)
// ---------------------------------------------------------------------------------------
void nasa7_h(double t, const Mechanism &m, double *h) {
  if (m.nasa == 9) {
    double cp[16];
    nasa9_h_cp(t, m, h, cp);
    return;
  }
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
  for (int i = 0; i < m.n_spec; ++i) {
    if (t < m.t_low[i] || t > m.t_high[i]) {
      const double tt = t < m.t_low[i] ? m.t_low[i] : m.t_high[i];
      const double *c = (t < m.t_low[i] ? m.lo.data() : m.hi.data()) + 7 * i;
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt5 = tt4 * tt;
      h[i] = c[0] * tt + 0.5 * c[1] * tt2 + c[2] * tt3 / 3 + 0.25 * c[3] * tt4 + 0.2 * c[4] * tt5 + c[5];
      const double cp = c[0] + c[1] * tt + c[2] * tt2 + c[3] * tt3 + c[4] * tt4;
      h[i] += cp * (t - tt);
    } else {
      const double *c = (t < m.t_mid[i] ? m.lo.data() : m.hi.data()) + 7 * i;
      h[i] = c[0] * t + 0.5 * c[1] * t2 + c[2] * t3 / 3 + 0.25 * c[3] * t4 + 0.2 * c[4] * t5 + c[5];
    }
    h[i] *= m.gas_const[i];
  }
}

void nasa7_cp(double t, const Mechanism &m, double *cp) {
  if (m.nasa == 9) {
    double h[16];
    nasa9_h_cp(t, m, h, cp);
    return;
  }
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t;
  for (int i = 0; i < m.n_spec; ++i) {
    if (t < m.t_low[i] || t > m.t_high[i]) {
      const double tt = t < m.t_low[i] ? m.t_low[i] : m.t_high[i];
      const double *c = (t < m.t_low[i] ? m.lo.data() : m.hi.data()) + 7 * i;
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt;
      cp[i] = c[0] + c[1] * tt + c[2] * tt2 + c[3] * tt3 + c[4] * tt4;
    } else {
      const double *c = (t < m.t_mid[i] ? m.lo.data() : m.hi.data()) + 7 * i;
      cp[i] = c[0] + c[1] * t + c[2] * t2 + c[3] * t3 + c[4] * t4;
    }
    cp[i] *= m.gas_const[i];
  }
}

// Mixture gamma, c, alpha_s and energy coefficients at (t, y) (src/Thermo.cuh:49-110, 1T).
void characteristic_thermo(double t, const double *y, const Mechanism &m, double *gamma, double *c, double *alpha,
                           double *ecoef, double *e_tr_out) {
  const double te = std::max(t, 1.0);
  double h[16], cp[16];
  nasa7_h_cp(te, m, h, cp);
  double e_tr = 0, r = 0, cpm = 0, cvm = 0;
  for (int l = 0; l < m.n_spec; ++l) {
    e_tr += y[l] * (h[l] - m.gas_const[l] * te);
    r += y[l] * m.gas_const[l];
    cpm += y[l] * cp[l];
    cvm += y[l] * (cp[l] - m.gas_const[l]);
  }
  const double g = cpm / std::max(cvm, 1e-8);
  const double cc = std::sqrt(std::max(g * r * te, 1e-12));
  *gamma = g;
  *c = cc;
  if (e_tr_out) *e_tr_out = e_tr;
  if (alpha) {
    const double gm1 = g - 1.0;
    const double c2 = std::max(cc * cc, 1e-30);
    const double inv_gm1 = 1.0 / std::max(gm1, 1e-12);
    for (int l = 0; l < m.n_spec; ++l) {
      const double a = (g * m.gas_const[l] * te - gm1 * h[l]) / c2;
      alpha[l] = a;
      ecoef[l] = -a * c2 * inv_gm1;
    }
  }
}

// ---------------------------------------------------------------------------------------
// WENO (src/WENO.cu:3033-3196)
// ---------------------------------------------------------------------------------------
// Plus side of WENO5 at i+1/2 from vp[0..4] (vp[2] = node i), src/WENO.cu:3035-3052.
double weno5_plus(const double *vp, double eps, bool if_shock) {
  const double one6th = 1.0 / 6;
  const double v0 = one6th * (2 * vp[2] + 5 * vp[3] - vp[4]);
  const double v1 = one6th * (-vp[1] + 5 * vp[2] + 2 * vp[3]);
  const double v2 = one6th * (2 * vp[0] - 7 * vp[1] + 11 * vp[2]);
  if (!if_shock) return 0.3 * v0 + 0.6 * v1 + 0.1 * v2;
  const double k13 = 13.0 / 12;
  const double b0 = k13 * sqr(vp[2] + vp[4] - 2 * vp[3]) + 0.25 * sqr(3 * vp[2] - 4 * vp[3] + vp[4]);
  const double b1 = k13 * sqr(vp[1] + vp[3] - 2 * vp[2]) + 0.25 * sqr(vp[1] - vp[3]);
  const double b2 = k13 * sqr(vp[0] + vp[2] - 2 * vp[1]) + 0.25 * sqr(vp[0] - 4 * vp[1] + 3 * vp[2]);
  const double a0 = 0.3 / sqr(eps + b0), a1 = 0.6 / sqr(eps + b1), a2 = 0.1 / sqr(eps + b2);
  return (a0 * v0 + a1 * v1 + a2 * v2) / (a0 + a1 + a2);
}

// Minus side of WENO5 at i+1/2 from vm[0..4] (vm[1] = node i), src/WENO.cu:3054-3072.
double weno5_minus(const double *vm, double eps, bool if_shock) {
  const double one6th = 1.0 / 6;
  const double v0 = one6th * (11 * vm[2] - 7 * vm[3] + 2 * vm[4]);
  const double v1 = one6th * (2 * vm[1] + 5 * vm[2] - vm[3]);
  const double v2 = one6th * (-vm[0] + 5 * vm[1] + 2 * vm[2]);
  if (!if_shock) return 0.1 * v0 + 0.6 * v1 + 0.3 * v2;
  const double k13 = 13.0 / 12;
  const double b0 = k13 * sqr(vm[2] + vm[4] - 2 * vm[3]) + 0.25 * sqr(3 * vm[2] - 4 * vm[3] + vm[4]);
  const double b1 = k13 * sqr(vm[1] + vm[3] - 2 * vm[2]) + 0.25 * sqr(vm[1] - vm[3]);
  const double b2 = k13 * sqr(vm[0] + vm[2] - 2 * vm[1]) + 0.25 * sqr(vm[0] - 4 * vm[1] + 3 * vm[2]);
  const double a0 = 0.1 / sqr(eps + b0), a1 = 0.6 / sqr(eps + b1), a2 = 0.3 / sqr(eps + b2);
  return (a0 * v0 + a1 * v1 + a2 * v2) / (a0 + a1 + a2);
}

double WENO5(const double *vp, const double *vm, double eps, bool if_shock) {
  return weno5_plus(vp, eps, if_shock) + weno5_minus(vm, eps, if_shock);
}

// One side of WENO7 with the reference's plus-side indexing (the minus side calls it with
// the mirrored stencil, which is what src/WENO.cu:3135-3173 writes out).
double weno7_one(const double *v, double eps, bool if_shock) {
  const double c0 = 1.0 / 35, c1 = 12.0 / 35, c2 = 18.0 / 35, c3 = 4.0 / 35, one12 = 1.0 / 12;
  const double q0 = -3 * v[0] + 13 * v[1] - 23 * v[2] + 25 * v[3];
  const double q1 = v[1] - 5 * v[2] + 13 * v[3] + 3 * v[4];
  const double q2 = -v[2] + 7 * v[3] + 7 * v[4] - v[5];
  const double q3 = 3 * v[3] + 13 * v[4] - 5 * v[5] + v[6];
  if (!if_shock) return one12 * (c0 * q0 + c1 * q1 + c2 * q2 + c3 * q3);
  const double one6 = 1.0 / 6, d12 = 13.0 / 12.0, d13 = 1043.0 / 960, d14 = 1.0 / 12;
  auto beta = [&](double s1, double s2, double s3) { return s1 * s1 + d12 * s2 * s2 + d13 * s3 * s3 + d14 * s1 * s3; };
  const double b0 = beta(one6 * (-2 * v[0] + 9 * v[1] - 18 * v[2] + 11 * v[3]), -v[0] + 4 * v[1] - 5 * v[2] + 2 * v[3],
                         -v[0] + 3 * v[1] - 3 * v[2] + v[3]);
  const double s2m = v[2] - 2 * v[3] + v[4];
  const double b1 = beta(one6 * (v[1] - 6 * v[2] + 3 * v[3] + 2 * v[4]), s2m, -v[1] + 3 * v[2] - 3 * v[3] + v[4]);
  const double b2 = beta(one6 * (-2 * v[2] - 3 * v[3] + 6 * v[4] - v[5]), s2m, -v[2] + 3 * v[3] - 3 * v[4] + v[5]);
  const double b3 = beta(one6 * (-11 * v[3] + 18 * v[4] - 9 * v[5] + 2 * v[6]), 2 * v[3] - 5 * v[4] + 4 * v[5] - v[6],
                         -v[3] + 3 * v[4] - 3 * v[5] + v[6]);
  double tau = b0 + 3 * b1 - 3 * b2 - b3;
  tau *= tau;
  const double a0 = c0 + c0 * tau / sqr(eps + b0);
  const double a1 = c1 + c1 * tau / sqr(eps + b1);
  const double a2 = c2 + c2 * tau / sqr(eps + b2);
  const double a3 = c3 + c3 * tau / sqr(eps + b3);
  return one12 * (a0 * q0 + a1 * q1 + a2 * q2 + a3 * q3) / (a0 + a1 + a2 + a3);
}

double WENO7(const double *vp, const double *vm, double eps, bool if_shock) {
  const double rm[7] = {vm[6], vm[5], vm[4], vm[3], vm[2], vm[1], vm[0]};
  return weno7_one(vp, eps, if_shock) + weno7_one(rm, eps, if_shock);
}

// ---------------------------------------------------------------------------------------
// Characteristic WENO flux at one interface (src/WENO.cu:1090-1457; air: :10-244)
// Q[v][m], F[f][m] hold the stencil nodes m = 0..2r-1 (interface between r-1 and r).
// ---------------------------------------------------------------------------------------
void weno_char_interface(const Param &p, int order, double Q[][8], double F[][8], double kx, double ky, double kz,
                         double eps_ref, bool if_shock, double *fc) {
  const int n_var = p.n_var, ns = p.n_spec;
  const int r = order == 5 ? 3 : 4;
  const int ic = r - 1;
  const double rho_l = Q[0][ic], rho_r = Q[0][ic + 1];
  double temp1 = std::sqrt(rho_l * rho_r);
  const double rlc = 1 / (rho_l + temp1), rrc = 1 / (temp1 + rho_r);
  const double um = rlc * Q[1][ic] + rrc * Q[1][ic + 1];
  const double vm = rlc * Q[2][ic] + rrc * Q[2][ic + 1];
  const double wm = rlc * Q[3][ic] + rrc * Q[3][ic + 1];
  double svm[16] = {}, alpha[16] = {}, ecoef[16] = {};
  double cm, gm1;
  if (ns == 0) {
    const double temp3 = (rlc * F[4][ic] + rrc * F[4][ic + 1]) / R_air;
    cm = std::sqrt(gamma_air * R_air * temp3);
    gm1 = gamma_air - 1;
  } else {
    for (int l = 0; l < n_var - 5; ++l) svm[l] = rlc * Q[l + 5][ic] + rrc * Q[l + 5][ic + 1];
    double rg = 0;
    for (int l = 0; l < ns; ++l) rg += svm[l] * p.mech.gas_const[l];
    const double temp3 = (rlc * F[4][ic] + rrc * F[4][ic + 1]) / std::max(rg, 1e-12);
    double gamma;
    if (p.i_eve >= 0) characteristic_thermo_2t(p, temp3, svm, &gamma, &cm, alpha, ecoef);
    else characteristic_thermo(temp3, svm, p.mech, &gamma, &cm, alpha, ecoef, nullptr);
    gm1 = gamma - 1;
  }
  temp1 = 1.0 / std::sqrt(kx * kx + ky * ky + kz * kz);
  kx *= temp1; ky *= temp1; kz *= temp1;
  const double Uk_bar = kx * um + ky * vm + kz * wm;
  double nx = 0, ny = 0, nz = 0;
  if (std::fabs(kx) > 0.8) { nx = -kz; nz = kx; }
  else { ny = kz; nz = -ky; }
  temp1 = 1.0 / std::sqrt(nx * nx + ny * ny + nz * nz);
  nx *= temp1; ny *= temp1; nz *= temp1;
  double qx = ky * nz - kz * ny, qy = kz * nx - kx * nz, qz = kx * ny - ky * nx;
  temp1 = 1.0 / std::sqrt(qx * qx + qy * qy + qz * qz);
  qx *= temp1; qy *= temp1; qz *= temp1;
  const double Un = nx * um + ny * vm + nz * wm;
  const double Uq = qx * um + qy * vm + qz * wm;
  const double temp2 = 1.0 / (cm * cm);
  const double temp3 = 0.5 * gm1 * (um * um + vm * vm + wm * wm);
  const int nst = 2 * r;  // stencil nodes
  double max_lambda = 0;
  for (int m = 0; m < nst; ++m) {
    const double lam = std::fabs(F[0][m]) + F[5][m];
    if (lam > max_lambda) max_lambda = lam;
  }
  double sumBetaQ[8] = {}, sumBetaF[8] = {};
  if (ns > 0) {
    for (int m = 0; m < nst; ++m) {
      double sp = 0, sm = 0;
      for (int n = 0; n < p.n_scalar_transported; ++n) {
        sp += alpha[n] * Q[5 + n][m];
        sm += alpha[n] * (Q[5 + n][m] * F[0][m]);
      }
      sumBetaQ[m] = sp;
      sumBetaF[m] = sm;
    }
  }
  double fChar[16] = {};
  for (int l = 0; l < 5; ++l) {
    double L[5], tc = 0.5;
    switch (l) {
      case 0:
        L[0] = (temp3 + Uk_bar * cm) * temp2 * 0.5;
        L[1] = -(gm1 * um + kx * cm) * temp2 * 0.5;
        L[2] = -(gm1 * vm + ky * cm) * temp2 * 0.5;
        L[3] = -(gm1 * wm + kz * cm) * temp2 * 0.5;
        L[4] = gm1 * temp2 * 0.5;
        break;
      case 1: tc = 0; L[0] = -Un; L[1] = nx; L[2] = ny; L[3] = nz; L[4] = 0; break;
      case 2: tc = 0; L[0] = -Uq; L[1] = qx; L[2] = qy; L[3] = qz; L[4] = 0; break;
      case 3:
        tc = -1;
        L[0] = 1 - temp3 * temp2;
        L[1] = gm1 * um * temp2;
        L[2] = gm1 * vm * temp2;
        L[3] = gm1 * wm * temp2;
        L[4] = -gm1 * temp2;
        break;
      default:
        L[0] = (temp3 - Uk_bar * cm) * temp2 * 0.5;
        L[1] = -(gm1 * um - kx * cm) * temp2 * 0.5;
        L[2] = -(gm1 * vm - ky * cm) * temp2 * 0.5;
        L[3] = -(gm1 * wm - kz * cm) * temp2 * 0.5;
        L[4] = gm1 * temp2 * 0.5;
    }
    double vP[8] = {}, vM[8] = {};
    for (int m = 0; m < nst; ++m) {
      double LF = L[0] * (Q[0][m] * F[0][m]) + L[1] * F[1][m] + L[2] * F[2][m] + L[3] * F[3][m] +
                  L[4] * ((Q[4][m] + F[4][m]) * F[0][m]);
      double LQ = L[0] * Q[0][m] + L[1] * Q[1][m] + L[2] * Q[2][m] + L[3] * Q[3][m] + L[4] * Q[4][m];
      if (ns > 0) {
        LF += tc * sumBetaF[m];
        LQ += tc * sumBetaQ[m];
      }
      if (m < nst - 1) vP[m] = 0.5 * F[6][m] * (LF + max_lambda * LQ);
      if (m > 0) vM[m - 1] = 0.5 * F[6][m] * (LF - max_lambda * LQ);
    }
    fChar[l] = order == 5 ? WENO5(vP, vM, eps_ref, if_shock) : WENO7(vP, vM, eps_ref, if_shock);
  }
  for (int l = 0; l < n_var - 5; ++l) {
    double vP[8] = {}, vM[8] = {};
    for (int m = 0; m < nst; ++m) {
      const double LQ = Q[5 + l][m] - svm[l] * Q[0][m];
      const double LF = F[0][m] * LQ;
      if (m < nst - 1) vP[m] = 0.5 * F[6][m] * (LF + max_lambda * LQ);
      if (m > 0) vM[m - 1] = 0.5 * F[6][m] * (LF - max_lambda * LQ);
    }
    fChar[5 + l] = order == 5 ? WENO5(vP, vM, eps_ref, if_shock) : WENO7(vP, vM, eps_ref, if_shock);
  }
  const double t1 = fChar[0] + fChar[3] + fChar[4];
  const double t3 = fChar[0] - fChar[4];
  fc[0] = t1;
  fc[1] = um * t1 - kx * cm * t3 + nx * fChar[1] + qx * fChar[2];
  fc[2] = vm * t1 - ky * cm * t3 + ny * fChar[1] + qy * fChar[2];
  fc[3] = wm * t1 - kz * cm * t3 + nz * fChar[1] + qz * fChar[2];
  const double hr = rlc * (Q[4][ic] + F[4][ic]) + rrc * (Q[4][ic + 1] + F[4][ic + 1]);
  fc[4] = hr * t1 - Uk_bar * cm * t3 + Un * fChar[1] + Uq * fChar[2] - cm * cm / gm1 * fChar[3];
  double e = 0;
  for (int l = 0; l < n_var - 5; ++l) {
    fc[5 + l] = svm[l] * t1 + fChar[l + 5];
    e += ecoef[l] * fChar[l + 5];
  }
  fc[4] += e;
}

// Index helper: node at offset m along direction dir from (i,j,k).
inline void shift(int dir, int m, int &i, int &j, int &k) {
  if (dir == 0) i += m;
  else if (dir == 1) j += m;
  else k += m;
}

// Positivity limiter of the species rows of a characteristic-WENO interface flux
// (src/WENO.cu:1459-1528): with alpha = 1/3 (3-D) or 1/2, each species flux is blended with a
// first-order flux f1 by theta = min(theta_p, theta_m) so that the two one-sided updates
// alpha J rho_Y -+ dt f stay non-negative.  Q/F are the node slots of the interface's stencil,
// l = left node, l + 1 = right node.
void positive_limit(const Param &p, const double Q[][8], const double F[][8], int l, double *fc) {
  const double dt = p.dt;
  const double alpha = p.dim == 3 ? 1.0 / 3.0 : 0.5;
  const double jl = F[6][l], jr = F[6][l + 1];
  const double alphaL = 0.5 * alpha * jl, alphaR = 0.5 * alpha * jr;
  // every transported scalar: the species and, in two temperatures, e_ve (src/WENO.cu:1471)
  const int nsc = p.n_var - 5;
  int start = -1;
  for (int s = 0; s < nsc; ++s) {
    const double up = alphaL * Q[s + 5][l] - dt * fc[s + 5];
    const double um = alphaR * Q[s + 5][l + 1] + dt * fc[s + 5];
    if (up < 0 || um < 0) {
      start = s;
      break;
    }
  }
  if (start < 0) return;
  const double U1 = F[0][l] * jl, U2 = F[0][l + 1] * jr;
  for (int s = start; s < nsc; ++s) {
    double f1 = 0, theta_p = 1, theta_m = 1;
    bool have_f1 = false;
    const double yl = Q[s + 5][l], yr = Q[s + 5][l + 1];
    const double fp = 0.5 * F[6][l] * (F[0][l] + F[5][l]) * yl;
    const double fm = 0.5 * F[6][l + 1] * (F[0][l + 1] - F[5][l + 1]) * yr;
    const double up = alphaL * yl - dt * fc[s + 5];
    if (up < 0) {
      f1 = 0.5 * (fp + U1 * yl) + 0.5 * (fm - U2 * yr);
      have_f1 = true;
      const double up_lf = alphaL * yl - dt * f1;
      if (std::abs(up - up_lf) > 1e-20 * p.rho_ref) {
        theta_p = (0 - up_lf) / (up - up_lf);
        if (theta_p > 1) theta_p = 1.0;
        else if (theta_p < 0) theta_p = 0;
      }
    }
    const double um = alphaR * yr + dt * fc[s + 5];
    if (um < 0) {
      if (!have_f1) f1 = 0.5 * (fp + U1 * yl) + 0.5 * (fm - U2 * yr);
      const double um_lf = alphaR * yr + dt * f1;
      if (std::abs(um - um_lf) > 1e-20 * p.rho_ref) {
        theta_m = (0 - um_lf) / (um - um_lf);
        if (theta_m > 1) theta_m = 1.0;
        else if (theta_m < 0) theta_m = 0;
      }
    }
    fc[s + 5] = std::min(theta_p, theta_m) * (fc[s + 5] - f1) + f1;
  }
}

void convective_term_weno_char(Zone &z, const Param &p, int dir) {
  const int order = (p.inviscid_scheme == 52) ? 5 : 7;
  const int r = order == 5 ? 3 : 4;
  const int ext[3] = {z.mx, z.my, z.mz};
  const double eps_ref = eps_weno * p.weno_eps_scale;
  const Arr &fc = dir == 0 ? z.fF : (dir == 1 ? z.gF : z.hF);
  std::vector<double> own;
  Arr F_out = fc;
  if (!fc) {  // flux scratch when the caller has no fFlux arrays
    own.assign(z.cv.sz * p.n_var, 0.0);
    F_out = Arr(own.data(), z.mx, z.my, z.mz, z.ngg);
  }
  int lo[3] = {0, 0, 0}, hi[3] = {z.mx, z.my, z.mz};
  lo[dir] = -1;
  hi[dir] = ext[dir];
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = lo[2]; k < hi[2]; ++k)
    for (int j = lo[1]; j < hi[1]; ++j)
      for (int i = lo[0]; i < hi[0]; ++i) {
        double Q[16][8], F[7][8];
        for (int m = 0; m < 2 * r; ++m) {
          int a = i, b = j, c = k;
          shift(dir, m - r + 1, a, b, c);
          const double q0 = z.cv(a, b, c, 0), q1 = z.cv(a, b, c, 1), q2 = z.cv(a, b, c, 2), q3 = z.cv(a, b, c, 3);
          const double m0 = z.metric(a, b, c, 3 * dir), m1 = z.metric(a, b, c, 3 * dir + 1),
                       m2 = z.metric(a, b, c, 3 * dir + 2);
          const double Uk = (q1 * m0 + q2 * m1 + q3 * m2) / q0;
          const double pk = z.bv(a, b, c, 4);
          for (int l = 0; l < p.n_var; ++l) Q[l][m] = z.cv(a, b, c, l);
          F[0][m] = Uk;
          F[1][m] = q1 * Uk + pk * m0;
          F[2][m] = q2 * Uk + pk * m1;
          F[3][m] = q3 * Uk + pk * m2;
          F[4][m] = pk;
          double cg = std::sqrt(m0 * m0 + m1 * m1 + m2 * m2);
          if (p.n_spec == 0) cg *= std::sqrt(gamma_air * R_air * z.bv(a, b, c, 5));
          else cg *= z.acoustic(a, b, c);
          F[5][m] = cg;
          F[6][m] = z.jac(a, b, c);
        }
        // face metric: x averages with i+1; y and z also average with i+1 (src/WENO.cu:1615, 2280)
        const double kx = 0.5 * (z.metric(i, j, k, 3 * dir) + z.metric(i + 1, j, k, 3 * dir));
        const double ky = 0.5 * (z.metric(i, j, k, 3 * dir + 1) + z.metric(i + 1, j, k, 3 * dir + 1));
        const double kz = 0.5 * (z.metric(i, j, k, 3 * dir + 2) + z.metric(i + 1, j, k, 3 * dir + 2));
        bool shock = true;
        if (p.sensor_threshold > 1e-10) {
          shock = false;
          for (int d = -z.ngg + 1; d <= z.ngg; ++d) {
            int a = i, b = j, c = k;
            shift(dir, d, a, b, c);
            if (z.shock(a, b, c) > p.sensor_threshold) { shock = true; break; }
          }
        }
        double f[16];
        weno_char_interface(p, order, Q, F, kx, ky, kz, eps_ref, shock, f);
        if (p.positive_preserving && p.n_spec > 0) positive_limit(p, Q, F, r - 1, f);
        for (int l = 0; l < p.n_var; ++l) F_out(i, j, k, l) = f[l];
      }
  // compute_derivative_{x,y,z} (src/WENO.cu:1532-1559)
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < z.mz; ++k)
    for (int j = 0; j < z.my; ++j)
      for (int i = 0; i < z.mx; ++i) {
        int a = i, b = j, c = k;
        shift(dir, -1, a, b, c);
        for (int l = 0; l < p.n_var; ++l) z.dq(i, j, k, l) -= F_out(i, j, k, l) - F_out(a, b, c, l);
      }
}

// Component-wise WENO with node-wise LLF splitting (inviscid_scheme 51/71,
// src/WENO.cu:890-1089 and the y/z twins)
void convective_term_weno_comp(Zone &z, const Param &p, int dir) {
  const int order = (p.inviscid_scheme == 51) ? 5 : 7;
  const int r = order == 5 ? 3 : 4;
  const int ext[3] = {z.mx, z.my, z.mz};
  const double eps_ref = eps_weno * p.weno_eps_scale;
  const double eps_scaled[3] = {eps_ref, eps_ref * p.v_ref * p.v_ref, eps_ref * p.v_ref * p.v_ref * p.v_ref * p.v_ref};
  std::vector<double> own((size_t)z.cv.sz * p.n_var, 0.0);
  Arr F_out(own.data(), z.mx, z.my, z.mz, z.ngg);
  int lo[3] = {0, 0, 0}, hi[3] = {z.mx, z.my, z.mz};
  lo[dir] = -1;
  hi[dir] = ext[dir];
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = lo[2]; k < hi[2]; ++k)
    for (int j = lo[1]; j < hi[1]; ++j)
      for (int i = lo[0]; i < hi[0]; ++i) {
        double fp[16][8], fm[16][8];
        for (int m = 0; m < 2 * r; ++m) {
          int a = i, b = j, c = k;
          shift(dir, m - r + 1, a, b, c);
          const double q0 = z.cv(a, b, c, 0), q1 = z.cv(a, b, c, 1), q2 = z.cv(a, b, c, 2), q3 = z.cv(a, b, c, 3),
                       q4 = z.cv(a, b, c, 4);
          double pk = z.bv(a, b, c, 4);
          const double m0 = z.metric(a, b, c, 3 * dir), m1 = z.metric(a, b, c, 3 * dir + 1),
                       m2 = z.metric(a, b, c, 3 * dir + 2);
          const double Uk = (q1 * m0 + q2 * m1 + q3 * m2) / q0;
          double cg = std::sqrt(m0 * m0 + m1 * m1 + m2 * m2);
          if (p.n_spec == 0) cg *= std::sqrt(gamma_air * R_air * z.bv(a, b, c, 5));
          else cg *= z.acoustic(a, b, c);
          const double lambda0 = std::fabs(Uk) + cg;
          const double jac = z.jac(a, b, c);
          const double sPlus = 0.5 * jac * (Uk + lambda0), sMinus = 0.5 * jac * (Uk - lambda0);
          pk *= 0.5 * jac;
          fp[0][m] = sPlus * q0;
          fp[1][m] = sPlus * q1 + pk * m0;
          fp[2][m] = sPlus * q2 + pk * m1;
          fp[3][m] = sPlus * q3 + pk * m2;
          fp[4][m] = sPlus * q4 + pk * Uk;
          fm[0][m] = sMinus * q0;
          fm[1][m] = sMinus * q1 + pk * m0;
          fm[2][m] = sMinus * q2 + pk * m1;
          fm[3][m] = sMinus * q3 + pk * m2;
          fm[4][m] = sMinus * q4 + pk * Uk;
          for (int l = 5; l < p.n_var; ++l) {
            const double ql = z.cv(a, b, c, l);
            fp[l][m] = sPlus * ql;
            fm[l][m] = sMinus * ql;
          }
        }
        bool shock = true;
        if (p.sensor_threshold > 1e-10) {
          shock = false;
          for (int d = -z.ngg + 1; d <= z.ngg; ++d) {
            int a = i, b = j, c = k;
            shift(dir, d, a, b, c);
            if (z.shock(a, b, c) > p.sensor_threshold) { shock = true; break; }
          }
        }
        for (int l = 0; l < p.n_var; ++l) {
          const double eps = (l >= 1 && l <= 3) ? eps_scaled[1] : (l == 4 ? eps_scaled[2] : eps_scaled[0]);
          F_out(i, j, k, l) =
              order == 5 ? WENO5(&fp[l][0], &fm[l][1], eps, shock) : WENO7(&fp[l][0], &fm[l][1], eps, shock);
        }
      }
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < z.mz; ++k)
    for (int j = 0; j < z.my; ++j)
      for (int i = 0; i < z.mx; ++i) {
        int a = i, b = j, c = k;
        shift(dir, -1, a, b, c);
        for (int l = 0; l < p.n_var; ++l) z.dq(i, j, k, l) -= F_out(i, j, k, l) - F_out(a, b, c, l);
      }
}

// ---------------------------------------------------------------------------------------
// Primitive reconstruction + Riemann solvers (src/InviscidScheme.cu:28-786,
// src/Reconstruction.cu, src/Limiter.cuh)
// ---------------------------------------------------------------------------------------
double minmod(double a, double b) {
  const double sa = a < 0 ? -1 : 1, sb = b < 0 ? -1 : 1;
  return 0.5 * (sa + sb) * std::min(std::fabs(a), std::fabs(b));
}

double pv_eps(const Param &p, int l) {
  double s = 1.0;
  if (l == 0) s = p.rho_ref;
  else if (l <= 3) s = p.v_ref;
  else if (l == 4) s = p.rho_ref * p.v_ref * p.v_ref;
  return eps_weno * s * s;
}

// pv[l][m] for stencil nodes m = 0..2r-1, interface between r-1 and r.
void reconstruct(const Param &p, double pv[][8], int r, double *pl, double *pr) {
  const int ic = r - 1;
  for (int l = 0; l < p.n_var; ++l) {
    switch (p.reconstruction) {
      case 2: {
        const double kappa = 1.0 / 3.0;
        const double di = pv[l][ic] - pv[l][ic - 1], di1 = pv[l][ic + 1] - pv[l][ic],
                     di2 = pv[l][ic + 2] - pv[l][ic + 1];
        const double dnl = minmod(di, di1), dpl = minmod(di1, di), dnr = minmod(di1, di2), dpr = minmod(di2, di1);
        pl[l] = pv[l][ic] + 0.25 * ((1 - kappa) * dnl + (1 + kappa) * dpl);
        pr[l] = pv[l][ic + 1] - 0.25 * ((1 - kappa) * dpr + (1 + kappa) * dnr);
        break;
      }
      case 3: {
        const double di = pv[l][ic] - pv[l][ic - 1], di1 = pv[l][ic + 1] - pv[l][ic],
                     di2 = pv[l][ic + 2] - pv[l][ic + 1];
        pl[l] = pv[l][ic] + 0.5 * minmod(di, di1);
        pr[l] = pv[l][ic + 1] - 0.5 * minmod(di1, di2);
        break;
      }
      case 5: case 7: {
        const double eps = pv_eps(p, l);
        const double *v = &pv[l][0];
        if (p.reconstruction == 5) {
          // left from nodes ic-2..ic+2, right from ic-1..ic+3 (WENO5 of src/WENO.cu:3033)
          double vp[5], wm[5];
          for (int m = 0; m < 5; ++m) { vp[m] = v[ic - 2 + m]; wm[m] = v[ic - 1 + m]; }
          pl[l] = weno5_plus(vp, eps, true);
          pr[l] = weno5_minus(wm, eps, true);
        } else {
          double vp[7], wm[7];
          for (int m = 0; m < 7; ++m) { vp[m] = v[ic - 3 + m]; wm[m] = v[ic - 2 + m]; }
          const double rm[7] = {wm[6], wm[5], wm[4], wm[3], wm[2], wm[1], wm[0]};
          pl[l] = weno7_one(vp, eps, true);
          pr[l] = weno7_one(rm, eps, true);
        }
        break;
      }
      default:
        pl[l] = pv[l][ic];
        pr[l] = pv[l][ic + 1];
    }
  }
  // energy and gamma of the reconstructed states (src/InviscidScheme.cu:184-218)
  const int nv = p.n_var;
  for (double *s : {pl, pr}) {
    const double ek = 0.5 * (s[1] * s[1] + s[2] * s[2] + s[3] * s[3]);
    if (p.n_spec == 0) {
      s[nv] = ek * s[0] + s[4] / (gamma_air - 1);
      s[nv + 1] = gamma_air;
    } else {
      double rg = 0;
      for (int l = 0; l < p.n_spec; ++l) rg += s[5 + l] * p.mech.gas_const[l];
      const double t = s[4] / std::max(s[0] * rg, 1e-12);
      double g, c, etr;
      if (p.i_eve >= 0) {
        // two temperatures: translational-rotational energy and gamma, plus e_ve (:197-211)
        characteristic_thermo_2t(p, t, s + 5, &g, &c, nullptr, nullptr, &etr);
        s[nv] = s[0] * (ek + etr + std::max(s[5 + p.i_eve], 0.0));
      } else {
        characteristic_thermo(t, s + 5, p.mech, &g, &c, nullptr, nullptr, &etr);
        s[nv] = s[0] * (ek + etr);
      }
      s[nv + 1] = g;
    }
  }
}

void ausm_plus(const Param &p, const double *pl, const double *pr, const double *ml, const double *mr, double jl,
               double jr, double *fc) {
  const int nv = p.n_var;
  const double k1 = 0.5 * (jl * ml[0] + jr * mr[0]);
  const double k2 = 0.5 * (jl * ml[1] + jr * mr[1]);
  const double k3 = 0.5 * (jl * ml[2] + jr * mr[2]);
  const double gk = std::sqrt(k1 * k1 + k2 * k2 + k3 * k3);
  const double ul = (k1 * pl[1] + k2 * pl[2] + k3 * pl[3]) / gk;
  const double ur = (k1 * pr[1] + k2 * pr[2] + k3 * pr[3]) / gk;
  const double c = 0.5 * (std::sqrt(pl[nv + 1] * pl[4] / pl[0]) + std::sqrt(pr[nv + 1] * pr[4] / pr[0]));
  const double mach_l = ul / c, mach_r = ur / c;
  double mlp, mrn, plp, prn;
  const double alpha = 3 / 16.0;
  if (std::fabs(mach_l) > 1) {
    mlp = 0.5 * (mach_l + std::fabs(mach_l));
    plp = mlp / mach_l;
  } else {
    const double a = (mach_l + 1) * (mach_l + 1) * 0.25, b = (mach_l * mach_l - 1) * (mach_l * mach_l - 1);
    mlp = a + 0.125 * b;
    plp = a * (2 - mach_l) + alpha * mach_l * b;
  }
  if (std::fabs(mach_r) > 1) {
    mrn = 0.5 * (mach_r - std::fabs(mach_r));
    prn = mrn / mach_r;
  } else {
    const double a = (mach_r - 1) * (mach_r - 1) * 0.25, b = (mach_r * mach_r - 1) * (mach_r * mach_r - 1);
    mrn = -a - 0.125 * b;
    prn = a * (2 + mach_r) - alpha * mach_r * b;
  }
  const double p_coeff = plp * pl[4] + prn * pr[4];
  const double m_half = mlp + mrn;
  const double mass = c * (pl[0] * (0.5 * (m_half + std::fabs(m_half))) + pr[0] * (0.5 * (m_half - std::fabs(m_half))));
  const double coeff = mass * gk;
  const double *s = mass >= 0 ? pl : pr;
  fc[0] = coeff;
  fc[1] = coeff * s[1] + p_coeff * k1;
  fc[2] = coeff * s[2] + p_coeff * k2;
  fc[3] = coeff * s[3] + p_coeff * k3;
  fc[4] = coeff * (s[nv] + s[4]) / s[0];
  for (int l = 5; l < nv; ++l) fc[l] = coeff * s[l];
}

void hllc(const Param &p, const double *pl, const double *pr, const double *ml, const double *mr, double jl,
          double jr, double *fc) {
  const int nv = p.n_var;
  const double rl_c = std::sqrt(pl[0]) / (std::sqrt(pl[0]) + std::sqrt(pr[0]));
  const double rr_c = std::sqrt(pr[0]) / (std::sqrt(pl[0]) + std::sqrt(pr[0]));
  const double ut = pl[1] * rl_c + pr[1] * rr_c, vt = pl[2] * rl_c + pr[2] * rr_c, wt = pl[3] * rl_c + pr[3] * rr_c;
  double c_tilde;
  if (p.n_spec == 0) {
    const double hl = (pl[nv] + pl[4]) / pl[0], hr = (pr[nv] + pr[4]) / pr[0];
    const double ht = hl * rl_c + hr * rr_c;
    const double ekt = 0.5 * (ut * ut + vt * vt + wt * wt);
    c_tilde = std::sqrt((gamma_air - 1) * (ht - ekt));
  } else {
    double svm[16] = {}, rg = 0;
    for (int l = 0; l < nv - 5; ++l) svm[l] = rl_c * pl[l + 5] + rr_c * pr[l + 5];
    for (int l = 0; l < p.n_spec; ++l) rg += svm[l] * p.mech.gas_const[l];
    const double t = (rl_c * (pl[4] / pl[0]) + rr_c * (pr[4] / pr[0])) / std::max(rg, 1e-12);
    double g;
    if (p.i_eve >= 0) characteristic_thermo_2t(p, t, svm, &g, &c_tilde, nullptr, nullptr);
    else characteristic_thermo(t, svm, p.mech, &g, &c_tilde, nullptr, nullptr, nullptr);
  }
  const double kx = 0.5 * (ml[0] + mr[0]), ky = 0.5 * (ml[1] + mr[1]), kz = 0.5 * (ml[2] + mr[2]);
  const double gK = std::sqrt(kx * kx + ky * ky + kz * kz);
  const double Utb = (kx * ut + ky * vt + kz * wt) / gK;
  const double ja = 0.5 * (jl + jr);
  const double Ul = kx * pl[1] + ky * pl[2] + kz * pl[3];
  const double cl = std::sqrt(pl[nv + 1] * pl[4] / pl[0]);
  const double sl = std::min(Ul / gK - cl, Utb - c_tilde);
  if (sl >= 0) {
    const double rU = pl[0] * Ul;
    fc[0] = ja * rU;
    fc[1] = ja * (rU * pl[1] + pl[4] * kx);
    fc[2] = ja * (rU * pl[2] + pl[4] * ky);
    fc[3] = ja * (rU * pl[3] + pl[4] * kz);
    fc[4] = ja * ((pl[nv] + pl[4]) * Ul);
    for (int l = 5; l < nv; ++l) fc[l] = ja * rU * pl[l];
    return;
  }
  const double Ur = kx * pr[1] + ky * pr[2] + kz * pr[3];
  const double cr = std::sqrt(pr[nv + 1] * pr[4] / pr[0]);
  const double sr = std::max(Ur / gK + cr, Utb + c_tilde);
  if (sr < 0) {
    const double rU = pr[0] * Ur;
    fc[0] = ja * rU;
    fc[1] = ja * (rU * pr[1] + pr[4] * kx);
    fc[2] = ja * (rU * pr[2] + pr[4] * ky);
    fc[3] = ja * (rU * pr[3] + pr[4] * kz);
    fc[4] = ja * ((pr[nv] + pr[4]) * Ur);
    for (int l = 5; l < nv; ++l) fc[l] = ja * rU * pr[l];
    return;
  }
  const double sm = ((pr[0] * Ur * (sr - Ur / gK) - pl[0] * Ul * (sl - Ul / gK)) / gK + pl[4] - pr[4]) /
                    (pr[0] * (sr - Ur / gK) - pl[0] * (sl - Ul / gK));
  const double pm = pl[0] * (sl - Ul / gK) * (sm - Ul / gK) + pl[4];
  if (sm >= 0) {
    const double pc = 1.0 / (sl - sm);
    const double Qc = ja * pc * sm * (sl * gK - Ul) * pl[0];
    fc[0] = Qc;
    const double dP = (sl * pm - sm * pl[4]) * pc * ja;
    fc[1] = Qc * pl[1] + dP * kx;
    fc[2] = Qc * pl[2] + dP * ky;
    fc[3] = Qc * pl[3] + dP * kz;
    fc[4] = Qc * pl[nv] / pl[0] + pc * ja * (sl * pm * sm * gK - sm * pl[4] * Ul);
    for (int l = 5; l < nv; ++l) fc[l] = Qc * pl[l];
  } else {
    const double pc = 1.0 / (sr - sm);
    const double Qc = ja * pc * sm * (sr * gK - Ur) * pr[0];
    fc[0] = Qc;
    const double dP = (sr * pm - sm * pr[4]) * pc * ja;
    fc[1] = Qc * pr[1] + dP * kx;
    fc[2] = Qc * pr[2] + dP * ky;
    fc[3] = Qc * pr[3] + dP * kz;
    fc[4] = Qc * pr[nv] / pr[0] + pc * ja * (sr * pm * sm * gK - sm * pr[4] * Ur);
    for (int l = 5; l < nv; ++l) fc[l] = Qc * pr[l];
  }
}

void roe_interface(const Param &p, const double *pl, const double *pr, const double *ml, const double *mr, double jl,
                   double jr, double efl, double efr, double *fc) {
  const int nv = p.n_var;
  // compute_half_sum_left_right_flux (src/InviscidScheme.cu:592-624)
  double JKx = jl * ml[0], JKy = jl * ml[1], JKz = jl * ml[2];
  double Uk = pl[1] * JKx + pl[2] * JKy + pl[3] * JKz;
  double co = Uk * pl[0];
  fc[0] = 0.5 * co;
  fc[1] = 0.5 * (co * pl[1] + pl[4] * JKx);
  fc[2] = 0.5 * (co * pl[2] + pl[4] * JKy);
  fc[3] = 0.5 * (co * pl[3] + pl[4] * JKz);
  fc[4] = 0.5 * Uk * (pl[4] + pl[nv]);
  for (int l = 5; l < nv; ++l) fc[l] = 0.5 * co * pl[l];
  JKx = jr * mr[0]; JKy = jr * mr[1]; JKz = jr * mr[2];
  Uk = pr[1] * JKx + pr[2] * JKy + pr[3] * JKz;
  co = Uk * pr[0];
  fc[0] += 0.5 * co;
  fc[1] += 0.5 * (co * pr[1] + pr[4] * JKx);
  fc[2] += 0.5 * (co * pr[2] + pr[4] * JKy);
  fc[3] += 0.5 * (co * pr[3] + pr[4] * JKz);
  fc[4] += 0.5 * Uk * (pr[4] + pr[nv]);
  for (int l = 5; l < nv; ++l) fc[l] += 0.5 * co * pr[l];
  // Roe dissipation (src/InviscidScheme.cu:626-746)
  const double dl = std::sqrt(pl[0]), dr = std::sqrt(pr[0]);
  const double idn = 1.0 / (dl + dr);
  const double u = (dl * pl[1] + dr * pr[1]) * idn, v = (dl * pl[2] + dr * pr[2]) * idn,
               w = (dl * pl[3] + dr * pr[3]) * idn;
  const double ek = 0.5 * (u * u + v * v + w * w);
  const double hl = (pl[nv] + pl[4]) / pl[0], hr = (pr[nv] + pr[4]) / pr[0];
  const double h = (dl * hl + dr * hr) * idn;
  double gamma = gamma_air;
  double c = std::sqrt((gamma - 1) * (h - ek));
  double svm[16] = {}, alpha[16] = {}, ecoef[16] = {};
  for (int l = 0; l < nv - 5; ++l) svm[l] = (dl * pl[l + 5] + dr * pr[l + 5]) * idn;
  if (p.n_spec > 0) {
    double rg = 0;
    for (int l = 0; l < p.n_spec; ++l) rg += svm[l] * p.mech.gas_const[l];
    const double t = (dl * (pl[4] / pl[0]) + dr * (pr[4] / pr[0])) * idn / std::max(rg, 1e-12);
    characteristic_thermo(t, svm, p.mech, &gamma, &c, alpha, ecoef, nullptr);
  }
  double kx = 0.5 * (ml[0] + mr[0]), ky = 0.5 * (ml[1] + mr[1]), kz = 0.5 * (ml[2] + mr[2]);
  const double gK = std::sqrt(kx * kx + ky * ky + kz * kz);
  Uk = kx * u + ky * v + kz * w;
  double ch[3] = {Uk - gK * c, Uk, Uk + gK * c};
  const double efd = 0.5 * (efl + efr);
  for (double &x : ch) {
    x = std::fabs(x);
    if (x < efd) x = 0.5 * (x * x / efd + efd);
  }
  kx /= gK; ky /= gK; kz /= gK; Uk /= gK;
  const double ja = 0.5 * (jl + jr);
  double dq[16] = {};
  dq[0] = ja * (pr[0] - pl[0]);
  for (int l = 1; l < nv; ++l) dq[l] = ja * (pr[0] * pr[l] - pl[0] * pl[l]);
  dq[4] = ja * (pr[nv] - pl[nv]);
  double c1 = (gamma - 1) * (ek * dq[0] - u * dq[1] - v * dq[2] - w * dq[3] + dq[4]) / (c * c);
  double c2 = (kx * dq[1] + ky * dq[2] + kz * dq[3] - Uk * dq[0]) / c;
  for (int l = 0; l < p.n_scalar_transported; ++l) c1 += alpha[l] * dq[l + 5];
  double c3 = dq[0] - c1;
  double LDq[16] = {};
  LDq[0] = 0.5 * (c1 - c2);
  LDq[1] = kx * c3 - ((kz * v - ky * w) * dq[0] - kz * dq[2] + ky * dq[3]) / c;
  LDq[2] = ky * c3 - ((kx * w - kz * u) * dq[0] - kx * dq[3] + kz * dq[1]) / c;
  LDq[3] = kz * c3 - ((ky * u - kx * v) * dq[0] - ky * dq[1] + kx * dq[2]) / c;
  LDq[4] = 0.5 * (c1 + c2);
  for (int l = 0; l < p.n_scalar_transported; ++l) LDq[l + 5] = dq[l + 5] - svm[l] * dq[0];
  double b[16];
  b[0] = -ch[0] * LDq[0];
  for (int l = 1; l < nv; ++l) b[l] = -ch[1] * LDq[l];
  b[4] = -ch[2] * LDq[4];
  const double c0 = kx * b[1] + ky * b[2] + kz * b[3];
  c1 = c0 + b[0] + b[4];
  c2 = c * (b[4] - b[0]);
  c3 = 0;
  for (int l = 0; l < p.n_scalar_transported; ++l) c3 += ecoef[l] * b[l + 5];
  fc[0] += 0.5 * c1;
  fc[1] += 0.5 * (u * c1 + kx * c2 - c * (kz * b[2] - ky * b[3]));
  fc[2] += 0.5 * (v * c1 + ky * c2 - c * (kx * b[3] - kz * b[1]));
  fc[3] += 0.5 * (w * c1 + kz * c2 - c * (ky * b[1] - kx * b[2]));
  fc[4] += 0.5 * (h * c1 + Uk * c2 - c * c * c0 / (gamma - 1) +
                  c * ((kz * v - ky * w) * b[1] + (kx * w - kz * u) * b[2] + (ky * u - kx * v) * b[3]) + c3);
  for (int l = 0; l < nv - 5; ++l) fc[5 + l] += 0.5 * (b[l + 5] + svm[l] * c1);
}

void lax_friedrichs(const Param &p, const double *pl, const double *pr, const double *ml, const double *mr, double jl,
                    double jr, double *fc) {
  const int nv = p.n_var;
  const double kx = 0.5 * (ml[0] + mr[0]), ky = 0.5 * (ml[1] + mr[1]), kz = 0.5 * (ml[2] + mr[2]);
  const double gK = std::sqrt(kx * kx + ky * ky + kz * kz);
  const double Ukl = pl[1] * kx + pl[2] * ky + pl[3] * kz, Ukr = pr[1] * kx + pr[2] * ky + pr[3] * kz;
  const double cl = std::sqrt(gamma_air * pl[4] / pl[0]), cr = std::sqrt(gamma_air * pr[4] / pr[0]);
  const double sr = std::max(std::fabs(Ukl) + cl * gK, std::fabs(Ukr) + cr * gK);
  const double hj = 0.5 * 0.5 * (jl + jr);
  const double rUl = pl[0] * Ukl, rUr = pr[0] * Ukr;
  fc[0] = (rUl + rUr - sr * (pr[0] - pl[0])) * hj;
  fc[1] = (rUl * pl[1] + rUr * pr[1] + kx * (pl[4] + pr[4]) - sr * (pr[1] * pr[0] - pl[1] * pl[0])) * hj;
  fc[2] = (rUl * pl[2] + rUr * pr[2] + ky * (pl[4] + pr[4]) - sr * (pr[2] * pr[0] - pl[2] * pl[0])) * hj;
  fc[3] = (rUl * pl[3] + rUr * pr[3] + kz * (pl[4] + pr[4]) - sr * (pr[3] * pr[0] - pl[3] * pl[0])) * hj;
  fc[4] = ((pl[nv] + pl[4]) * Ukl + (pr[nv] + pr[4]) * Ukr - sr * (pr[nv] - pl[nv])) * hj;
}

void entropy_fix_delta(Zone &z, const Param &p) {
  // src/InviscidScheme.cu:269-304, over [-1, m] in every direction
  for (int k = -1; k <= z.mz; ++k)
    for (int j = -1; j <= z.my; ++j)
      for (int i = -1; i <= z.mx; ++i) {
        const Arr &M = z.metric;
        const double u = z.bv(i, j, k, 1), v = z.bv(i, j, k, 2), w = z.bv(i, j, k, 3);
        const double U = std::fabs(u * M(i, j, k, 0) + v * M(i, j, k, 1) + w * M(i, j, k, 2));
        const double V = std::fabs(u * M(i, j, k, 3) + v * M(i, j, k, 4) + w * M(i, j, k, 5));
        const double W = std::fabs(u * M(i, j, k, 6) + v * M(i, j, k, 7) + w * M(i, j, k, 8));
        const double kx = std::sqrt(sqr(M(i, j, k, 0)) + sqr(M(i, j, k, 1)) + sqr(M(i, j, k, 2)));
        const double ky = std::sqrt(sqr(M(i, j, k, 3)) + sqr(M(i, j, k, 4)) + sqr(M(i, j, k, 5)));
        const double kz = std::sqrt(sqr(M(i, j, k, 6)) + sqr(M(i, j, k, 7)) + sqr(M(i, j, k, 8)));
        const double a =
            p.n_spec == 0 ? std::sqrt(gamma_air * z.bv(i, j, k, 4) / z.bv(i, j, k, 0)) : z.acoustic(i, j, k);
        z.efd(i, j, k) = p.dim == 2 ? p.entropy_fix_factor * (U + V + a * 0.5 * (kx + ky))
                                    : p.entropy_fix_factor * (U + V + W + a * (kx + ky + kz) / 3.0);
      }
}

void convective_term_pv(Zone &z, const Param &p, int dir) {
  const int r = (p.reconstruction == 5) ? 3 : (p.reconstruction == 7 ? 4 : 2);
  const int nv = p.n_var;
  const int ext[3] = {z.mx, z.my, z.mz};
  int lo[3] = {0, 0, 0}, hi[3] = {z.mx, z.my, z.mz};
  lo[dir] = -1;
  hi[dir] = ext[dir];
  std::vector<double> flux((size_t)(z.mx + 1) * (z.my + 1) * (z.mz + 1) * nv, 0.0);
  auto fidx = [&](int i, int j, int k) { return ((size_t)((k + 1) * (z.my + 1) + (j + 1)) * (z.mx + 1) + (i + 1)) * nv; };
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = lo[2]; k < hi[2]; ++k)
    for (int j = lo[1]; j < hi[1]; ++j)
      for (int i = lo[0]; i < hi[0]; ++i) {
        double pv[16][8], mt[3][8], jac[8], ef[8];
        for (int m = 0; m < 2 * r; ++m) {
          int a = i, b = j, c = k;
          shift(dir, m - r + 1, a, b, c);
          for (int l = 0; l < 5; ++l) pv[l][m] = z.bv(a, b, c, l);
          for (int l = 0; l < p.n_scalar; ++l) pv[5 + l][m] = z.sv(a, b, c, l);
          for (int l = 0; l < 3; ++l) mt[l][m] = z.metric(a, b, c, 3 * dir + l);
          jac[m] = z.jac(a, b, c);
          ef[m] = (p.inviscid_scheme == 2 && z.efd && m >= r - 1 && m <= r) ? z.efd(a, b, c) : 0.0;
        }
        double pl[18], pr[18];
        reconstruct(p, pv, r, pl, pr);
        const int ic = r - 1;
        const double ml[3] = {mt[0][ic], mt[1][ic], mt[2][ic]}, mr[3] = {mt[0][ic + 1], mt[1][ic + 1], mt[2][ic + 1]};
        double *fc = &flux[fidx(i, j, k)];
        switch (p.inviscid_scheme) {
          case 3: ausm_plus(p, pl, pr, ml, mr, jac[ic], jac[ic + 1], fc); break;
          case 4: hllc(p, pl, pr, ml, mr, jac[ic], jac[ic + 1], fc); break;
          case 2: roe_interface(p, pl, pr, ml, mr, jac[ic], jac[ic + 1], ef[ic], ef[ic + 1], fc); break;
          default: lax_friedrichs(p, pl, pr, ml, mr, jac[ic], jac[ic + 1], fc);
        }
      }
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < z.mz; ++k)
    for (int j = 0; j < z.my; ++j)
      for (int i = 0; i < z.mx; ++i) {
        int a = i, b = j, c = k;
        shift(dir, -1, a, b, c);
        const double *fr = &flux[fidx(i, j, k)], *fl = &flux[fidx(a, b, c)];
        for (int l = 0; l < nv; ++l) z.dq(i, j, k, l) -= fr[l] - fl[l];
      }
}

// ---------------------------------------------------------------------------------------
// Viscous fluxes (src/ViscousScheme.cu)
// ---------------------------------------------------------------------------------------
// 8th-order derivative with one-sided closures (d_dXi etc., src/ViscousScheme.cu:140-468)
template <typename F>
double d8(F f, int n, int nx, bool bl, bool br) {
  bool done = false;
  double df = 0;
  if (bl) {
    if (n == 0) { df = -25.0 / 12 * f(0) + 4.0 * f(1) - 3 * f(2) + 4.0 / 3 * f(3) - 0.25 * f(4); done = true; }
    else if (n == 1) { df = -0.25 * f(-1) - 5.0 / 6 * f(0) + 1.5 * f(1) - 0.5 * f(2) + 1.0 / 12 * f(3); done = true; }
    else if (n == 2) { df = -1.0 / 12 * (f(2) - f(-2)) + 2.0 / 3 * (f(1) - f(-1)); done = true; }
    else if (n == 3) { df = 0.75 * (f(1) - f(-1)) - 0.15 * (f(2) - f(-2)) + 1.0 / 60 * (f(3) - f(-3)); done = true; }
  }
  if (br) {
    if (n == nx - 1) { df = 25.0 / 12 * f(0) - 4.0 * f(-1) + 3 * f(-2) - 4.0 / 3 * f(-3) + 0.25 * f(-4); done = true; }
    else if (n == nx - 2) { df = 0.25 * f(1) + 5.0 / 6 * f(0) - 1.5 * f(-1) + 0.5 * f(-2) - 1.0 / 12 * f(-3); done = true; }
    else if (n == nx - 3) { df = -1.0 / 12 * (f(2) - f(-2)) + 2.0 / 3 * (f(1) - f(-1)); done = true; }
    else if (n == nx - 4) { df = 0.75 * (f(1) - f(-1)) - 0.15 * (f(2) - f(-2)) + 1.0 / 60 * (f(3) - f(-3)); done = true; }
  }
  if (!done) {
    const double a1 = 0.8, a2 = -0.2, a3 = 4.0 / 105, a4 = -1.0 / 280;
    df = a1 * (f(1) - f(-1)) + a2 * (f(2) - f(-2)) + a3 * (f(3) - f(-3)) + a4 * (f(4) - f(-4));
  }
  return df;
}

// phase 0: the whole term; 1: the node fluxes only; 2: their periodic exchange and the divergence
// (a multi-block grid exchanges the node fluxes across its inner faces in between)
void viscous_8th_nodes(Zone &z, const Param &p);
void viscous_8th_divergence(Zone &z, const Param &p);
void viscous_8th(Zone &z, const Param &p, int phase) {
  if (phase != 2) viscous_8th_nodes(z, p);
  if (phase != 1) viscous_8th_divergence(z, p);
}

void viscous_8th_nodes(Zone &z, const Param &p) {
  // collocated node fluxes (src/ViscousScheme.cu:470-585), then for mixtures the species
  // diffusion, its enthalpy and (two temperatures) the e_ve terms (:587-788)
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < z.mz; ++k)
    for (int j = 0; j < z.my; ++j)
      for (int i = 0; i < z.mx; ++i) {
        const bool bil = z.il[j + k * z.my] != 0, bir = z.ir[j + k * z.my] != 0;
        const bool bjl = z.jl[i + k * z.mx] != 0, bjr = z.jr[i + k * z.mx] != 0;
        const bool bkl = z.kl[i + j * z.mx] != 0, bkr = z.kr[i + j * z.mx] != 0;
        double d[6][3];
        for (int c : {1, 2, 3, 5}) {
          d[c][0] = d8([&](int m) { return z.bv(i + m, j, k, c); }, i, z.mx, bil, bir);
          d[c][1] = d8([&](int m) { return z.bv(i, j + m, k, c); }, j, z.my, bjl, bjr);
          d[c][2] = d8([&](int m) { return z.bv(i, j, k + m, c); }, k, z.mz, bkl, bkr);
        }
        const Arr &M = z.metric;
        const double xi_x = M(i, j, k, 0), xi_y = M(i, j, k, 1), xi_z = M(i, j, k, 2);
        const double eta_x = M(i, j, k, 3), eta_y = M(i, j, k, 4), eta_z = M(i, j, k, 5);
        const double zeta_x = M(i, j, k, 6), zeta_y = M(i, j, k, 7), zeta_z = M(i, j, k, 8);
        auto gx = [&](int c) { return d[c][0] * xi_x + d[c][1] * eta_x + d[c][2] * zeta_x; };
        auto gy = [&](int c) { return d[c][0] * xi_y + d[c][1] * eta_y + d[c][2] * zeta_y; };
        auto gz = [&](int c) { return d[c][0] * xi_z + d[c][1] * eta_z + d[c][2] * zeta_z; };
        const double u_x = gx(1), u_y = gy(1), u_z = gz(1), v_x = gx(2), v_y = gy(2), v_z = gz(2);
        const double w_x = gx(3), w_y = gy(3), w_z = gz(3);
        const double mul = z.mul(i, j, k);
        const double txx = mul * (4 * u_x - 2 * v_y - 2 * w_z) / 3.0;
        const double tyy = mul * (4 * v_y - 2 * u_x - 2 * w_z) / 3.0;
        const double tzz = mul * (4 * w_z - 2 * u_x - 2 * v_y) / 3.0;
        const double txy = mul * (u_y + v_x), txz = mul * (u_z + w_x), tyz = mul * (v_z + w_y);
        z.fF(i, j, k, 1) = xi_x * txx + xi_y * txy + xi_z * txz;
        z.fF(i, j, k, 2) = xi_x * txy + xi_y * tyy + xi_z * tyz;
        z.fF(i, j, k, 3) = xi_x * txz + xi_y * tyz + xi_z * tzz;
        z.gF(i, j, k, 1) = eta_x * txx + eta_y * txy + eta_z * txz;
        z.gF(i, j, k, 2) = eta_x * txy + eta_y * tyy + eta_z * tyz;
        z.gF(i, j, k, 3) = eta_x * txz + eta_y * tyz + eta_z * tzz;
        z.hF(i, j, k, 1) = zeta_x * txx + zeta_y * txy + zeta_z * txz;
        z.hF(i, j, k, 2) = zeta_x * txy + zeta_y * tyy + zeta_z * tyz;
        z.hF(i, j, k, 3) = zeta_x * txz + zeta_y * tyz + zeta_z * tzz;
        const double t_x = gx(5), t_y = gy(5), t_z = gz(5);
        const double cp = gamma_air * R_air / (gamma_air - 1);
        const double cond = p.n_spec == 0 ? mul / p.Pr * cp : z.kappa(i, j, k);
        const double u = z.bv(i, j, k, 1), v = z.bv(i, j, k, 2), w = z.bv(i, j, k, 3);
        const double Ex = u * txx + v * txy + w * txz + cond * t_x;
        const double Ey = u * txy + v * tyy + w * tyz + cond * t_y;
        const double Ez = u * txz + v * tyz + w * tzz + cond * t_z;
        z.fF(i, j, k, 4) = xi_x * Ex + xi_y * Ey + xi_z * Ez;
        z.gF(i, j, k, 4) = eta_x * Ex + eta_y * Ey + eta_z * Ez;
        z.hF(i, j, k, 4) = zeta_x * Ex + zeta_y * Ey + zeta_z * Ez;
        if (p.n_spec == 0) continue;
        // node gradient of a field c of array f projected on grad xi, grad eta, grad zeta
        auto proj = [&](const Arr &f, int c, double *g3) {
          const double a0 = d8([&](int m) { return f(i + m, j, k, c); }, i, z.mx, bil, bir);
          const double a1 = d8([&](int m) { return f(i, j + m, k, c); }, j, z.my, bjl, bjr);
          const double a2 = d8([&](int m) { return f(i, j, k + m, c); }, k, z.mz, bkl, bkr);
          const double fx = a0 * xi_x + a1 * eta_x + a2 * zeta_x;
          const double fy = a0 * xi_y + a1 * eta_y + a2 * zeta_y;
          const double fz = a0 * xi_z + a1 * eta_z + a2 * zeta_z;
          g3[0] = xi_x * fx + xi_y * fy + xi_z * fz;
          g3[1] = eta_x * fx + eta_y * fy + eta_z * fz;
          g3[2] = zeta_x * fx + zeta_y * fy + zeta_z * fz;
        };
        const bool tt = p.i_eve >= 0;
        double ef[3] = {0, 0, 0};
        if (tt) {  // kappa_ve grad T_ve in the energy flux (the collocated kernel's last lines)
          double gv3[3];
          proj(z.tve, 0, gv3);
          const double kve = z.kappa_ve(i, j, k);
          for (int a = 0; a < 3; ++a) ef[a] = kve * gv3[a];
          z.fF(i, j, k, 4) += ef[0];
          z.gF(i, j, k, 4) += ef[1];
          z.hF(i, j, k, 4) += ef[2];
        }
        const int ns = p.n_spec;
        double dif[16], yk[16], force[16][3], sw[3] = {0, 0, 0}, corr[3] = {0, 0, 0}, mwt = 0, srdy = 0;
        for (int l = 0; l < ns; ++l) {
          yk[l] = z.sv(i, j, k, l);
          dif[l] = z.rhoD(i, j, k, l);
          proj(z.sv, l, force[l]);
          for (int a = 0; a < 3; ++a) corr[a] += dif[l] * force[l][a];
          for (int a = 0; a < 3; ++a) sw[a] += force[l][a] * p.mech.imw[l];
          mwt += yk[l] * p.mech.imw[l];
          srdy += dif[l] * yk[l];
        }
        mwt = 1.0 / mwt;
        for (int a = 0; a < 3; ++a) corr[a] -= mwt * srdy * sw[a];
        if (p.gradP) {
          double gp[3];
          proj(z.bv, 4, gp);
          for (int a = 0; a < 3; ++a) gp[a] /= z.bv(i, j, k, 4);
          for (int l = 0; l < ns; ++l) {
            const double co = (mwt * p.mech.imw[l] - 1) * yk[l];
            for (int a = 0; a < 3; ++a) {
              force[l][a] += co * gp[a];
              corr[a] += co * gp[a] * dif[l];
            }
          }
        }
        double h[16];
        const double tm = z.bv(i, j, k, 5);
        nasa7_h(tm, p.mech, h);
        const double tve_m = tt ? z.tve(i, j, k) : tm;
        Arr *F[3] = {&z.fF, &z.gF, &z.hF};
        for (int l = 0; l < ns; ++l) {
          const double hd = tt ? h[l] - ve_energy(p, l, tm) + ve_energy(p, l, tve_m) : h[l];
          const double ev = tt ? ve_energy(p, l, tve_m) : 0.0;
          for (int a = 0; a < 3; ++a) {
            const double jd = dif[l] * (force[l][a] - mwt * yk[l] * sw[a]) - yk[l] * corr[a];
            (*F[a])(i, j, k, 5 + l) = jd;
            (*F[a])(i, j, k, 4) += hd * jd;
            if (tt) ef[a] += ev * jd;
          }
        }
        if (tt)
          for (int a = 0; a < 3; ++a) (*F[a])(i, j, k, 5 + p.i_eve) = ef[a];
      }
}

void viscous_8th_divergence(Zone &z, const Param &p) {
  // periodic exchange of the node fluxes (src/DataCommunication.cu:665-712)
  for (const auto &f : z.faces) {
    if (f.type != CB2_BC_PERIODIC) continue;
    int dir[3] = {0, 0, 0};
    dir[f.face] = f.direction;
    for (int k = f.start[2]; k <= f.end[2]; ++k)
      for (int j = f.start[1]; j <= f.end[1]; ++j)
        for (int i = f.start[0]; i <= f.end[0]; ++i) {
          int o[3] = {i, j, k};
          const int ext[3] = {z.mx, z.my, z.mz};
          o[f.face] = f.direction < 0 ? ext[f.face] - 1 : 0;
          for (int l = 0; l < p.n_var; ++l)
            for (const Arr *a : {&z.fF, &z.gF, &z.hF}) {
              const double ave = 0.5 * ((*a)(i, j, k, l) + (*a)(o[0], o[1], o[2], l));
              (*a)(i, j, k, l) = ave;
              (*a)(o[0], o[1], o[2], l) = ave;
            }
          for (int g = 1; g <= z.ngg; ++g)
            for (int l = 0; l < p.n_var; ++l)
              for (const Arr *a : {&z.fF, &z.gF, &z.hF})
                (*a)(i + g * dir[0], j + g * dir[1], k + g * dir[2], l) =
                    (*a)(o[0] + g * dir[0], o[1] + g * dir[1], o[2] + g * dir[2], l);
        }
  }
  // divergence (src/ViscousScheme.cu:790-834)
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < z.mz; ++k)
    for (int j = 0; j < z.my; ++j)
      for (int i = 0; i < z.mx; ++i) {
        const bool bil = z.il[j + k * z.my] != 0, bir = z.ir[j + k * z.my] != 0;
        const bool bjl = z.jl[i + k * z.mx] != 0, bjr = z.jr[i + k * z.mx] != 0;
        const bool bkl = z.kl[i + j * z.mx] != 0, bkr = z.kr[i + j * z.mx] != 0;
        const double jac = z.jac(i, j, k);
        for (int l = 1; l < p.n_var; ++l) {
          z.dq(i, j, k, l) += (d8([&](int m) { return z.fF(i + m, j, k, l); }, i, z.mx, bil, bir) +
                               d8([&](int m) { return z.gF(i, j + m, k, l); }, j, z.my, bjl, bjr) +
                               d8([&](int m) { return z.hF(i, j, k + m, l); }, k, z.mz, bkl, bkr)) *
                              jac;
        }
      }
}

// 2nd-order face flux at the face between (i,j,k) and its +1 neighbour along dir
// (compute_{fv,gv,hv}_2nd_order, src/ViscousScheme.cu:836-1512).
void viscous_face_2nd(const Zone &z, const Param &p, int dir, int i, int j, int k, double *fv) {
  int n[3] = {i, j, k};
  n[dir] += 1;
  const int in = n[0], jn = n[1], kn = n[2];
  const Arr &M = z.metric;
  double mt[9];
  for (int c = 0; c < 9; ++c) mt[c] = 0.5 * (M(i, j, k, c) + M(in, jn, kn, c));
  auto der = [&](const Arr &f, int c, double *d) {
    for (int a = 0; a < 3; ++a) {
      if (a == dir) d[a] = f(in, jn, kn, c) - f(i, j, k, c);
      else {
        int s[3] = {0, 0, 0};
        s[a] = 1;
        d[a] = 0.25 * (f(i + s[0], j + s[1], k + s[2], c) - f(i - s[0], j - s[1], k - s[2], c) +
                       f(in + s[0], jn + s[1], kn + s[2], c) - f(in - s[0], jn - s[1], kn - s[2], c));
      }
    }
  };
  double du[3], dv[3], dw[3], dt[3];
  der(z.bv, 1, du);
  der(z.bv, 2, dv);
  der(z.bv, 3, dw);
  der(z.bv, 5, dt);
  auto cx = [&](const double *d) { return d[0] * mt[0] + d[1] * mt[3] + d[2] * mt[6]; };
  auto cy = [&](const double *d) { return d[0] * mt[1] + d[1] * mt[4] + d[2] * mt[7]; };
  auto cz = [&](const double *d) { return d[0] * mt[2] + d[1] * mt[5] + d[2] * mt[8]; };
  const double u_x = cx(du), u_y = cy(du), u_z = cz(du), v_x = cx(dv), v_y = cy(dv), v_z = cz(dv);
  const double w_x = cx(dw), w_y = cy(dw), w_z = cz(dw);
  const double mul = 0.5 * (z.mul(i, j, k) + z.mul(in, jn, kn));
  const double txx = mul * (4 * u_x - 2 * v_y - 2 * w_z) / 3.0;
  const double tyy = mul * (4 * v_y - 2 * u_x - 2 * w_z) / 3.0;
  const double tzz = mul * (4 * w_z - 2 * u_x - 2 * v_y) / 3.0;
  const double txy = mul * (u_y + v_x), txz = mul * (u_z + w_x), tyz = mul * (v_z + w_y);
  const double jl = z.jac(i, j, k), jr = z.jac(in, jn, kn);
  const double kxj = 0.5 * (M(i, j, k, 3 * dir) * jl + M(in, jn, kn, 3 * dir) * jr);
  const double kyj = 0.5 * (M(i, j, k, 3 * dir + 1) * jl + M(in, jn, kn, 3 * dir + 1) * jr);
  const double kzj = 0.5 * (M(i, j, k, 3 * dir + 2) * jl + M(in, jn, kn, 3 * dir + 2) * jr);
  fv[0] = kxj * txx + kyj * txy + kzj * txz;
  fv[1] = kxj * txy + kyj * tyy + kzj * tyz;
  fv[2] = kxj * txz + kyj * tyz + kzj * tzz;
  const double um = 0.5 * (z.bv(i, j, k, 1) + z.bv(in, jn, kn, 1));
  const double vm = 0.5 * (z.bv(i, j, k, 2) + z.bv(in, jn, kn, 2));
  const double wm = 0.5 * (z.bv(i, j, k, 3) + z.bv(in, jn, kn, 3));
  const double t_x = cx(dt), t_y = cy(dt), t_z = cz(dt);
  double cond;
  if (p.n_spec == 0) cond = mul / p.Pr * (gamma_air * R_air / (gamma_air - 1));
  else cond = 0.5 * (z.kappa(i, j, k) + z.kappa(in, jn, kn));
  fv[3] = um * fv[0] + vm * fv[1] + wm * fv[2] + cond * (kxj * t_x + kyj * t_y + kzj * t_z);
  if (p.n_spec > 0) {
    const int ns = p.n_spec;
    double dif[16], yk[16], force[16];
    double sum_gy_w = 0, sum_rdy = 0, corr = 0, mwt = 0;
    for (int l = 0; l < ns; ++l) {
      yk[l] = 0.5 * (z.sv(i, j, k, l) + z.sv(in, jn, kn, l));
      dif[l] = 0.5 * (z.rhoD(i, j, k, l) + z.rhoD(in, jn, kn, l));
      double dy[3];
      der(z.sv, l, dy);
      const double gdy = kxj * cx(dy) + kyj * cy(dy) + kzj * cz(dy);
      force[l] = gdy;
      corr += dif[l] * gdy;
      sum_gy_w += gdy * p.mech.imw[l];
      mwt += yk[l] * p.mech.imw[l];
      sum_rdy += dif[l] * yk[l];
    }
    mwt = 1.0 / mwt;
    corr -= mwt * sum_rdy * sum_gy_w;
    if (p.gradP) {
      double dp[3];
      der(z.bv, 4, dp);
      const double gp = (kxj * cx(dp) + kyj * cy(dp) + kzj * cz(dp)) / (0.5 * (z.bv(in, jn, kn, 4) + z.bv(i, j, k, 4)));
      for (int l = 0; l < ns; ++l) {
        force[l] += (mwt * p.mech.imw[l] - 1) * yk[l] * gp;
        corr += (mwt * p.mech.imw[l] - 1) * yk[l] * gp * dif[l];
      }
    }
    double h[16];
    const double tm = 0.5 * (z.bv(i, j, k, 5) + z.bv(in, jn, kn, 5));
    nasa7_h(tm, p.mech, h);
    const bool tt = p.i_eve >= 0;
    const double tve_m = tt ? 0.5 * (z.tve(i, j, k) + z.tve(in, jn, kn)) : tm;
    for (int l = 0; l < ns; ++l) {
      const double jd = dif[l] * (force[l] - mwt * yk[l] * sum_gy_w) - yk[l] * corr;
      fv[4 + l] = jd;
      // two-temperature: the diffusing enthalpy carries e_ve at T_ve
      // (compute_nonequilibrium_diffusion_enthalpy, src/Thermo.cuh:43-47)
      const double hd = tt ? h[l] - ve_energy(p, l, tm) + ve_energy(p, l, tve_m) : h[l];
      fv[3] += hd * jd;
    }
    if (tt) {
      // e_ve conduction kappa_ve grad T_ve in the energy flux, and the e_ve flux
      // (src/ViscousScheme.cu:1024-1039)
      double dtv[3];
      der(z.tve, 0, dtv);
      const double kve = 0.5 * (z.kappa_ve(i, j, k) + z.kappa_ve(in, jn, kn));
      const double cond_ve = kve * (kxj * cx(dtv) + kyj * cy(dtv) + kzj * cz(dtv));
      fv[3] += cond_ve;
      double ef = cond_ve;
      for (int l = 0; l < ns; ++l) ef += ve_energy(p, l, tve_m) * fv[4 + l];
      fv[4 + p.i_eve] = ef;
    }
  }
}

void viscous_2nd(Zone &z, const Param &p) {
  const int ndir = z.mz == 1 ? 2 : 3;
  const int nf = p.n_var - 1;
  for (int dir = 0; dir < ndir; ++dir) {
    int lo[3] = {0, 0, 0};
    lo[dir] = -1;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = lo[2]; k < z.mz; ++k)
      for (int j = lo[1]; j < z.my; ++j)
        for (int i = lo[0]; i < z.mx; ++i) {
          double fv[16];
          viscous_face_2nd(z, p, dir, i, j, k, fv);
          for (int c = 0; c < nf; ++c) z.visf(i, j, k, c) = fv[c];
        }
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < z.mz; ++k)
      for (int j = 0; j < z.my; ++j)
        for (int i = 0; i < z.mx; ++i) {
          int a = i, b = j, c = k;
          shift(dir, -1, a, b, c);
          for (int q = 0; q < nf; ++q) z.dq(i, j, k, q + 1) += z.visf(i, j, k, q) - z.visf(a, b, c, q);
        }
  }
}

// Mixture-averaged transport (src/Transport.cu:43-150)
void transport(double t, double mw_total, const double *y, const double *cp, const Mechanism &m, double &mu,
               double &kappa, double *rhoD) {
  const int ns = m.n_spec;
  double X[16], vs[16];
  double temp = std::sqrt(t);
  for (int l = 0; l < ns; ++l) {
    X[l] = y[l] * mw_total / m.mw[l];
    const double tdl = t * m.lj_inv[l];
    vs[l] = m.vis_coeff[l] * temp / (1.147 * std::pow(tdl, -0.145) + std::pow(tdl + 0.5, -2));
  }
  const double t32 = t * temp;
  double visc = 0, cond = 0;
  for (int a = 0; a < ns; ++a) {
    double R = m.gas_const[a];
    double lambda = 15 * 0.25 * vs[a] * R;
    const double geom = m.geometry[a];
    if (geom == 1 || geom == 2) {
      const double t_red = t * m.kbe[a * ns + a];
      const double tri = 1 / t_red;
      const double tt = std::sqrt(tri * pi) * pi;
      const double FT = 1 + 0.5 * tt + (2 + 0.25 * pi * pi) * tri + tt * tri;
      const double omega = 1.0548 * std::pow(t_red, -0.15504) + std::pow(t_red + 0.55909, -2.1705);
      const double rd = m.bdc[a * ns + a] * t32 / (omega * R * t);
      if (geom == 1) {
        const double ad = (2.5 * vs[a] - rd) / ((pi * m.zrot[a] / FT * vs[a] + 10.0 / 3 * vs[a] + 2.0 * rd));
        lambda += -5 * ad * vs[a] * R + rd * cp[a] + rd * (2 * ad - 2.5) * R;
      } else {
        const double ad = (2.5 * vs[a] - rd) / ((pi * m.zrot[a] / FT * vs[a] + 5 * vs[a] + 2.0 * rd));
        lambda += -7.5 * ad * vs[a] * R + rd * cp[a] + rd * (3 * ad - 2.5) * R;
      }
    }
    double den = 0;
    R = std::sqrt(vs[a]);
    for (int b = 0; b < ns; ++b) {
      double phi = 1.0;
      if (a != b) {
        const double num = 1.0 + (1.0 / std::sqrt(vs[b])) * (R * m.wjwi14[a * ns + b]);
        phi = num * num * m.sqwiwj8[a * ns + b];
      }
      den += phi * X[b];
    }
    visc += vs[a] * X[a] / den;
    cond += lambda * X[a] / (1.065 * den - 0.065 * X[a]);
  }
  mu = visc;
  kappa = cond;
  const double eps = 1e-12;
  double num[16], dsum[16], sum = 0;
  for (int l = 0; l < ns; ++l) {
    num[l] = (X[l] + eps) * m.mw[l];
    sum += num[l];
    dsum[l] = 0;
  }
  for (int l = 0; l < ns; ++l) num[l] = sum - num[l];
  for (int l = 0; l < ns; ++l)
    for (int n = l + 1; n < ns; ++n) {
      const double tr = t * m.kbe[l * ns + n];
      const double omega = 1.0548 * std::pow(tr, -0.15504) + std::pow(tr + 0.55909, -2.1705);
      const double inv = omega / (m.bdc[l * ns + n] * t32);
      dsum[l] += (X[n] + eps) * inv;
      dsum[n] += (X[l] + eps) * inv;
    }
  const double ti = 1.0 / (t * R_u);
  for (int l = 0; l < ns; ++l) rhoD[l] = num[l] * ti / dsum[l];
}

// ---------------------------------------------------------------------------------------
// Finite-rate chemistry (src/FiniteRateChem.cu:1406-1681, generic mechanisms, 1T)
// ---------------------------------------------------------------------------------------
void gibbs_div_rt(double t, const Mechanism &m, double *g) {
  // compute_gibbs_div_rt (src/Thermo.cu:576-605)
  if (m.nasa == 9) {
    nasa9_gibbs_rt(t, m, g);
    return;
  }
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t_inv = 1 / t, log_t = std::log(t);
  for (int i = 0; i < m.n_spec; ++i) {
    if (t < m.t_low[i] || t > m.t_high[i]) {
      const double tt = t < m.t_low[i] ? m.t_low[i] : m.t_high[i];
      const double *c = (t < m.t_low[i] ? m.lo.data() : m.hi.data()) + 7 * i;
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt_inv = 1 / tt, log_tt = std::log(tt);
      g[i] = c[0] * (1.0 - log_tt) - 0.5 * c[1] * tt - c[2] * tt2 / 6.0 - c[3] * tt3 / 12.0 - c[4] * tt4 * 0.05 +
             c[5] * tt_inv - c[6];
    } else {
      const double *c = (t < m.t_mid[i] ? m.lo.data() : m.hi.data()) + 7 * i;
      g[i] = c[0] * (1.0 - log_t) - 0.5 * c[1] * t - c[2] * t2 / 6.0 - c[3] * t3 / 12.0 - c[4] * t4 * 0.05 +
             c[5] * t_inv - c[6];
    }
  }
}

double arrhenius(double t, double A, double b, double Ea) { return A * std::pow(t, b) * std::exp(-Ea / t); }

// Forward and backward rates of progress q1, q2 [mol/(cm^3 s)] of every reaction at t [K] and
// concentrations c [mol/cm^3].
// reaction_temperature / smooth_reaction_temperature (src/FiniteRateChem.cu:1490-1503)
double reaction_temperature(double t, double tve, double a, double b) {
  const double trx = std::pow(std::max(t, 1.0), a) * std::pow(std::max(tve, 1.0), b);
  constexpr double t_min = 800.0, eps = 80.0;
  return 0.5 * (trx + t_min + std::sqrt((trx - t_min) * (trx - t_min) + eps * eps));
}

void rates_of_progress(const Mechanism &m, double t0, double tve, const double *c, double *q1, double *q2) {
  const int ns = m.n_spec, nr = m.n_reac;
  double kf[32], kb[32];
  // forward_reaction_rate (:1505-1554); with the control-temperature model each reaction runs
  // at its own smoothed T^a Tve^b
  for (int i = 0; i < nr; ++i) {
    const double t = m.park ? reaction_temperature(t0, tve, m.tcf_a[i], m.tcf_b[i]) : t0;
    kf[i] = arrhenius(t, m.A[i], m.b[i], m.Ea[i]);
    const int ty = m.reac_type[i];
    if (ty == 3) {
      kf[i] += arrhenius(t, m.A2[i], m.b2[i], m.Ea2[i]);
    } else if (ty > 3) {
      double cc = 0;
      for (int l = 0; l < ns; ++l) cc += c[l] * m.tbc[i * ns + l];
      if (ty == 4) {
        kf[i] *= cc;
      } else {
        const double kf_low = arrhenius(t, m.A2[i], m.b2[i], m.Ea2[i]);
        const double kf_high = kf[i];
        if (kf_high < 1e-25 && kf_low < 1e-25) {
          kf[i] = 0;
          continue;
        }
        const double pr = kf_low * cc / kf_high;
        double F = 1.0;
        if (ty > 5) {
          double fc = (1 - m.troe_alpha[i]) * std::exp(-t / m.troe_t3[i]) + m.troe_alpha[i] * std::exp(-t / m.troe_t1[i]);
          if (ty == 7) fc += std::exp(-m.troe_t2[i] / t);
          const double lfc = std::log10(fc);
          const double cq = -0.4 - 0.67 * lfc;
          const double nq = 0.75 - 1.27 * lfc;
          const double lpr = std::log10(pr);
          const double tempo = (lpr + cq) / (nq - 0.14 * (lpr + cq));
          const double pp = lfc / (1.0 + tempo * tempo);
          F = std::pow(10, pp);
        }
        kf[i] = kf_high * pr / (1.0 + pr) * F;
      }
    }
  }
  // backward_reaction_rate (:1560-1592) with the control-temperature model: per reaction at
  // its own backward temperature, g/RT evaluated there
  if (m.park) {
    for (int i = 0; i < nr; ++i) {
      const double thb = reaction_temperature(t0, tve, m.tcb_a[i], m.tcb_b[i]);
      if (m.reac_type[i] == 0) {
        kb[i] = 0;
        continue;
      }
      if (m.rev_type[i] == 1) {
        kb[i] = arrhenius(thb, m.A2[i], m.b2[i], m.Ea2[i]);
        if (m.reac_type[i] == 4) {
          double cc = 0;
          for (int l = 0; l < ns; ++l) cc += c[l] * m.tbc[i * ns + l];
          kb[i] *= cc;
        }
        continue;
      }
      double g[16];
      gibbs_div_rt(thb, m, g);
      const double temp_t = p_atm / R_u * 1e-3 / thb;
      double dg = 0;
      for (int l = 0; l < ns; ++l) dg += g[l] * (m.stoi_b[i * ns + l] - m.stoi_f[i * ns + l]);
      const double kc = std::pow(temp_t, m.reac_order[i]) * std::exp(-dg);
      kb[i] = kf[i] / kc;
    }
  }
  // backward_reaction_rate (:1593-1636)
  const double t = t0;
  int n_gibbs = m.park ? 0 : nr;
  for (int i = 0; i < nr && !m.park; ++i) {
    if (m.reac_type[i] == 0) {
      kb[i] = 0;
      --n_gibbs;
    } else if (m.rev_type[i] == 1) {
      kb[i] = arrhenius(t, m.A2[i], m.b2[i], m.Ea2[i]);
      if (m.reac_type[i] == 4) {
        double cc = 0;
        for (int l = 0; l < ns; ++l) cc += c[l] * m.tbc[i * ns + l];
        kb[i] *= cc;
      }
      --n_gibbs;
    }
  }
  if (n_gibbs >= 1) {
    double g[16];
    gibbs_div_rt(t, m, g);
    const double temp_p = p_atm / R_u * 1e-3;
    const double temp_t = temp_p / t;
    for (int i = 0; i < nr; ++i) {
      if (m.reac_type[i] != 2 && m.reac_type[i] != 0) {
        double dg = 0;
        for (int l = 0; l < ns; ++l) dg += g[l] * (m.stoi_b[i * ns + l] - m.stoi_f[i * ns + l]);
        const double kc = std::pow(temp_t, m.reac_order[i]) * std::exp(-dg);
        kb[i] = kf[i] / kc;
      }
    }
  }
  // rate_of_progress (:1638-1663)
  for (int i = 0; i < nr; ++i) {
    q1[i] = 1.0;
    q2[i] = m.reac_type[i] != 0 ? 1.0 : 0.0;
    for (int j = 0; j < ns; ++j) {
      q1[i] *= std::pow(c[j], m.stoi_f[i * ns + j]);
      if (m.reac_type[i] != 0) q2[i] *= std::pow(c[j], m.stoi_b[i * ns + j]);
    }
    q1[i] *= kf[i];
    if (m.reac_type[i] != 0) q2[i] *= kb[i];
  }
}

void chemistry_point(const Mechanism &m, double rho, double t, double tve, const double *y, double *omega,
                     double *omega_d) {
  const int ns = m.n_spec, nr = m.n_reac;
  double c[16], q1[32], q2[32];
  for (int l = 0; l < ns; ++l) c[l] = rho * y[l] * m.imw[l] * 1e-3;
  rates_of_progress(m, t, tve, c, q1, q2);
  // chemical_source (:1665-1681)
  for (int i = 0; i < ns; ++i) {
    double creation = 0;
    omega_d[i] = 0;
    for (int j = 0; j < nr; ++j) {
      creation += q2[j] * m.stoi_f[j * ns + i] + q1[j] * m.stoi_b[j * ns + i];
      omega_d[i] += q1[j] * m.stoi_f[j * ns + i] + q2[j] * m.stoi_b[j * ns + i];
    }
    creation *= 1e+3 / m.imw[i];
    omega_d[i] *= 1e+3 / m.imw[i];
    omega[i] = creation - omega_d[i];
  }
}

void finite_rate_chemistry(Zone &z, const Param &p) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < z.mz; ++k)
    for (int j = 0; j < z.my; ++j)
      for (int i = 0; i < z.mx; ++i) {
        const int ns = p.n_spec;
        double y[16], om[16], od[16];
        for (int l = 0; l < ns; ++l) y[l] = z.sv(i, j, k, l);
        const double rho = z.bv(i, j, k, 0), t = z.bv(i, j, k, 5);
        // the rates see max(T_ve, 1) (:1450-1451)
        const double tve = p.i_eve >= 0 ? std::max(z.tve(i, j, k), 1.0) : t;
        chemistry_point(p.mech, rho, t, tve, y, om, od);
        double ts = 1e+6;
        for (int l = 0; l < ns; ++l) {
          z.dq(i, j, k, l + 5) += z.jac(i, j, k) * om[l];
          if (y[l] > 1e-25 && std::fabs(od[l]) > 1e-25) ts = std::min(ts, std::fabs(rho * y[l] / od[l]));
        }
        if (p.i_eve >= 0) {
          // compute_two_temperature_chemical_source (:19-31): sum_l omega_l e_ve,l(T_ve)
          double tv = z.tve(i, j, k);
          if (tv <= 0.0) tv = std::max(t, 1.0);
          double src = 0.0;
          for (int l = 0; l < ns; ++l) src += om[l] * ve_energy(p, l, tv);
          z.dq(i, j, k, 5 + p.i_eve) += z.jac(i, j, k) * src;
        }
        if (z.rts) z.rts(i, j, k) = ts;
      }
}

double sutherland(double t) { return 1.7894e-5 * std::pow(t / 288.16, 1.5) * (288.16 + 110) / (t + 110); }

void cv_point(Zone &z, const Param &p, int i, int j, int k) {
  // compute_cv_from_bv_1_point + compute_total_energy (src/FieldOperation.cuh:90-181)
  const double rho = z.bv(i, j, k, 0);
  z.cv(i, j, k, 0) = rho;
  z.cv(i, j, k, 1) = rho * z.bv(i, j, k, 1);
  z.cv(i, j, k, 2) = rho * z.bv(i, j, k, 2);
  z.cv(i, j, k, 3) = rho * z.bv(i, j, k, 3);
  if (p.i_eve >= 0) sync_two_temperature(z, p, i, j, k);
  for (int l = 0; l < p.n_scalar; ++l) z.cv(i, j, k, 5 + l) = rho * z.sv(i, j, k, l);
  if (p.i_eve >= 0) {
    z.cv(i, j, k, 4) = total_energy_2t(z, p, i, j, k);
    return;
  }
  const double V2 = z.bv(i, j, k, 1) * z.bv(i, j, k, 1) + z.bv(i, j, k, 2) * z.bv(i, j, k, 2) +
                    z.bv(i, j, k, 3) * z.bv(i, j, k, 3);
  double E = 0.5 * V2;
  if (p.n_spec == 0) {
    E *= z.bv(i, j, k, 0);
    E += z.bv(i, j, k, 4) / (gamma_air - 1);
  } else {
    double h[16];
    nasa7_h(z.bv(i, j, k, 5), p.mech, h);
    for (int l = 0; l < p.n_spec; ++l) E += h[l] * z.sv(i, j, k, l);
    E *= z.bv(i, j, k, 0);
    E -= z.bv(i, j, k, 4);
  }
  z.cv(i, j, k, 4) = E;
}

}  // namespace

void reaction_rates(const Mechanism &m, double t, const double *c, double *q1, double *q2) {
  rates_of_progress(m, t, t, c, q1, q2);
}

void nasa7_h_cp(double t, const Mechanism &m, double *h, double *cp) {
  // compute_enthalpy_and_cp (src/Thermo.cu:453-523)
  if (m.nasa == 9) {
    nasa9_h_cp(t, m, h, cp);
    return;
  }
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
  for (int i = 0; i < m.n_spec; ++i) {
    if (t < m.t_low[i] || t > m.t_high[i]) {
      const double tt = t < m.t_low[i] ? m.t_low[i] : m.t_high[i];
      const double *c = (t < m.t_low[i] ? m.lo.data() : m.hi.data()) + 7 * i;
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt5 = tt4 * tt;
      h[i] = c[0] * tt + 0.5 * c[1] * tt2 + c[2] * tt3 / 3 + 0.25 * c[3] * tt4 + 0.2 * c[4] * tt5 + c[5];
      cp[i] = c[0] + c[1] * tt + c[2] * tt2 + c[3] * tt3 + c[4] * tt4;
      h[i] += cp[i] * (t - tt);
    } else {
      const double *c = (t < m.t_mid[i] ? m.lo.data() : m.hi.data()) + 7 * i;
      h[i] = c[0] * t + 0.5 * c[1] * t2 + c[2] * t3 / 3 + 0.25 * c[3] * t4 + 0.2 * c[4] * t5 + c[5];
      cp[i] = c[0] + c[1] * t + c[2] * t2 + c[3] * t3 + c[4] * t4;
    }
    h[i] *= m.gas_const[i];
    cp[i] *= m.gas_const[i];
  }
}

static long long g_step = 0;
void set_step(long long step) { g_step = step; }

Param make_param(const cb2_param_view &pv) {
  Param p;
  p.dim = pv.dim;
  p.n_var = pv.n_var;
  p.n_spec = pv.n_spec;
  p.n_scalar = pv.n_scalar;
  p.n_scalar_transported = pv.n_scalar_transported;
  p.inviscid_scheme = pv.inviscid_scheme;
  p.reconstruction = pv.reconstruction;
  p.limiter = pv.limiter;
  p.viscous_order = pv.viscous_order;
  p.positive_preserving = pv.positive_preserving;
  p.gradP = pv.gradP_in_diffusion_flux;
  p.reaction = pv.reaction;
  p.shock_sensor = pv.shock_sensor;
  p.sensor_eps = pv.sensor_eps;
  p.sensor_threshold = pv.sensor_threshold;
  p.entropy_fix_factor = pv.entropy_fix_factor;
  p.Pr = pv.Pr;
  p.cfl = pv.cfl;
  p.rho_ref = pv.rho_ref;
  p.v_ref = pv.v_ref;
  p.weno_eps_scale = pv.rho_ref * pv.v_ref * pv.rho_ref * pv.v_ref;
  p.mu_constant = pv.mu_constant;
  p.dt = pv.dt;
  p.limit_flow = pv.limit_flow;
  if (p.limit_flow) {
    // src/DParameter.cu:371-387
    p.lf_ll[0] = 1e-6 * pv.rho_ref;
    p.lf_ul[0] = 1e+3 * pv.rho_ref;
    const double vref = std::fabs(pv.v_ref) < 1 ? pv.c_ref : pv.v_ref;
    for (int l = 1; l < 4; ++l) {
      p.lf_ll[l] = -1000 * vref;
      p.lf_ul[l] = 1000 * vref;
    }
    p.lf_ll[4] = 1e-6 * pv.p_ref;
    p.lf_ul[4] = 1e+3 * pv.p_ref;
  }
  if (pv.mech) {
    const cb2_mechanism &m = *pv.mech;
    Mechanism &o = p.mech;
    const int ns = m.n_spec, nr = m.n_reac;
    o.n_spec = ns;
    o.n_reac = nr;
    p.n_reac = nr;
    auto cp = [](const double *s, size_t n) { return s ? std::vector<double>(s, s + n) : std::vector<double>(n, 0.0); };
    auto cpi = [](const int *s, size_t n) { return s ? std::vector<int>(s, s + n) : std::vector<int>(n, 0); };
    o.imw.resize(ns);
    o.gas_const.resize(ns);
    o.mw.resize(ns);
    for (int s = 0; s < ns; ++s) {
      o.imw[s] = 1.0 / m.mw[s];              // src/DParameter.cu:96
      o.gas_const[s] = R_u / m.mw[s];        // src/DParameter.cu:97
      o.mw[s] = 1.0 / o.imw[s];              // src/Transport.cu:57
    }
    if (m.therm_nasa_7_9 == 9) {
      o.nasa = 9;
      o.max_range = m.max_range;
      o.n_range = cpi(m.n_temperature_range, ns);
      o.t_cut = cp(m.temperature_range, ns * (m.max_range + 1));
      o.poly9 = cp(m.therm_poly_coeff, ns * m.max_range * 9);
    }
    o.park = m.two_temperature_reaction_temperature != 0;
    if (o.park) {
      o.tcf_a = cp(m.tcf_a, nr);
      o.tcf_b = cp(m.tcf_b, nr);
      o.tcb_a = cp(m.tcb_a, nr);
      o.tcb_b = cp(m.tcb_b, nr);
    }
    o.lo = cp(m.low_temp_coeff, ns * 7);
    o.hi = cp(m.high_temp_coeff, ns * 7);
    o.t_low = cp(m.t_low, ns);
    o.t_mid = cp(m.t_mid, ns);
    o.t_high = cp(m.t_high, ns);
    o.geometry = cp(m.geometry, ns);
    o.lj_inv = cp(m.LJ_potent_inv, ns);
    o.vis_coeff = cp(m.vis_coeff, ns);
    o.wjwi14 = cp(m.WjDivWi_to_One4th, ns * ns);
    o.sqwiwj8 = cp(m.sqrt_WiDivWjPl1Mul8, ns * ns);
    o.bdc = cp(m.binary_diffusivity_coeff, ns * ns);
    o.kbe = cp(m.kb_over_eps_jk, ns * ns);
    o.zrot = cp(m.ZRotF298, ns);
    o.reac_type = cpi(m.reac_type, nr);
    o.rev_type = cpi(m.rev_type, nr);
    o.stoi_f = cpi(m.stoi_f, nr * ns);
    o.stoi_b = cpi(m.stoi_b, nr * ns);
    o.reac_order = cpi(m.reac_order, nr);
    o.A = cp(m.A, nr);
    o.b = cp(m.b, nr);
    o.Ea = cp(m.Ea, nr);
    o.A2 = cp(m.A2, nr);
    o.b2 = cp(m.b2, nr);
    o.Ea2 = cp(m.Ea2, nr);
    o.tbc = cp(m.third_body_coeff, nr * ns);
    o.troe_alpha = cp(m.troe_alpha, nr);
    o.troe_t3 = cp(m.troe_t3, nr);
    o.troe_t1 = cp(m.troe_t1, nr);
    o.troe_t2 = cp(m.troe_t2, nr);
  }
  if (pv.two_t && pv.mech) {
    // DParameter two-temperature tables (src/DParameter.cu:150-200); i_eve = n_spec
    // (src/Parameter.cpp:647-656)
    const cb2_two_temperature &t = *pv.two_t;
    const int ns = t.n_spec, ml = t.max_level;
    TwoTemperature &o = p.tt;
    o.on = true;
    o.enable_vt = t.enable_vt_relaxation != 0;
    o.max_level = ml;
    o.theta_v.assign(t.theta_v, t.theta_v + ns);
    o.n_level.assign(t.n_level, t.n_level + ns);
    o.elec_theta.assign(t.elec_theta, t.elec_theta + ns * ml);
    o.elec_g.assign(t.elec_g, t.elec_g + ns * ml);
    o.lt_a.assign(t.lt_a, t.lt_a + ns * ns);
    o.lt_b.assign(t.lt_b, t.lt_b + ns * ns);
    o.park_sigma.assign(t.park_sigma, t.park_sigma + ns);
    p.i_eve = p.n_spec;
  }
  p.step = g_step;
  return p;
}

Zone make_zone(const cb2_zone_view &v, const cb2_face_bc *faces, int n_faces, const Param &p) {
  Zone z;
  z.mx = v.mx; z.my = v.my; z.mz = v.mz; z.ngg = v.ngg;
  const int g = v.ngg;
  auto A = [&](double *ptr, int gg) { return Arr(ptr, v.mx, v.my, v.mz, gg); };
  z.cv = A(v.cv, g); z.bv = A(v.bv, g); z.sv = A(v.sv, g); z.qn = A(v.qn, g); z.dq = A(v.dq, 0);
  z.metric = A(v.metric, g); z.jac = A(v.jac, g); z.mul = A(v.mul, g); z.kappa = A(v.thermal_conductivity, g);
  z.rhoD = A(v.rho_D, g); z.acoustic = A(v.acoustic_speed, g); z.gamma = A(v.gamma, g); z.mach = A(v.mach, g);
  z.fF = A(v.fFlux, g); z.gF = A(v.gFlux, g); z.hF = A(v.hFlux, g); z.visf = A(v.vis_flux, 1);
  z.shock = A(v.shock_sensor, g); z.dtl = A(v.dt_local, 0); z.rts = A(v.reaction_timeScale, g);
  z.efd = A(v.entropy_fix_delta, 1);
  z.tve = A(v.temperature_ve, g);
  z.kappa_ve = A(v.thermal_conductivity_ve, g);
  const int mx = v.mx, my = v.my, mz = v.mz;
  z.il.assign(my * mz, 0); z.ir.assign(my * mz, 0); z.jl.assign(mx * mz, 0); z.jr.assign(mx * mz, 0);
  z.kl.assign(mx * my, 0); z.kr.assign(mx * my, 0);
  const bool extend = p.viscous_order == 2;
  for (int f = 0; f < n_faces; ++f) {
    const cb2_face_bc &b = faces[f];
    FaceBC o;
    o.type = b.type & ~CB2_BC_NONREFLECTING;
    o.nonreflecting = (b.type & CB2_BC_NONREFLECTING) != 0;
    o.face = b.face; o.direction = b.direction;
    for (int a = 0; a < 3; ++a) { o.start[a] = b.range_start[a]; o.end[a] = b.range_end[a]; }
    // register_boundary (src/Mesh.cpp:14-32)
    const int gx = extend ? g : 0;
    for (int a = 0; a < p.dim; ++a) {
      if (a == o.face) continue;
      if (o.end[a] < o.start[a]) std::swap(o.start[a], o.end[a]);
      o.start[a] -= gx;
      o.end[a] += gx;
    }
    if (p.dim == 2) { o.start[2] = -gx; o.end[2] = gx; }
    o.rho = b.rho; o.u = b.u; o.v = b.v; o.w = b.w; o.p = b.p; o.T = b.T; o.wall_T = b.wall_temperature;
    o.wall_Tve = b.wall_temperature_ve;
    // a wall's sv: its mass fractions when fully catalytic (Wall::yk, n_spec values)
    if (b.sv) o.sv.assign(b.sv, b.sv + (o.type == CB2_BC_WALL ? p.n_spec : p.n_scalar));
    o.blow = o.type == CB2_BC_WALL && b.blow_shock_wave != 0;
    o.blow_start = b.blow_start_step;
    o.blow_end = b.blow_end_step;
    o.blow_coef = b.blow_coefficient;
    z.faces.push_back(o);
    if (b.type == CB2_BC_PERIODIC) continue;
    int lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::max(0, std::min(b.range_start[a], b.range_end[a]));
      hi[a] = std::max(b.range_start[a], b.range_end[a]);
    }
    hi[0] = std::min(hi[0], mx - 1); hi[1] = std::min(hi[1], my - 1); hi[2] = std::min(hi[2], mz - 1);
    for (int k = lo[2]; k <= hi[2]; ++k)
      for (int j = lo[1]; j <= hi[1]; ++j)
        for (int i = lo[0]; i <= hi[0]; ++i) {
          if (b.face == 0) (b.direction < 0 ? z.il : z.ir)[j + k * my] = o.type;
          else if (b.face == 1) (b.direction < 0 ? z.jl : z.jr)[i + k * mx] = o.type;
          else (b.direction < 0 ? z.kl : z.kr)[i + j * mx] = o.type;
        }
  }
  return z;
}

// update_cv_and_bv_rk (src/RK.cuh:277-367) with compute_temperature_and_pressure
// (src/FieldOperation.cu:4-94)
// limit_flow (src/TimeAdvanceFunc.cuh:129-232), read from the state the stage update left: a
// bad node (NaN or rho, u, v, w, p outside the bounds) takes the mean of the good nodes of its
// 3x3x3 neighbourhood, or its own clamped values if none is good; then T and cv.  The
// reference updates in place from parallel threads; reading only the pre-limit state is the
// race-free reading of the same rule.
static bool lf_bad(const Zone &z, const Param &p, int i, int j, int k) {
  for (int l = 0; l < 5; ++l) {
    const double v = z.bv(i, j, k, l);
    if (std::isnan(v) || v < p.lf_ll[l] || v > p.lf_ul[l]) return true;
  }
  return false;
}

void limit_flow(Zone &z, const Param &p) {
  std::vector<std::array<double, 6>> fix;
  for (int k = 0; k < z.mz; ++k)
    for (int j = 0; j < z.my; ++j)
      for (int i = 0; i < z.mx; ++i) {
        if (!lf_bad(z, p, i, j, k)) continue;
        double v[5] = {0, 0, 0, 0, 0};
        int kn = 0;
        for (int ka = -1; ka < 2; ++ka) {
          const int k1 = k + ka;
          if (k1 < 0 || k1 >= z.mz) continue;
          for (int ja = -1; ja < 2; ++ja) {
            const int j1 = j + ja;
            if (j1 < 0 || j1 >= z.my) continue;
            for (int ia = -1; ia < 2; ++ia) {
              const int i1 = i + ia;
              if (i1 < 0 || i1 >= z.mx) continue;
              if (lf_bad(z, p, i1, j1, k1)) continue;
              for (int l = 0; l < 5; ++l) v[l] += z.bv(i1, j1, k1, l);
              ++kn;
            }
          }
        }
        if (kn > 0) {
          const double inv = 1.0 / kn;
          for (double &x : v) x *= inv;
        } else {
          for (int l = 0; l < 5; ++l) v[l] = std::min(std::max(z.bv(i, j, k, l), p.lf_ll[l]), p.lf_ul[l]);
        }
        const double idx = (double)((k * z.my + j) * z.mx + i);
        fix.push_back({idx, v[0], v[1], v[2], v[3], v[4]});
      }
  for (const auto &f : fix) {
    const long n = (long)f[0];
    const int i = (int)(n % z.mx), j = (int)((n / z.mx) % z.my), k = (int)(n / ((long)z.mx * z.my));
    for (int l = 0; l < 5; ++l) z.bv(i, j, k, l) = f[1 + l];
    if (p.n_spec == 0) {
      z.bv(i, j, k, 5) = f[5] * mw_air / (f[1] * R_u);
    } else {
      double r = 0;
      for (int s = 0; s < p.n_spec; ++s) r += z.sv(i, j, k, s) * p.mech.gas_const[s];
      z.bv(i, j, k, 5) = f[5] / (f[1] * r);
    }
    cv_point(z, p, i, j, k);
  }
}

void update_cv_and_bv_rk(Zone &z, const Param &p, double dt, int rk) {
  const double A[3] = {1.0, 0.75, 1.0 / 3.0}, B[3] = {0.0, 0.25, 2.0 / 3.0}, C[3] = {1.0, 0.25, 2.0 / 3.0};
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < z.mz; ++k)
    for (int j = 0; j < z.my; ++j)
      for (int i = 0; i < z.mx; ++i) {
        const double dt_div_jac = dt / z.jac(i, j, k);
        for (int l = 0; l < p.n_var; ++l)
          z.cv(i, j, k, l) = A[rk] * z.qn(i, j, k, l) + B[rk] * z.cv(i, j, k, l) + C[rk] * dt_div_jac * z.dq(i, j, k, l);
        if (z.mz == 1) z.cv(i, j, k, 3) = 0;
        z.bv(i, j, k, 0) = z.cv(i, j, k, 0);
        const double dinv = 1.0 / z.cv(i, j, k, 0);
        z.bv(i, j, k, 1) = z.cv(i, j, k, 1) * dinv;
        z.bv(i, j, k, 2) = z.cv(i, j, k, 2) * dinv;
        z.bv(i, j, k, 3) = z.cv(i, j, k, 3) * dinv;
        const double V2 = z.bv(i, j, k, 1) * z.bv(i, j, k, 1) + z.bv(i, j, k, 2) * z.bv(i, j, k, 2) +
                          z.bv(i, j, k, 3) * z.bv(i, j, k, 3);
        if (p.n_spec == 0) {
          z.bv(i, j, k, 4) = (gamma_air - 1) * (z.cv(i, j, k, 4) - 0.5 * z.bv(i, j, k, 0) * V2);
          z.bv(i, j, k, 5) = z.bv(i, j, k, 4) * mw_air * dinv / R_u;
          continue;
        }
        double sum = 0;
        for (int l = 0; l < p.n_spec; ++l) {
          if (z.cv(i, j, k, 5 + l) < 0) z.cv(i, j, k, 5 + l) = 0;
          else sum += z.cv(i, j, k, l + 5);
        }
        if (p.i_eve >= 0) z.cv(i, j, k, 5 + p.i_eve) = std::max(z.cv(i, j, k, 5 + p.i_eve), 0.0);
        sum = 1.0 / sum;
        const double scale = z.cv(i, j, k, 0) * sum;
        for (int l = 0; l < p.n_spec; ++l) {
          z.sv(i, j, k, l) = z.cv(i, j, k, 5 + l) * sum;
          z.cv(i, j, k, 5 + l) *= scale;
        }
        for (int l = p.n_spec; l < p.n_scalar; ++l) z.sv(i, j, k, l) = z.cv(i, j, k, 5 + l) * dinv;
        if (p.i_eve >= 0) {
          temperature_2t(z, p, i, j, k, z.cv(i, j, k, 4));
          continue;
        }
        // Newton T from e (1T), |1 - T1/T| < 1e-5, at most 1000 iterations
        double gc = 0;
        for (int l = 0; l < p.n_spec; ++l) gc += z.sv(i, j, k, l) * p.mech.gas_const[l];
        const double rho = z.bv(i, j, k, 0);
        const double e = z.cv(i, j, k, 4) / rho - 0.5 * V2;
        double err = 1, t = z.bv(i, j, k, 5);
        int iter = 0;
        double h[16], cp[16];
        while (err > 1e-5 && iter++ < 1000) {
          nasa7_h_cp(t, p.mech, h, cp);
          double cpt = 0, hh = 0;
          for (int l = 0; l < p.n_spec; ++l) {
            cpt += cp[l] * z.sv(i, j, k, l);
            hh += h[l] * z.sv(i, j, k, l);
          }
          const double et = hh - gc * t, cv = cpt - gc;
          const double t1 = t - (et - e) / cv;
          err = std::fabs(1 - t1 / t);
          t = t1;
        }
        z.bv(i, j, k, 5) = t;
        z.bv(i, j, k, 4) = rho * t * gc;
      }
  // two-temperature: VT relaxation over the stage's share of the step, rk_stage_dt_scale
  // {1, 1/4, 2/3} (src/RK.cuh:91, 199-203)
  if (p.i_eve >= 0) apply_vt_relaxation(z, p, C[rk] * dt);
  if (p.limit_flow) limit_flow(z, p);
}

void compute_cv_from_bv(Zone &z, const Param &p) {
  const int g = z.ngg;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = -g; k < z.mz + g; ++k)
    for (int j = -g; j < z.my + g; ++j)
      for (int i = -g; i < z.mx + g; ++i) cv_point(z, p, i, j, k);
}

void compute_inviscid_flux(Zone &z, const Param &p) {
  const int ndir = z.mz > 1 ? 3 : 2;
  const bool ch = p.inviscid_scheme == 52 || p.inviscid_scheme == 72;
  const bool cp = p.inviscid_scheme == 51 || p.inviscid_scheme == 71;
  if (!ch && !cp && p.inviscid_scheme == 2) entropy_fix_delta(z, p);
  for (int d = 0; d < ndir; ++d) {
    if (ch) convective_term_weno_char(z, p, d);
    else if (cp) convective_term_weno_comp(z, p, d);
    else convective_term_pv(z, p, d);
  }
}

void compute_chemistry(Zone &z, const Param &p) { finite_rate_chemistry(z, p); }

void chemistry_source(const Mechanism &m, double rho, double t, const double *y, double *omega, double *omega_d) {
  chemistry_point(m, rho, t, t, y, omega, omega_d);
}

void species_gibbs_rt(double t, const Mechanism &m, double *g) { gibbs_div_rt(t, m, g); }

void chemistry_source_2t(const Mechanism &m, double rho, double t, double tve, const double *y, double *omega,
                         double *omega_d) {
  chemistry_point(m, rho, t, tve, y, omega, omega_d);
}

void compute_viscous_flux(Zone &z, const Param &p, int phase) {
  if (p.viscous_order == 8) viscous_8th(z, p, phase);
  else if (p.viscous_order == 2 && phase != 2) viscous_2nd(z, p);
}

// exchange_value task 1 over the inner faces (inner_exchange, src/DataCommunication.cu:437-527):
// the node fluxes averaged on each coincident face layer, copied into the ghost layers
void inner_flux_exchange(std::vector<Zone> &zones, const Param &p) {
  for (auto &z : zones)
    for (const auto &f : z.inner) {
      Zone &t = zones[f.target_block];
      const int face_layer = f.direction > 0 ? f.range_start[f.face] : f.range_end[f.face];
      for (int n2 = 0; n2 < f.n_point[2]; ++n2)
        for (int n1 = 0; n1 < f.n_point[1]; ++n1)
          for (int n0 = 0; n0 < f.n_point[0]; ++n0) {
            const int n[3] = {n0, n1, n2};
            int idx[3], it[3], d[3];
            for (int a = 0; a < 3; ++a) {
              d[a] = f.loop_dir[a] * n[a];
              idx[a] = f.range_start[a] + d[a];
            }
            for (int a = 0; a < 3; ++a) it[a] = f.target_start[a] + f.target_loop_dir[a] * d[f.src_tar[a]];
            const bool coincident = idx[f.face] == face_layer;
            for (int l = 0; l < p.n_var; ++l) {
              const Arr *mine[3] = {&z.fF, &z.gF, &z.hF}, *theirs[3] = {&t.fF, &t.gF, &t.hF};
              for (int a = 0; a < 3; ++a) {
                double &x = (*mine[a])(idx[0], idx[1], idx[2], l);
                double &y = (*theirs[a])(it[0], it[1], it[2], l);
                if (coincident) {
                  const double ave = 0.5 * (x + y);
                  x = ave;
                  y = ave;
                } else {
                  x = y;
                }
              }
            }
          }
    }
}

// compute_viscous_flux over the whole mesh (src/ViscousScheme.cu:14-100): every zone's dq starts
// from zero and takes its viscous term; 8th-order node fluxes are exchanged across inner faces
// between the node fluxes and the divergences
void viscous_all(std::vector<Zone> &zones, const Param &p) {
  for (auto &z : zones) {
    std::memset(z.dq.p, 0, (size_t)z.dq.sz * p.n_var * sizeof(double));
    compute_viscous_flux(z, p, p.viscous_order == 8 ? 1 : 0);
  }
  if (p.viscous_order == 8) {
    inner_flux_exchange(zones, p);
    for (auto &z : zones) compute_viscous_flux(z, p, 2);
  }
}

// update_physical_properties (src/FieldOperation.cuh:183-247)
void update_physical_properties(Zone &z, const Param &p) {
  const int g = z.ngg;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = -g; k < z.mz + g; ++k)
    for (int j = -g; j < z.my + g; ++j)
      for (int i = -g; i < z.mx + g; ++i) {
        const double t = z.bv(i, j, k, 5);
        const double V = std::sqrt(sqr(z.bv(i, j, k, 1)) + sqr(z.bv(i, j, k, 2)) + sqr(z.bv(i, j, k, 3)));
        if (p.n_spec == 0) {
          if (z.mul) z.mul(i, j, k) = p.mu_constant > 0 ? p.mu_constant : sutherland(t);
          if (z.mach) z.mach(i, j, k) = V / std::sqrt(gamma_air * R_u / mw_air * t);
          continue;
        }
        const int ns = p.n_spec;
        double cp[16], y[16], imw = 0, cpt = 0;
        nasa7_cp(t, p.mech, cp);
        for (int l = 0; l < ns; ++l) {
          y[l] = z.sv(i, j, k, l);
          imw += y[l] * p.mech.imw[l];
          cpt += y[l] * cp[l];
        }
        const double mw = 1 / std::max(imw, 1e-12);
        const double R = R_u * imw;
        if (p.i_eve >= 0) {
          // two-temperature (src/FieldOperation.cuh:207-226): gamma and c of the
          // translational-rotational mode, T_ve defaulted to T, kappa_ve = kappa cv_ve(T_ve) / cp
          double cv_tr, cp_tr, r_mix;
          tr_heat_capacities(p, t, y, cv_tr, cp_tr, r_mix);
          const double gam = cp_tr / std::max(cv_tr, 1e-8);
          z.gamma(i, j, k) = gam;
          const double a = std::sqrt(std::max(gam * r_mix * t, 1e-12));
          z.acoustic(i, j, k) = a;
          if (z.mach) z.mach(i, j, k) = V / a;
          if (z.tve(i, j, k) <= 0) z.tve(i, j, k) = t;
        } else {
          const double gam = cpt / (cpt - R);
          z.gamma(i, j, k) = gam;
          const double c = std::sqrt(gam * R * t);
          z.acoustic(i, j, k) = c;
          if (z.mach) z.mach(i, j, k) = V / c;
        }
        double mu, kap, rd[16];
        transport(t, mw, y, cp, p.mech, mu, kap, rd);
        z.mul(i, j, k) = mu;
        z.kappa(i, j, k) = kap;
        for (int l = 0; l < ns; ++l) z.rhoD(i, j, k, l) = rd[l];
        if (p.i_eve >= 0 && z.kappa_ve) {
          double cv_ve = 0;
          mixture_ve_energy(p, z.tve(i, j, k), y, &cv_ve);
          z.kappa_ve(i, j, k) = kap * cv_ve / std::max(cpt, 1e-8);
        }
      }
}

bool flag_at(const std::vector<int> &f, int a, int na, int b, int nb) {
  return a >= 0 && a < na && b >= 0 && b < nb && f[a + b * na] != 0;
}

// project_to_interior of apply_wall (src/BoundCond.cu:3070-3088)
void project_to_interior(const Zone &z, int &i, int &j, int &k) {
  if (i <= 0 && flag_at(z.il, j, z.my, k, z.mz)) i = 1;
  else if (i >= z.mx - 1 && flag_at(z.ir, j, z.my, k, z.mz)) i = z.mx - 2;
  if (j <= 0 && flag_at(z.jl, i, z.mx, k, z.mz)) j = 1;
  else if (j >= z.my - 1 && flag_at(z.jr, i, z.mx, k, z.mz)) j = z.my - 2;
  if (z.mz > 1) {
    if (k <= 0 && flag_at(z.kl, i, z.mx, j, z.my)) k = 1;
    else if (k >= z.mz - 1 && flag_at(z.kr, i, z.mx, j, z.my)) k = z.mz - 2;
  }
}

double mix_r(const Zone &z, const Param &p, int i, int j, int k) {
  if (p.n_spec == 0) return R_air;
  double R = 0;
  for (int l = 0; l < p.n_spec; ++l) R += z.sv(i, j, k, l) * p.mech.gas_const[l];
  return R;
}

// gamma = cp / (cp - R) of a node's mixture at its temperature (apply_outflow's back-pressure
// branch, src/BoundCond.cu:2232-2243)
double node_gamma(const Zone &z, const Param &p, int i, int j, int k) {
  if (p.n_spec == 0) return gamma_air;
  std::vector<double> cp(p.n_spec);
  nasa7_cp(z.bv(i, j, k, 5), p.mech, cp.data());  // compute_cp (NASA9 tables when loaded)
  double cpm = 0, r = 0;
  for (int l = 0; l < p.n_spec; ++l) {
    cpm += z.sv(i, j, k, l) * cp[l];
    r += z.sv(i, j, k, l) * p.mech.gas_const[l];
  }
  return cpm / (cpm - r);
}

// set_boundary_state (src/BoundCond.cu:55-76)
void set_boundary_state(Zone &z, const Param &p, int i, int j, int k, const double *st, const double *sv,
                        double tve) {
  for (int l = 0; l < 6; ++l) z.bv(i, j, k, l) = st[l];
  for (int l = 0; l < p.n_scalar; ++l) z.sv(i, j, k, l) = sv[l];
  if (p.i_eve >= 0) z.tve(i, j, k) = std::max(tve, 1.0);
  cv_point(z, p, i, j, k);
}

// apply_farfield (src/BoundCond.cu:2351-2482) at face node (i, j, k)
void farfield_point(Zone &z, const Param &p, const FaceBC &f, const int *dir, int i, int j, int k) {
  int in[3] = {i - dir[0], j - dir[1], k - dir[2]};
  project_to_interior(z, in[0], in[1], in[2]);
  double nx = z.metric(i, j, k, f.face * 3), ny = z.metric(i, j, k, f.face * 3 + 1),
         nz = z.metric(i, j, k, f.face * 3 + 2);
  const double gni = f.direction / std::sqrt(nx * nx + ny * ny + nz * nz);
  nx *= gni; ny *= gni; nz *= gni;
  const double rho_in = z.bv(in[0], in[1], in[2], 0), u_in = z.bv(in[0], in[1], in[2], 1),
               v_in = z.bv(in[0], in[1], in[2], 2), w_in = z.bv(in[0], in[1], in[2], 3),
               p_in = z.bv(in[0], in[1], in[2], 4), t_in = z.bv(in[0], in[1], in[2], 5);
  const double c_in = p.n_spec == 0 ? std::sqrt(std::max(gamma_air * R_air * t_in, 1e-12))
                                    : std::max(z.acoustic(in[0], in[1], in[2]), 1e-12);
  const double rho_c_in = std::max(rho_in * c_in, 1e-12);
  const double mn_in = (u_in * nx + v_in * ny + w_in * nz) / c_in;
  std::vector<double> sv_b(std::max(p.n_scalar, 1), 0.0);
  auto r_mix = [&]() {
    if (p.n_spec == 0) return R_air;
    double r = 0;
    for (int l = 0; l < p.n_spec; ++l) r += sv_b[l] * p.mech.gas_const[l];
    return std::max(r, 1e-12);
  };
  double rho_b = rho_in, u_b = u_in, v_b = v_in, w_b = w_in, p_b = p_in, t_b = t_in, tve_b = t_in;
  if (p.i_eve >= 0) tve_b = z.tve(in[0], in[1], in[2]) > 0.0 ? z.tve(in[0], in[1], in[2]) : t_in;
  if (mn_in < 0.0) {  // supersonic or subsonic inflow
    for (int l = 0; l < p.n_scalar; ++l) sv_b[l] = f.sv[l];
    if (mn_in <= -1.0) {
      rho_b = f.rho; u_b = f.u; v_b = f.v; w_b = f.w; p_b = f.p; t_b = f.T;
    } else {
      const double du_n = (f.u - u_in) * nx + (f.v - v_in) * ny + (f.w - w_in) * nz;
      p_b = std::max(0.5 * (p_in + f.p - rho_in * c_in * du_n), 0.1 * std::max(f.p, 1.0));
      rho_b = std::max(f.rho + (p_b - f.p) / (c_in * c_in), 0.1 * std::max(f.rho, 1e-12));
      u_b = f.u - (p_b - f.p) * nx / rho_c_in;
      v_b = f.v - (p_b - f.p) * ny / rho_c_in;
      w_b = f.w - (p_b - f.p) * nz / rho_c_in;
      t_b = p_b / std::max(rho_b * r_mix(), 1e-12);
    }
    if (p.i_eve >= 0) tve_b = f.wall_Tve > 0.0 ? f.wall_Tve : t_b;
  } else {  // subsonic or supersonic outflow
    for (int l = 0; l < p.n_scalar; ++l) sv_b[l] = z.sv(in[0], in[1], in[2], l);
    if (mn_in < 1.0) {
      p_b = f.p;
      const double dp = p_b - p_in;
      rho_b = std::max(rho_in + dp / (c_in * c_in), 0.1 * std::max(rho_in, 1e-12));
      u_b = u_in - dp * nx / rho_c_in;
      v_b = v_in - dp * ny / rho_c_in;
      w_b = w_in - dp * nz / rho_c_in;
      t_b = p_b / std::max(rho_b * r_mix(), 1e-12);
    }
  }
  const double st[6] = {rho_b, u_b, v_b, w_b, p_b, t_b};
  set_boundary_state(z, p, i, j, k, st, sv_b.data(), tve_b);
  for (int g = 1; g <= z.ngg; ++g) {
    int ii[3] = {i - g * dir[0], j - g * dir[1], k - g * dir[2]};
    project_to_interior(z, ii[0], ii[1], ii[2]);
    double sg[6] = {rho_b, u_b, v_b, w_b, p_b, t_b};
    if (mn_in > -1.0 && mn_in < 1.0) {
      sg[0] = std::max(2 * rho_b - z.bv(ii[0], ii[1], ii[2], 0), 0.1 * std::max(rho_b, 1e-12));
      sg[4] = std::max(2 * p_b - z.bv(ii[0], ii[1], ii[2], 4), 0.1 * std::max(p_b, 1.0));
      sg[1] = 2 * u_b - z.bv(ii[0], ii[1], ii[2], 1);
      sg[2] = 2 * v_b - z.bv(ii[0], ii[1], ii[2], 2);
      sg[3] = 2 * w_b - z.bv(ii[0], ii[1], ii[2], 3);
      sg[5] = sg[4] / std::max(sg[0] * r_mix(), 1e-12);
    }
    set_boundary_state(z, p, i + g * dir[0], j + g * dir[1], k + g * dir[2], sg, sv_b.data(), tve_b);
  }
}

// the back-pressure branch of apply_outflow (src/BoundCond.cu:2219-2320) at face node (i, j, k)
void back_pressure_point(Zone &z, const Param &p, const FaceBC &f, const int *dir, int i, int j, int k) {
  double nx = z.metric(i, j, k, f.face * 3), ny = z.metric(i, j, k, f.face * 3 + 1),
         nz = z.metric(i, j, k, f.face * 3 + 2);
  const double gni = f.direction / std::sqrt(nx * nx + ny * ny + nz * nz);
  nx *= gni; ny *= gni; nz *= gni;
  double u_b = z.bv(i, j, k, 1), v_b = z.bv(i, j, k, 2), w_b = z.bv(i, j, k, 3);
  const double u_face = nx * u_b + ny * v_b + nz * w_b;
  double p_b = z.bv(i, j, k, 4), rho_b = z.bv(i, j, k, 0);
  const double a_b = std::sqrt(node_gamma(z, p, i, j, k) * p_b / rho_b);
  if (std::fabs(u_face / a_b) < 1) {
    p_b = f.p;
    const int i1 = i - dir[0], j1 = j - dir[1], k1 = k - dir[2];
    const double d1 = z.bv(i1, j1, k1, 0), u1 = z.bv(i1, j1, k1, 1), v1 = z.bv(i1, j1, k1, 2),
                 w1 = z.bv(i1, j1, k1, 3), p1 = z.bv(i1, j1, k1, 4);
    const double c1 = std::sqrt(node_gamma(z, p, i1, j1, k1) * p1 / d1);
    const double temp = (p_b - p1) / c1;
    rho_b = d1 + temp / c1;
    u_b = u1 - nx * temp / d1;
    v_b = v1 - ny * temp / d1;
    w_b = w1 - nz * temp / d1;
    for (int g = 1; g <= z.ngg; ++g) {
      const int gi = i + g * dir[0], gj = j + g * dir[1], gk = k + g * dir[2];
      const int ii = i - g * dir[0], ij = j - g * dir[1], ik = k - g * dir[2];
      const double p_g = 2 * p_b - z.bv(ii, ij, ik, 4), rho_g = 2 * rho_b - z.bv(ii, ij, ik, 0);
      z.bv(gi, gj, gk, 0) = rho_g;
      z.bv(gi, gj, gk, 1) = 2 * u_b - z.bv(ii, ij, ik, 1);
      z.bv(gi, gj, gk, 2) = 2 * v_b - z.bv(ii, ij, ik, 2);
      z.bv(gi, gj, gk, 3) = 2 * w_b - z.bv(ii, ij, ik, 3);
      z.bv(gi, gj, gk, 4) = p_g;
      for (int l = 0; l < p.n_scalar; ++l) z.sv(gi, gj, gk, l) = 2 * z.sv(i, j, k, l) - z.sv(ii, ij, ik, l);
      z.bv(gi, gj, gk, 5) = p_g / (rho_g * mix_r(z, p, gi, gj, gk));
      if (p.i_eve >= 0) {
        const double tve_b = z.tve(i, j, k) > 0.0 ? z.tve(i, j, k) : z.bv(i, j, k, 5);
        const double tve_i = z.tve(ii, ij, ik) > 0.0 ? z.tve(ii, ij, ik) : z.bv(ii, ij, ik, 5);
        z.tve(gi, gj, gk) = std::max(2 * tve_b - tve_i, 1.0);
      }
      cv_point(z, p, gi, gj, gk);
    }
  } else {
    for (int g = 1; g <= z.ngg; ++g) {
      const int gi = i + g * dir[0], gj = j + g * dir[1], gk = k + g * dir[2];
      const double st[6] = {rho_b, u_b, v_b, w_b, p_b, z.bv(i, j, k, 5)};
      for (int l = 0; l < 6; ++l) z.bv(gi, gj, gk, l) = st[l];
      for (int l = 0; l < p.n_scalar; ++l) z.sv(gi, gj, gk, l) = z.sv(i, j, k, l);
      if (p.i_eve >= 0) z.tve(gi, gj, gk) = z.tve(i, j, k) > 0.0 ? z.tve(i, j, k) : z.bv(i, j, k, 5);
      cv_point(z, p, gi, gj, gk);
    }
  }
}

// apply_boundary_conditions (src/BoundCond.cu:3846-3998) in its priority order
// apply_outflow_nr_conserv (src/BoundCond.cu:3580-3817), run by nonReflectingBoundary
// (:3818-3845) over the outflow faces flagged nonReflecting, after the inviscid flux
// (src/RK.cuh:190-193).  Restricted to the face's own nodes: the reference's launch also covers
// the tangential ghost nodes of an extended face (viscous_order 2), whose dq writes fall on
// other nodes of the ghost-free dq array.
void outflow_nonreflecting(Zone &z, const Param &p) {
  const int ext[3] = {z.mx, z.my, z.mz};
  for (const FaceBC &f : z.faces) {
    if (!f.nonreflecting) continue;
    int lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
      lo[a] = f.start[a]; hi[a] = f.end[a];
      if (a == f.face) continue;
      lo[a] = std::max(lo[a], 0); hi[a] = std::min(hi[a], ext[a] - 1);
    }
    const int face = f.face;
    const double cc[3] = {-1.5, 2, -0.5};
    const bool start_face = f.direction == -1;
    const int sgn = start_face ? 1 : -1;
    for (int k = lo[2]; k <= hi[2]; ++k)
      for (int j = lo[1]; j <= hi[1]; ++j)
        for (int i = lo[0]; i <= hi[0]; ++i) {
          double dR = 0, dRU = 0, dRV = 0, dRW = 0, dRE = 0;
          std::vector<double> dRY(std::max(p.n_scalar, 1), 0.0);
          for (int l = 0; l <= 2; ++l) {
            const double c = sgn * cc[l];
            const int ii = i + (face == 0 ? sgn * l : 0), jj = j + (face == 1 ? sgn * l : 0),
                      kk = k + (face == 2 ? sgn * l : 0);
            dR += c * z.cv(ii, jj, kk, 0);
            dRU += c * z.cv(ii, jj, kk, 1);
            dRV += c * z.cv(ii, jj, kk, 2);
            dRW += c * z.cv(ii, jj, kk, 3);
            dRE += c * z.cv(ii, jj, kk, 4);
            for (int ls = 0; ls < p.n_scalar; ++ls) dRY[ls] += c * z.cv(ii, jj, kk, 5 + ls);
          }
          const double r = z.bv(i, j, k, 0), u = z.bv(i, j, k, 1), v = z.bv(i, j, k, 2), w = z.bv(i, j, k, 3),
                       pr = z.bv(i, j, k, 4);
          double kx = z.metric(i, j, k, face * 3), ky = z.metric(i, j, k, face * 3 + 1),
                 kz = z.metric(i, j, k, face * 3 + 2);
          const double gki = 1 / std::sqrt(kx * kx + ky * ky + kz * kz);
          kx *= gki; ky *= gki; kz *= gki;
          const double Uk = u * kx + v * ky + w * kz;
          double gam = gamma_air;
          const double T = z.bv(i, j, k, 5);
          std::vector<double> h(std::max(p.n_spec, 1)), cp(std::max(p.n_spec, 1));
          if (p.n_spec > 0) {
            nasa7_h_cp(T, p.mech, h.data(), cp.data());
            double cpm = 0, cvm = 0;
            for (int l = 0; l < p.n_spec; ++l) {
              cpm += z.sv(i, j, k, l) * cp[l];
              cvm += z.sv(i, j, k, l) * (cp[l] - p.mech.gas_const[l]);
            }
            gam = cpm / cvm;
          }
          const double c2 = gam * pr / r, c = std::sqrt(c2), ic2 = 1 / c2, cgk = c / gki;
          double lam[3] = {Uk - cgk, Uk, Uk + cgk};
          for (double &x : lam) x = start_face ? std::min(x, 0.0) : std::max(x, 0.0);
          const double ek = 0.5 * (u * u + v * v + w * w), gm1 = gam - 1, alpha = gm1 * ek;
          double aY = 0;
          std::vector<double> al(std::max(p.n_spec, 1), 0.0);
          for (int l = 0; l < p.n_spec; ++l) {
            al[l] = gam * p.mech.gas_const[l] * T - gm1 * h[l];
            aY += al[l] * dRY[l];
          }
          double L[5];
          L[0] = lam[0] * 0.5 * ic2 *
                 ((alpha + Uk * c) * dR - (gm1 * u + kx * c) * dRU - (gm1 * v + ky * c) * dRV -
                  (gm1 * w + kz * c) * dRW + gm1 * dRE + aY);
          double tk = gm1 * kx;
          L[1] = lam[1] * ic2 *
                 ((kx * (c2 - alpha) - c * (kz * v - ky * w)) * dR + (tk * u) * dRU + (tk * v + kz * c) * dRV +
                  (tk * w - ky * c) * dRW - tk * dRE - kx * aY);
          tk = gm1 * ky;
          L[2] = lam[1] * ic2 *
                 ((ky * (c2 - alpha) - c * (kx * w - kz * u)) * dR + (tk * u - kz * c) * dRU + (tk * v) * dRV +
                  (tk * w + kx * c) * dRW - tk * dRE - ky * aY);
          tk = gm1 * kz;
          L[3] = lam[1] * ic2 *
                 ((kz * (c2 - alpha) - c * (ky * u - kx * v)) * dR + (tk * u + ky * c) * dRU +
                  (tk * v - kx * c) * dRV + (tk * w) * dRW - tk * dRE - kz * aY);
          L[4] = lam[2] * 0.5 * ic2 *
                 ((alpha - Uk * c) * dR - (gm1 * u - kx * c) * dRU - (gm1 * v - ky * c) * dRV -
                  (gm1 * w - kz * c) * dRW + gm1 * dRE + aY);
          const double hh = (z.cv(i, j, k, 4) + pr) / r, igm1 = 1 / gm1;
          const double sum = L[0] + kx * L[1] + ky * L[2] + kz * L[3] + L[4];
          double d[5];
          d[0] = sum;
          d[1] = u * sum + c * (kx * (L[4] - L[0]) - kz * L[2] + ky * L[3]);
          d[2] = v * sum + c * (ky * (L[4] - L[0]) + kz * L[1] - kx * L[3]);
          d[3] = w * sum + c * (kz * (L[4] - L[0]) - ky * L[1] + kx * L[2]);
          d[4] = hh * sum + c * (Uk * (L[4] - L[0]) + (kz * v - ky * w - kx * c * igm1) * L[1] +
                                 (kx * w - kz * u - ky * c * igm1) * L[2] + (ky * u - kx * v - kz * c * igm1) * L[3]);
          const double mj = -z.jac(i, j, k);
          double add = 0;
          for (int l = 0; l < p.n_spec; ++l) {
            const double Ls = lam[1] * (dRY[l] - z.sv(i, j, k, l) * dR);
            z.dq(i, j, k, 5 + l) += mj * (Ls + z.sv(i, j, k, l) * sum);
            add += al[l] * Ls;
          }
          d[4] -= add * igm1;
          for (int l = 0; l < 5; ++l) z.dq(i, j, k, l) += mj * d[l];
        }
  }
}

void apply_boundary_conditions(Zone &z, const Param &p) {
  for (int type : {CB2_BC_FARFIELD, CB2_BC_OUTFLOW, CB2_BC_INFLOW, CB2_BC_SYMMETRY, CB2_BC_WALL, CB2_BC_PERIODIC}) {
    for (const auto &f : z.faces) {
      if (f.type != type) continue;
      int dir[3] = {0, 0, 0};
      dir[f.face] = f.direction;
      for (int k = f.start[2]; k <= f.end[2]; ++k)
        for (int j = f.start[1]; j <= f.end[1]; ++j)
          for (int i = f.start[0]; i <= f.end[0]; ++i) {
            if (type == CB2_BC_FARFIELD) {
              farfield_point(z, p, f, dir, i, j, k);
            } else if (type == CB2_BC_OUTFLOW && f.p > 0) {
              back_pressure_point(z, p, f, dir, i, j, k);
            } else if (type == CB2_BC_OUTFLOW) {  // src/BoundCond.cu:2328-2347
              for (int g = 1; g <= z.ngg; ++g) {
                const int gi = i + g * dir[0], gj = j + g * dir[1], gk = k + g * dir[2];
                for (int l = 0; l < 6; ++l) z.bv(gi, gj, gk, l) = z.bv(i, j, k, l);
                for (int l = 0; l < p.n_scalar; ++l) z.sv(gi, gj, gk, l) = z.sv(i, j, k, l);
                // two-temperature ghost T_ve, the starting guess of its inversion (:2339-2345)
                if (p.i_eve >= 0) z.tve(gi, gj, gk) = z.tve(i, j, k) > 0.0 ? z.tve(i, j, k) : z.bv(i, j, k, 5);
                cv_point(z, p, gi, gj, gk);
              }
            } else if (type == CB2_BC_INFLOW) {  // constant supersonic state
              for (int g = 0; g <= z.ngg; ++g) {
                const int gi = i + g * dir[0], gj = j + g * dir[1], gk = k + g * dir[2];
                const double st[6] = {f.rho, f.u, f.v, f.w, f.p, f.T};
                for (int l = 0; l < 6; ++l) z.bv(gi, gj, gk, l) = st[l];
                for (int l = 0; l < p.n_scalar; ++l) z.sv(gi, gj, gk, l) = l < (int)f.sv.size() ? f.sv[l] : 0.0;
                cv_point(z, p, gi, gj, gk);
              }
            } else if (type == CB2_BC_SYMMETRY) {  // src/BoundCond.cu:2130-2202
              const int in[3] = {i - dir[0], j - dir[1], k - dir[2]};
              double kx = z.metric(i, j, k, f.face * 3), ky = z.metric(i, j, k, f.face * 3 + 1),
                     kz = z.metric(i, j, k, f.face * 3 + 2);
              const double km = std::sqrt(kx * kx + ky * ky + kz * kz);
              kx /= km; ky /= km; kz /= km;
              const double u1 = z.bv(in[0], in[1], in[2], 1), v1 = z.bv(in[0], in[1], in[2], 2),
                           w1 = z.bv(in[0], in[1], in[2], 3);
              double uk = kx * u1 + ky * v1 + kz * w1;
              z.bv(i, j, k, 1) = u1 - kx * uk;
              z.bv(i, j, k, 2) = v1 - ky * uk;
              z.bv(i, j, k, 3) = w1 - kz * uk;
              z.bv(i, j, k, 0) = z.bv(in[0], in[1], in[2], 0);
              z.bv(i, j, k, 4) = z.bv(in[0], in[1], in[2], 4);
              z.bv(i, j, k, 5) = z.bv(in[0], in[1], in[2], 5);
              for (int l = 0; l < p.n_scalar; ++l) z.sv(i, j, k, l) = z.sv(in[0], in[1], in[2], l);
              if (p.i_eve >= 0) z.tve(i, j, k) = z.tve(in[0], in[1], in[2]);
              cv_point(z, p, i, j, k);
              for (int g = 1; g <= z.ngg; ++g) {
                const int gi = i + g * dir[0], gj = j + g * dir[1], gk = k + g * dir[2];
                const int ii = i - g * dir[0], ij = j - g * dir[1], ik = k - g * dir[2];
                if (p.i_eve >= 0) z.tve(gi, gj, gk) = z.tve(ii, ij, ik);
                z.bv(gi, gj, gk, 0) = z.bv(ii, ij, ik, 0);
                const double u = z.bv(ii, ij, ik, 1), v = z.bv(ii, ij, ik, 2), w = z.bv(ii, ij, ik, 3);
                uk = kx * u + ky * v + kz * w;
                z.bv(gi, gj, gk, 1) = u - 2 * uk * kx;
                z.bv(gi, gj, gk, 2) = v - 2 * uk * ky;
                z.bv(gi, gj, gk, 3) = w - 2 * uk * kz;
                z.bv(gi, gj, gk, 4) = z.bv(ii, ij, ik, 4);
                z.bv(gi, gj, gk, 5) = z.bv(ii, ij, ik, 5);
                for (int l = 0; l < p.n_scalar; ++l) z.sv(gi, gj, gk, l) = z.sv(ii, ij, ik, l);
                cv_point(z, p, gi, gj, gk);
              }
            } else if (type == CB2_BC_WALL) {  // src/BoundCond.cu:3055-3389
              // a fully catalytic wall (catalytic_type 1) sets the face node and its ghosts to the
              // wall's mass fractions (Wall::yk, :3197-3203 and :3344-3357)
              const bool cat = p.n_spec > 0 && !f.sv.empty();
              int idx[3] = {i - dir[0], j - dir[1], k - dir[2]};
              project_to_interior(z, idx[0], idx[1], idx[2]);
              const bool iso = f.wall_T > 0;
              const bool tt = p.i_eve >= 0;
              const double t_wall = iso ? f.wall_T : z.bv(idx[0], idx[1], idx[2], 5);
              double tve_wall = t_wall;
              if (tt) {  // the wall's T_ve (src/BoundCond.cu:3157-3167)
                const double tve_in = z.tve(idx[0], idx[1], idx[2]) > 0.0 ? z.tve(idx[0], idx[1], idx[2])
                                                                         : z.bv(idx[0], idx[1], idx[2], 5);
                tve_wall = !iso ? tve_in : (f.wall_Tve > 0.0 ? f.wall_Tve : t_wall);
              }
              const double pw = z.bv(idx[0], idx[1], idx[2], 4);
              for (int l = 0; l < p.n_spec; ++l) z.sv(i, j, k, l) = cat ? f.sv[l] : z.sv(idx[0], idx[1], idx[2], l);
              double R = mix_r(z, p, i, j, k);
              z.bv(i, j, k, 0) = pw / (t_wall * R);
              // the wall's velocity: at rest, or blowing (if_blow_shock_wave, :3226-3245)
              double wall_u[3] = {0, 0, 0};
              if (f.blow && p.step >= f.blow_start && p.step <= f.blow_end) {
                double n[3] = {z.metric(i, j, k, f.face * 3), z.metric(i, j, k, f.face * 3 + 1),
                               z.metric(i, j, k, f.face * 3 + 2)};
                const double ninv = f.direction / std::max(std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]), 1e-30);
                for (double &c : n) c *= ninv;
                const double vn_local = n[0] * z.bv(idx[0], idx[1], idx[2], 1) + n[1] * z.bv(idx[0], idx[1], idx[2], 2) +
                                        n[2] * z.bv(idx[0], idx[1], idx[2], 3);
                const double vn_inf = n[0] * f.u + n[1] * f.v + n[2] * f.w;  // the freestream (ux_inf, ...)
                const double seed = p.step <= 50 ? std::max(vn_inf, 0.0) : 0.0;
                const double blow = std::max(f.blow_coef, 0.0) * std::max(std::max(vn_local, 0.0), seed);
                for (int c = 0; c < 3; ++c) wall_u[c] = -blow * n[c];
              }
              for (int c = 0; c < 3; ++c) z.bv(i, j, k, 1 + c) = wall_u[c];
              z.bv(i, j, k, 4) = pw;
              z.bv(i, j, k, 5) = t_wall;
              if (tt) {
                double y[16];
                for (int l = 0; l < p.n_spec; ++l) y[l] = z.sv(i, j, k, l);
                z.tve(i, j, k) = tve_wall;
                z.sv(i, j, k, p.i_eve) = mixture_ve_energy(p, tve_wall, y, nullptr);
              }
              cv_point(z, p, i, j, k);
              for (int g = 1; g <= z.ngg; ++g) {
                int in[3] = {i - g * dir[0], j - g * dir[1], k - g * dir[2]};
                project_to_interior(z, in[0], in[1], in[2]);
                const int gh[3] = {i + g * dir[0], j + g * dir[1], k + g * dir[2]};
                const double p_i = z.bv(in[0], in[1], in[2], 4), t_i = z.bv(in[0], in[1], in[2], 5);
                double t_g = t_i;
                if (iso) {
                  t_g = 2 * t_wall - t_i;
                  if (t_g <= 0.1 * t_wall) t_g = tt ? 0.1 * t_wall : t_wall;
                }
                double tve_g = t_g;
                if (tt) {  // src/BoundCond.cu:3319-3330
                  const double tve_i = z.tve(in[0], in[1], in[2]) > 0.0 ? z.tve(in[0], in[1], in[2]) : t_i;
                  tve_g = tve_i;
                  if (iso) {
                    tve_g = 2 * tve_wall - tve_i;
                    const double floor_ve = 0.1 * std::max(tve_wall, 1.0);
                    if (tve_g <= floor_ve) tve_g = floor_ve;
                  }
                }
                for (int l = 0; l < p.n_spec; ++l)
                  z.sv(gh[0], gh[1], gh[2], l) = cat ? f.sv[l] : z.sv(in[0], in[1], in[2], l);
                R = cat ? mix_r(z, p, i, j, k) : mix_r(z, p, in[0], in[1], in[2]);
                z.bv(gh[0], gh[1], gh[2], 0) = p_i / (t_g * R);
                for (int c = 1; c <= 3; ++c) z.bv(gh[0], gh[1], gh[2], c) = 2 * wall_u[c - 1] - z.bv(in[0], in[1], in[2], c);
                z.bv(gh[0], gh[1], gh[2], 4) = p_i;
                z.bv(gh[0], gh[1], gh[2], 5) = t_g;
                if (tt) {
                  double y[16];
                  for (int l = 0; l < p.n_spec; ++l) y[l] = z.sv(gh[0], gh[1], gh[2], l);
                  z.tve(gh[0], gh[1], gh[2]) = tve_g;
                  z.sv(gh[0], gh[1], gh[2], p.i_eve) = mixture_ve_energy(p, tve_g, y, nullptr);
                }
                cv_point(z, p, gh[0], gh[1], gh[2]);
              }
            } else {  // periodic, src/BoundCond.cu:3390-3440
              int o[3] = {i, j, k};
              const int ext[3] = {z.mx, z.my, z.mz};
              o[f.face] = f.direction < 0 ? ext[f.face] - 1 : 0;
              for (int l = 0; l < 6; ++l) {
                const double ave = 0.5 * (z.bv(i, j, k, l) + z.bv(o[0], o[1], o[2], l));
                z.bv(i, j, k, l) = ave;
                z.bv(o[0], o[1], o[2], l) = ave;
              }
              for (int l = 0; l < p.n_scalar; ++l) {
                const double ave = 0.5 * (z.sv(i, j, k, l) + z.sv(o[0], o[1], o[2], l));
                z.sv(i, j, k, l) = ave;
                z.sv(o[0], o[1], o[2], l) = ave;
              }
              cv_point(z, p, i, j, k);
              for (int g = 1; g <= z.ngg; ++g) {
                const int gi = i + g * dir[0], gj = j + g * dir[1], gk = k + g * dir[2];
                const int ii = o[0] + g * dir[0], ij = o[1] + g * dir[1], ik = o[2] + g * dir[2];
                for (int l = 0; l < 6; ++l) z.bv(gi, gj, gk, l) = z.bv(ii, ij, ik, l);
                for (int l = 0; l < p.n_scalar; ++l) z.sv(gi, gj, gk, l) = z.sv(ii, ij, ik, l);
                cv_point(z, p, gi, gj, gk);
              }
            }
          }
    }
  }
  if (p.dim == 2 && z.mz == 1) {  // eliminate_k_gradient (src/FieldOperation.cu:96-121)
    const int g = z.ngg;
    for (int j = -g; j < z.my + g; ++j)
      for (int i = -g; i < z.mx + g; ++i)
        for (int k = 1; k <= g; ++k) {
          for (int l = 0; l < 6; ++l) z.bv(i, j, k, l) = z.bv(i, j, -k, l) = z.bv(i, j, 0, l);
          for (int l = 0; l < p.n_scalar; ++l) z.sv(i, j, k, l) = z.sv(i, j, -k, l) = z.sv(i, j, 0, l);
          for (int l = 0; l < p.n_var; ++l) z.cv(i, j, k, l) = z.cv(i, j, -k, l) = z.cv(i, j, 0, l);
        }
  }
}

// local_time_step (src/TimeAdvanceFunc.cuh:28-127) + min_of_arr (src/TimeAdvanceFunc.cu:145-164)
double local_time_step_min(Zone &z, const Param &p) {
  double dt_min = 1e+6;
  const int dim = z.mz == 1 ? 2 : 3;
#pragma omp parallel for collapse(2) reduction(min : dt_min) schedule(static)
  for (int k = 0; k < z.mz; ++k)
    for (int j = 0; j < z.my; ++j)
      for (int i = 0; i < z.mx; ++i) {
        const Arr &M = z.metric;
        const double gxi = std::sqrt(sqr(M(i, j, k, 0)) + sqr(M(i, j, k, 1)) + sqr(M(i, j, k, 2)));
        const double geta = std::sqrt(sqr(M(i, j, k, 3)) + sqr(M(i, j, k, 4)) + sqr(M(i, j, k, 5)));
        const double gzeta = std::sqrt(sqr(M(i, j, k, 6)) + sqr(M(i, j, k, 7)) + sqr(M(i, j, k, 8)));
        const double u = z.bv(i, j, k, 1), v = z.bv(i, j, k, 2), w = z.bv(i, j, k, 3);
        const double U = u * M(i, j, k, 0) + v * M(i, j, k, 1) + w * M(i, j, k, 2);
        const double V = u * M(i, j, k, 3) + v * M(i, j, k, 4) + w * M(i, j, k, 5);
        const double W = u * M(i, j, k, 6) + v * M(i, j, k, 7) + w * M(i, j, k, 8);
        const double a = p.n_spec == 0 ? std::sqrt(gamma_air * R_air * z.bv(i, j, k, 5)) : z.acoustic(i, j, k);
        double lam = std::max(std::fabs(U) + a * gxi, std::fabs(V) + a * geta);
        if (dim == 3) lam = std::max(lam, std::fabs(W) + a * gzeta);
        if (p.viscous_order > 0) {
          double len = std::max(gxi, geta);
          if (dim == 3) len = std::max(len, gzeta);
          const double irho = 1.0 / z.bv(i, j, k, 0);
          double dv;
          if (p.n_spec == 0) {
            dv = std::max(gamma_air, 4.0 / 3.0) * irho;
            dv *= z.mul(i, j, k) / p.Pr;
          } else {
            double cpl[16], cp = 0, mrd = 0;
            nasa7_cp(z.bv(i, j, k, 5), p.mech, cpl);
            for (int l = 0; l < p.n_spec; ++l) {
              cp += cpl[l] * z.sv(i, j, k, l);
              mrd = std::max(mrd, z.rhoD(i, j, k, l));
            }
            dv = z.mul(i, j, k) * irho;
            dv = std::max(dv, z.kappa(i, j, k) * irho * z.gamma(i, j, k) / cp);
            dv = std::max(dv, mrd * irho);
            if (p.i_eve >= 0 && z.kappa_ve) {
              // two-temperature e_ve conduction (src/TimeAdvanceFunc.cuh:95-106)
              const double tve = z.tve(i, j, k) > 0.0 ? z.tve(i, j, k) : std::max(z.bv(i, j, k, 5), 1.0);
              double y[16], cv_ve = 0;
              for (int l = 0; l < p.n_spec; ++l) y[l] = z.sv(i, j, k, l);
              mixture_ve_energy(p, tve, y, &cv_ve);
              dv = std::max(dv, z.kappa_ve(i, j, k) * irho / std::max(cv_ve, 1e-8));
            }
          }
          lam = std::max(lam, len * len * dv);
        }
        double dt = p.cfl / lam;
        if (p.n_spec > 0 && p.n_reac > 0 && z.rts) {
          const double rdt = p.cfl * z.rts(i, j, k);
          if (rdt > 1e-20 && rdt < 1e-5) dt = std::min(dt, rdt);
        }
        if (z.dtl) z.dtl(i, j, k) = dt;
        dt_min = std::min(dt_min, dt);
      }
  return dt_min;
}

// compute_shock_sensor (src/FieldOperation.cu:123-228) on interior nodes
void compute_shock_sensor(Zone &z, const Param &p) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < z.mz; ++k)
    for (int j = 0; j < z.my; ++j)
      for (int i = 0; i < z.mx; ++i) {
        const Arr &bv = z.bv;
        double sensor = 1;
        if (p.shock_sensor == 1) {
          const double twoP = bv(i, j, k, 4) * 2;
          const double pI = bv(i + 1, j, k, 4) + bv(i - 1, j, k, 4);
          const double pJ = bv(i, j + 1, k, 4) + bv(i, j - 1, k, 4);
          const double pK = bv(i, j, k + 1, 4) + bv(i, j, k - 1, 4);
          sensor = std::fabs(pI - twoP) / (pI + twoP) + std::fabs(pJ - twoP) / (pJ + twoP) +
                   std::fabs(pK - twoP) / (pK + twoP);
        } else if (p.shock_sensor == 2) {
          const double rho = bv(i, j, k, 0), rhoI = 1.0 / rho, pr = bv(i, j, k, 4), pI = 1.0 / pr;
          double s = 0;
          s = std::max(s, std::fabs(bv(i + 1, j, k, 0) - rho) * rhoI);
          s = std::max(s, std::fabs(bv(i, j + 1, k, 0) - rho) * rhoI);
          s = std::max(s, std::fabs(bv(i, j, k + 1, 0) - rho) * rhoI);
          s = std::max(s, std::fabs(bv(i + 1, j, k, 4) - pr) * pI);
          s = std::max(s, std::fabs(bv(i, j + 1, k, 4) - pr) * pI);
          s = std::max(s, std::fabs(bv(i, j, k + 1, 4) - pr) * pI);
          sensor = s;
        } else {
          const double c12 = 1.0 / 12.0, c23 = 2.0 / 3.0;
          double d[3][3];
          for (int c = 0; c < 3; ++c) {
            d[c][0] = c12 * bv(i - 2, j, k, 1 + c) - c23 * bv(i - 1, j, k, 1 + c) + c23 * bv(i + 1, j, k, 1 + c) -
                      c12 * bv(i + 2, j, k, 1 + c);
            d[c][1] = c12 * bv(i, j - 2, k, 1 + c) - c23 * bv(i, j - 1, k, 1 + c) + c23 * bv(i, j + 1, k, 1 + c) -
                      c12 * bv(i, j + 2, k, 1 + c);
            d[c][2] = c12 * bv(i, j, k - 2, 1 + c) - c23 * bv(i, j, k - 1, 1 + c) + c23 * bv(i, j, k + 1, 1 + c) -
                      c12 * bv(i, j, k + 2, 1 + c);
          }
          auto cart = [&](int c, int x) {
            return d[c][0] * z.metric(i, j, k, x) + d[c][1] * z.metric(i, j, k, 3 + x) +
                   d[c][2] * z.metric(i, j, k, 6 + x);
          };
          double div = cart(0, 0) + cart(1, 1) + cart(2, 2);
          if (div > 0) sensor = 0;
          else {
            const double duDy = cart(0, 1), duDz = cart(0, 2), dvDx = cart(1, 0), dvDz = cart(1, 2);
            const double dwDx = cart(2, 0), dwDy = cart(2, 1);
            div *= div;
            const double curl2 =
                (dwDy - dvDz) * (dwDy - dvDz) + (duDz - dwDx) * (duDz - dwDx) + (dvDx - duDy) * (dvDx - duDy);
            sensor = div / (div + curl2 + p.sensor_eps);
          }
        }
        z.shock(i, j, k) = sensor;
      }
}

// One SSP-RK3 step over all zones (src/RK.cuh:107-237, single process, no MPI)
// inner_communication over every inner face of every zone (src/DataCommunication.cu:6-124),
// then eliminate_k_gradient for 2-D zones (src/RK.cuh:218-226).
void inner_exchange(std::vector<Zone> &zones, const Param &p) {
  for (auto &z : zones) {
    for (const auto &f : z.inner) {
      Zone &t = zones[f.target_block];
      const int face_layer = f.direction > 0 ? f.range_start[f.face] : f.range_end[f.face];
      for (int n2 = 0; n2 < f.n_point[2]; ++n2)
        for (int n1 = 0; n1 < f.n_point[1]; ++n1)
          for (int n0 = 0; n0 < f.n_point[0]; ++n0) {
            const int n[3] = {n0, n1, n2};
            int idx[3], it[3], d[3];
            for (int a = 0; a < 3; ++a) {
              d[a] = f.loop_dir[a] * n[a];
              idx[a] = f.range_start[a] + d[a];
            }
            for (int a = 0; a < 3; ++a) it[a] = f.target_start[a] + f.target_loop_dir[a] * d[f.src_tar[a]];
            if (idx[f.face] == face_layer) {
              const double u_this = std::sqrt(sqr(z.bv(idx[0], idx[1], idx[2], 1)) + sqr(z.bv(idx[0], idx[1], idx[2], 2)) +
                                              sqr(z.bv(idx[0], idx[1], idx[2], 3)));
              if (std::fabs(u_this) > 1e-15) {
                const double u_that = std::sqrt(sqr(t.bv(it[0], it[1], it[2], 1)) + sqr(t.bv(it[0], it[1], it[2], 2)) +
                                                sqr(t.bv(it[0], it[1], it[2], 3)));
                if (std::fabs(u_that) < 1e-15) {
                  for (int l = 0; l < 6; ++l) z.bv(idx[0], idx[1], idx[2], l) = t.bv(it[0], it[1], it[2], l);
                  for (int l = 0; l < p.n_scalar; ++l) z.sv(idx[0], idx[1], idx[2], l) = t.sv(it[0], it[1], it[2], l);
                  if (p.i_eve >= 0) z.tve(idx[0], idx[1], idx[2]) = t.tve(it[0], it[1], it[2]);
                } else {
                  for (int l = 0; l < 6; ++l) {
                    const double ave = 0.5 * (t.bv(it[0], it[1], it[2], l) + z.bv(idx[0], idx[1], idx[2], l));
                    z.bv(idx[0], idx[1], idx[2], l) = ave;
                    t.bv(it[0], it[1], it[2], l) = ave;
                  }
                  for (int l = 0; l < p.n_scalar; ++l) {
                    const double ave = 0.5 * (t.sv(it[0], it[1], it[2], l) + z.sv(idx[0], idx[1], idx[2], l));
                    z.sv(idx[0], idx[1], idx[2], l) = ave;
                    t.sv(it[0], it[1], it[2], l) = ave;
                  }
                  if (p.i_eve >= 0) {
                    const double ave = 0.5 * (t.tve(it[0], it[1], it[2]) + z.tve(idx[0], idx[1], idx[2]));
                    z.tve(idx[0], idx[1], idx[2]) = ave;
                    t.tve(it[0], it[1], it[2]) = ave;
                  }
                  cv_point(t, p, it[0], it[1], it[2]);
                }
              }
            } else {
              for (int l = 0; l < 6; ++l) z.bv(idx[0], idx[1], idx[2], l) = t.bv(it[0], it[1], it[2], l);
              for (int l = 0; l < p.n_scalar; ++l) z.sv(idx[0], idx[1], idx[2], l) = t.sv(it[0], it[1], it[2], l);
              if (p.i_eve >= 0) z.tve(idx[0], idx[1], idx[2]) = t.tve(it[0], it[1], it[2]);
            }
            cv_point(z, p, idx[0], idx[1], idx[2]);
          }
    }
  }
  for (auto &z : zones) {
    if (z.inner.empty() || !(p.dim == 2 && z.mz == 1)) continue;
    const int g = z.ngg;
    for (int j = -g; j < z.my + g; ++j)
      for (int i = -g; i < z.mx + g; ++i)
        for (int k = 1; k <= g; ++k) {
          for (int l = 0; l < 6; ++l) z.bv(i, j, k, l) = z.bv(i, j, -k, l) = z.bv(i, j, 0, l);
          for (int l = 0; l < p.n_scalar; ++l) z.sv(i, j, k, l) = z.sv(i, j, -k, l) = z.sv(i, j, 0, l);
          for (int l = 0; l < p.n_var; ++l) z.cv(i, j, k, l) = z.cv(i, j, -k, l) = z.cv(i, j, 0, l);
        }
  }
}

void rk3_step(std::vector<Zone> &zones, const Param &p_in, double &dt, bool fixed_dt) {
  Param p = p_in;
  g_step = ++p.step;  // the step this call takes, counted before its stages (src/RK.cuh:108)
  for (auto &z : zones) {
    const size_t n = (size_t)z.cv.sz * p.n_var;
    std::memcpy(z.qn.p, z.cv.p, n * sizeof(double));
  }
  if (p.sensor_threshold > 1e-10)
    for (auto &z : zones) compute_shock_sensor(z, p);
  if (!fixed_dt) {
    double m = 1e+6;
    for (auto &z : zones) m = std::min(m, local_time_step_min(z, p));
    dt = m;
  }
  p.dt = dt;
  for (int rk = 0; rk < 3; ++rk) {
    viscous_all(zones, p);
    for (auto &z : zones) {
      if (p.reaction) finite_rate_chemistry(z, p);
      compute_inviscid_flux(z, p);
      outflow_nonreflecting(z, p);
      update_cv_and_bv_rk(z, p, dt, rk);
      apply_boundary_conditions(z, p);
    }
    inner_exchange(zones, p);
    for (auto &z : zones) update_physical_properties(z, p);
  }
}

}  // namespace oracle
