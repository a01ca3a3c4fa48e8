// FP64 host oracle of the two-temperature (vibrational-electronic) terms of COREFL's stage
// update: species and mixture e_ve, the T_ve and T inversions, and the Landau-Teller VT
// relaxation step with Millikan-White + Park relaxation times.
//
// TEST INFRASTRUCTURE ONLY (see oracle.hpp).  Each function restates the reference's DEVICE
// routine it cites (the library must match those), in the same arithmetic order; the golden
// fixture tests/golden/h2_two_temperature.json holds the reference's host twins of the same
// formulas (src/ChemData.cpp:236-322, src/ConstVolumeReactor.cpp:805-998) evaluated on seeded
// states.
#include <cmath>
#include "oracle.hpp"

namespace oracle {

namespace {
constexpr double avogadro = 6.02214076e26;  // src/Constants.h:11

double vib_energy(const Param &p, int i, double t) {
  // compute_vib_energy (src/Thermo.cu:656-668)
  if (!p.tt.on || i < 0 || i >= p.n_spec) return 0.0;
  const double temp = std::max(t, 1.0);
  const double r = p.mech.gas_const[i];
  double e = 0.0;
  if (p.tt.theta_v[i] > 0) {
    const double x = p.tt.theta_v[i] / temp;
    if (x < 200) e += r * p.tt.theta_v[i] / std::expm1(x);
  }
  return e;
}

double vib_cv(const Param &p, int i, double t) {
  // compute_vib_cv (src/Thermo.cu:695-709)
  if (!p.tt.on || i < 0 || i >= p.n_spec) return 0.0;
  const double temp = std::max(t, 1.0);
  const double r = p.mech.gas_const[i];
  double c = 0.0;
  if (p.tt.theta_v[i] > 0) {
    const double x = p.tt.theta_v[i] / temp;
    if (x < 200) {
      const double ex = std::exp(x);
      const double d = ex - 1.0;
      c += r * x * x * ex / (d * d);
    }
  }
  return c;
}

double mixture_vib_energy(const Param &p, double t, const double *y, double *cv_v) {
  // compute_mixture_vib_energy (src/Thermo.cu:725-737)
  double ev = 0.0, cvv = 0.0;
  if (p.tt.on)
    for (int i = 0; i < p.n_spec; ++i) {
      ev += y[i] * vib_energy(p, i, t);
      cvv += y[i] * vib_cv(p, i, t);
    }
  if (cv_v) *cv_v = cvv;
  return ev;
}

double mixture_tr_energy(const Param &p, double t, const double *y, double *cv_tr, double *cp_tr = nullptr,
                         double *r_mix = nullptr) {
  // compute_mixture_tr_energy (src/Thermo.cu:739-761)
  double h[16], cp[16];
  nasa7_h_cp(t, p.mech, h, cp);
  double e = 0.0, cpm = 0.0, rm = 0.0;
  for (int i = 0; i < p.n_spec; ++i) {
    cpm += y[i] * cp[i];
    rm += y[i] * p.mech.gas_const[i];
    e += y[i] * (h[i] - p.mech.gas_const[i] * t);
  }
  double cv_eq = 0.0;
  const double eve_eq = mixture_ve_energy(p, t, y, &cv_eq);
  const double cv_total = cpm - rm;
  if (cv_tr) *cv_tr = cv_total - cv_eq;
  if (cp_tr) *cp_tr = cpm - cv_eq;
  if (r_mix) *r_mix = rm;
  return e - eve_eq;
}

double mw_from_imw(double imw) { return 1.0 / std::max(imw, 1e-20); }

double pair_mw_time(const Param &p, int iv, int ip, double t, double pr) {
  // compute_pair_mw_relaxation_time (src/Thermo.cu:800-821)
  if (pr <= 1e-16 || t <= 1.0) return 1e30;
  const int ns = p.n_spec;
  const double mv = mw_from_imw(p.mech.imw[iv]);
  const double mp = mw_from_imw(p.mech.imw[ip]);
  const double mu = mv * mp / std::max(mv + mp, 1e-20);
  double a = p.tt.lt_a[iv * ns + ip];
  double b = p.tt.lt_b[iv * ns + ip];
  if (a <= 0.0 || b <= 0.0) {
    a = 1.16e-3 * std::sqrt(std::max(mu, 1e-20)) * std::pow(std::max(p.tt.theta_v[iv], 0.0), 4.0 / 3.0);
    b = 0.015 * std::pow(std::max(mu, 1e-20), 0.25);
  }
  const double ex = a * (std::pow(t, -1.0 / 3.0) - b) - 18.421;
  return std::max(std::exp(ex) * p_atm / pr, 1e-30);
}

double species_vt_time(const Param &p, int iv, double density, double t, double pr, const double *y) {
  // compute_species_vt_relaxation_time (src/Thermo.cu:823-853)
  double conc = 0.0, denom = 0.0;
  for (int j = 0; j < p.n_spec; ++j) {
    const double yj = std::max(y[j], 0.0);
    if (yj <= 0.0) continue;
    const double ml = yj / mw_from_imw(p.mech.imw[j]);
    const double tau = pair_mw_time(p, iv, j, t, pr);
    conc += ml;
    denom += ml / tau;
  }
  if (conc <= 0.0 || denom <= 0.0) return 1e30;
  const double tau_mw = conc / denom;
  const double sigma = std::max(p.tt.park_sigma[iv], 1e-30) * (2.5e9 / std::max(t * t, 1.0));
  const double n_total = density * conc * avogadro;
  const double mv = mw_from_imw(p.mech.imw[iv]);
  const double cs = std::sqrt(std::max(8.0 * R_u * t / (pi * mv), 1e-30));
  const double tau_park = 1.0 / std::max(sigma * cs * n_total, 1e-30);
  return std::max(tau_mw + tau_park, 1e-30);
}

void gather_y(const Zone &z, const Param &p, int i, int j, int k, double *y) {
  // gather_species_mass_fractions: the first n_spec scalars
  for (int l = 0; l < p.n_spec; ++l) y[l] = z.sv(i, j, k, l);
}
}  // namespace

double ve_energy(const Param &p, int i, double t) {
  // compute_ve_energy (src/Thermo.cu:635-654)
  if (!p.tt.on || i < 0 || i >= p.n_spec) return 0.0;
  const double temp = std::max(t, 1.0);
  const double r = p.mech.gas_const[i];
  double e = 0.0;
  e += vib_energy(p, i, temp);
  const int nl = p.tt.n_level[i];
  if (nl > 0) {
    double zs = 0.0, w = 0.0;
    for (int l = 0; l < nl; ++l) {
      const double th = p.tt.elec_theta[i * p.tt.max_level + l];
      const double g = p.tt.elec_g[i * p.tt.max_level + l];
      const double bz = g * std::exp(-th / temp);
      zs += bz;
      w += bz * th;
    }
    if (zs > 0) e += r * w / zs;
  }
  return e;
}

double ve_cv(const Param &p, int i, double t) {
  // compute_ve_cv (src/Thermo.cu:670-693)
  if (!p.tt.on || i < 0 || i >= p.n_spec) return 0.0;
  const double temp = std::max(t, 1.0);
  const double r = p.mech.gas_const[i];
  double c = 0.0;
  c += vib_cv(p, i, temp);
  const int nl = p.tt.n_level[i];
  if (nl > 0) {
    double zs = 0.0, b = 0.0, cc = 0.0;
    for (int l = 0; l < nl; ++l) {
      const double th = p.tt.elec_theta[i * p.tt.max_level + l];
      const double g = p.tt.elec_g[i * p.tt.max_level + l];
      const double bz = g * std::exp(-th / temp);
      zs += bz;
      b += bz * th;
      cc += bz * th * th;
    }
    if (zs > 0) {
      const double mean = b / zs;
      c += r * (cc / zs - mean * mean) / (temp * temp);
    }
  }
  return c;
}

double mixture_ve_energy(const Param &p, double t, const double *y, double *cv_ve) {
  // compute_mixture_ve_energy (src/Thermo.cu:711-723)
  double e = 0.0, c = 0.0;
  if (p.tt.on)
    for (int i = 0; i < p.n_spec; ++i) {
      e += y[i] * ve_energy(p, i, t);
      c += y[i] * ve_cv(p, i, t);
    }
  if (cv_ve) *cv_ve = c;
  return e;
}

double invert_tve_from_eve(const Param &p, double eve_target, const double *y, double t_init) {
  // invert_tve_from_eve (src/Thermo.cu:763-779): Newton on T_ve, at most 80 iterations
  double tve = std::max(t_init, 1.0);
  for (int it = 0; it < 80; ++it) {
    double cv = 0.0;
    const double eve = mixture_ve_energy(p, tve, y, &cv);
    const double res = eve - eve_target;
    if (std::fabs(res) < 1e-8 * std::max(1.0, std::fabs(eve_target))) break;
    const double next = std::max(1.0, tve - res / std::max(cv, 1e-8));
    if (std::fabs(next - tve) < 1e-8 * std::max(1.0, tve)) {
      tve = next;
      break;
    }
    tve = next;
  }
  return tve;
}

double vt_relaxation_source(const Param &p, double density, double t, double tve, const double *y, double *eve_eq,
                            double *tau_eff) {
  // compute_vt_relaxation_source (src/Thermo.cu:856-901)
  if (!p.tt.on || density <= 0.0) {
    if (eve_eq) *eve_eq = 0.0;
    if (tau_eff) *tau_eff = 1e30;
    return 0.0;
  }
  double rm = 0.0;
  for (int i = 0; i < p.n_spec; ++i) rm += std::max(y[i], 0.0) * p.mech.gas_const[i];
  const double pr = density * rm * std::max(t, 1.0);
  double eq_mix = 0.0, e_mix = 0.0, src = 0.0;
  for (int i = 0; i < p.n_spec; ++i) {
    if (p.tt.theta_v[i] <= 0.0) continue;
    const double yi = std::max(y[i], 0.0);
    if (yi <= 0.0) continue;
    const double e_eq = vib_energy(p, i, t);
    const double e_i = vib_energy(p, i, tve);
    const double d = e_eq - e_i;
    eq_mix += yi * e_eq;
    e_mix += yi * e_i;
    if (std::fabs(d) <= 1e-16) continue;
    const double tau = species_vt_time(p, i, density, t, pr, y);
    if (tau < 1e29) src += density * yi * d / tau;
  }
  if (eve_eq) *eve_eq = eq_mix;
  if (tau_eff) {
    const double dm = eq_mix - e_mix;
    if (std::fabs(dm) > 1e-16 && std::fabs(src) > 1e-16) *tau_eff = std::max(density * dm / src, 1e-30);
    else *tau_eff = 1e30;
  }
  return src;
}

void temperature_2t(Zone &z, const Param &p, int i, int j, int k, double total_energy) {
  // compute_temperature_and_pressure, two-temperature branch (src/FieldOperation.cu:4-63)
  const double density = z.bv(i, j, k, 0);
  double gc = 0;
  for (int l = 0; l < p.n_spec; ++l) gc += z.sv(i, j, k, l) * p.mech.gas_const[l];
  const double e = total_energy / density - 0.5 * (z.bv(i, j, k, 1) * z.bv(i, j, k, 1) +
                                                   z.bv(i, j, k, 2) * z.bv(i, j, k, 2) +
                                                   z.bv(i, j, k, 3) * z.bv(i, j, k, 3));
  double y[16];
  gather_y(z, p, i, j, k, y);
  double eve = std::max(z.sv(i, j, k, p.i_eve), 0.0);
  double tve = z.tve(i, j, k);
  if (tve <= 0) tve = std::max(z.bv(i, j, k, 5), 1.0);
  tve = invert_tve_from_eve(p, eve, y, tve);
  const double max_tve = std::max(1.0e7, 1000.0 * std::max(z.bv(i, j, k, 5), 1.0));
  if (!std::isfinite(eve) || !std::isfinite(tve) || tve <= 0.0 || tve > max_tve) {
    tve = std::max(z.bv(i, j, k, 5), 1.0);
    eve = mixture_ve_energy(p, tve, y, nullptr);
    z.sv(i, j, k, p.i_eve) = eve;
    z.cv(i, j, k, 5 + p.i_eve) = density * eve;
  }
  z.tve(i, j, k) = tve;
  double err = 1, t = std::max(z.bv(i, j, k, 5), 1.0);
  int iter = 0;
  while (err > 1e-5 && iter++ < 1000) {
    double cv_tr = 0;
    const double e_tr = mixture_tr_energy(p, t, y, &cv_tr);
    const double t1 = std::max(1.0, t - (e_tr - (e - eve)) / std::max(cv_tr, 1e-8));
    err = std::fabs(1 - t1 / t);
    t = t1;
  }
  z.bv(i, j, k, 5) = t;
  z.bv(i, j, k, 4) = density * t * gc;
}

void sync_two_temperature(Zone &z, const Param &p, int i, int j, int k) {
  // sync_two_temperature_state_from_sv (src/FieldOperation.cuh:28-58)
  if (p.i_eve < 0) return;
  double y[16];
  gather_y(z, p, i, j, k, y);
  const double t = std::max(z.bv(i, j, k, 5), 1.0);
  double tve = z.tve(i, j, k);
  const double max_guess = std::max(1.0e7, 1000.0 * t);
  if (!std::isfinite(tve) || tve <= 0.0 || tve > max_guess) tve = t;
  double &eve = z.sv(i, j, k, p.i_eve);
  if (!std::isfinite(eve) || eve <= 0.0) {
    eve = mixture_ve_energy(p, tve, y, nullptr);
  } else {
    const double tv = invert_tve_from_eve(p, eve, y, tve);
    if (std::isfinite(tv) && tv > 0.0 && tv <= max_guess) {
      tve = tv;
    } else {
      tve = t;
      eve = mixture_ve_energy(p, tve, y, nullptr);
    }
  }
  z.tve(i, j, k) = tve;
}

double total_energy_2t(Zone &z, const Param &p, int i, int j, int k) {
  // compute_total_energy, two-temperature branch (src/FieldOperation.cuh:90-109)
  const double V2 = z.bv(i, j, k, 1) * z.bv(i, j, k, 1) + z.bv(i, j, k, 2) * z.bv(i, j, k, 2) +
                    z.bv(i, j, k, 3) * z.bv(i, j, k, 3);
  double E = 0.5 * V2;
  double h[16], cp[16], y[16];
  const double t = z.bv(i, j, k, 5);
  nasa7_h_cp(t, p.mech, h, cp);
  gather_y(z, p, i, j, k, y);
  for (int l = 0; l < p.n_spec; ++l) E += (h[l] - p.mech.gas_const[l] * t) * y[l];
  E -= mixture_ve_energy(p, t, y, nullptr);
  E += z.sv(i, j, k, p.i_eve);
  E *= z.bv(i, j, k, 0);
  return E;
}

void apply_vt_relaxation(Zone &z, const Param &p, double dt_stage) {
  // apply_vt_relaxation_rk -> apply_vt_relaxation_1_point (src/RK.cuh:20-28,
  // src/FieldOperation.cuh:60-88) on every interior node
  if (!p.tt.on || !p.tt.enable_vt || p.i_eve < 0 || dt_stage <= 0.0) return;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < z.mz; ++k)
    for (int j = 0; j < z.my; ++j)
      for (int i = 0; i < z.mx; ++i) {
        const double density = z.cv(i, j, k, 0);
        if (density <= 0.0) continue;
        const double tve = z.tve(i, j, k) > 0.0 ? z.tve(i, j, k) : std::max(z.bv(i, j, k, 5), 1.0);
        double y[16];
        gather_y(z, p, i, j, k, y);
        double ev_eq = 0, tau = 0;
        vt_relaxation_source(p, density, z.bv(i, j, k, 5), tve, y, &ev_eq, &tau);
        if (tau >= 1e29 || !std::isfinite(tau)) continue;
        const double rev_old = std::max(z.cv(i, j, k, 5 + p.i_eve), 0.0);
        const double alpha = std::exp(-dt_stage / std::max(tau, 1e-30));
        const double ev_old = mixture_vib_energy(p, tve, y, nullptr);
        const double ev_new = ev_old * alpha + ev_eq * (1.0 - alpha);
        const double rev_new = rev_old + density * (ev_new - ev_old);
        z.cv(i, j, k, 5 + p.i_eve) = std::max(rev_new, 0.0);
        z.sv(i, j, k, p.i_eve) = z.cv(i, j, k, 5 + p.i_eve) / density;
        z.tve(i, j, k) = invert_tve_from_eve(p, z.sv(i, j, k, p.i_eve), y, tve);
        temperature_2t(z, p, i, j, k, z.cv(i, j, k, 4));
      }
}

void tr_heat_capacities(const Param &p, double t, const double *y, double &cv_tr, double &cp_tr, double &r_mix) {
  mixture_tr_energy(p, t, y, &cv_tr, &cp_tr, &r_mix);
}

// Roe-state characteristic thermo with two temperatures (src/Thermo.cuh:49-110,
// two_temperature on): h_tr = h - e_ve(T), cp_tr = cp - cv_ve(T); the e_ve row
// alpha = -(gamma - 1)/c^2 with energy coefficient 1.
void characteristic_thermo_2t(const Param &p, double t, const double *y, double *gamma, double *c, double *alpha,
                              double *ecoef, double *e_tr_out) {
  const double te = std::max(t, 1.0);
  double h[16], cp[16], htr[16];
  nasa7_h_cp(te, p.mech, h, cp);
  double r = 0, cpm = 0, cvm = 0, e_tr = 0;
  for (int l = 0; l < p.n_spec; ++l) {
    htr[l] = h[l] - ve_energy(p, l, te);
    const double cp_tr = cp[l] - ve_cv(p, l, te);
    e_tr += y[l] * (htr[l] - p.mech.gas_const[l] * te);
    r += y[l] * p.mech.gas_const[l];
    cpm += y[l] * cp_tr;
    cvm += y[l] * (cp_tr - p.mech.gas_const[l]);
  }
  const double g = cpm / std::max(cvm, 1e-8);
  const double cc = std::sqrt(std::max(g * r * te, 1e-12));
  *gamma = g;
  *c = cc;
  if (e_tr_out) *e_tr_out = e_tr;
  if (!alpha || !ecoef) return;
  const double gm1 = g - 1.0;
  const double c2 = std::max(cc * cc, 1e-30);
  const double inv_gm1 = 1.0 / std::max(gm1, 1e-12);
  for (int l = 0; l < p.n_spec; ++l) {
    const double a = (g * p.mech.gas_const[l] * te - gm1 * htr[l]) / c2;
    alpha[l] = a;
    ecoef[l] = -a * c2 * inv_gm1;
  }
  alpha[p.i_eve] = -gm1 / c2;
  ecoef[p.i_eve] = 1.0;
}

}  // namespace oracle
