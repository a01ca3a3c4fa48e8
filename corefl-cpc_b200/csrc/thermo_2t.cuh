// Two-temperature (vibrational-electronic) model: species and mixture e_ve and cv_ve, the T_ve
// and T inversions, and the Landau-Teller VT relaxation with Millikan-White + Park relaxation
// times (src/Thermo.cu:635-901, src/FieldOperation.cu:24-63, src/FieldOperation.cuh:28-109).
// e_ve lives as the scalar i_eve = NS of sv, rho*e_ve as comp 5 + NS of cv, T_ve in z.tve.
// All FP64 in every form: these are the temperature inversions and the exponentials.
#pragma once
#include "common.cuh"
#include "thermo.cuh"

namespace cb2 {

constexpr double kAvogadro = 6.02214076e26;  // 1/kmol
constexpr double kPi = 3.141592653589793;

// Vibrational energy and heat capacity of species i (compute_vib_energy / compute_vib_cv,
// src/Thermo.cu:656-668, 695-709): harmonic oscillator R theta / (exp(theta/T) - 1).
__device__ __forceinline__ double vib_energy(int i, double t, const Mech &m) {
  const double temp = fmax(t, 1.0);
  const double th = __ldg(m.theta_v + i);
  double e = 0.0;
  if (th > 0) {
    const double x = th / temp;
    if (x < 200) e += __ldg(m.gas_const + i) * th / expm1(x);
  }
  return e;
}

__device__ __forceinline__ double vib_cv(int i, double t, const Mech &m) {
  const double temp = fmax(t, 1.0);
  const double th = __ldg(m.theta_v + i);
  double c = 0.0;
  if (th > 0) {
    const double x = th / temp;
    if (x < 200) {
      const double ex = exp(x);
      const double d = ex - 1.0;
      c += __ldg(m.gas_const + i) * x * x * ex / (d * d);
    }
  }
  return c;
}

// e_ve of species i: vibration plus the electronic levels' Boltzmann average (compute_ve_energy,
// src/Thermo.cu:635-654); with cv: its heat capacity too (compute_ve_cv, :670-693).
// The level sums run in the reference's order and stop at the first level l >= 2 with
// theta_l - theta_1 > A_i T (A_i = m.elec_cut[i], set at mechanism upload): every remaining
// term is then below half an ulp of each running sum, so adding it would leave the sums -- and
// the result -- unchanged.  At the cold freestream of a hypersonic case this skips most of the
// 46 exponentials of AIR5.
__device__ __forceinline__ double ve_energy(int i, double t, const Mech &m, double *cv) {
  const double temp = fmax(t, 1.0);
  const double r = __ldg(m.gas_const + i);
  double e = vib_energy(i, temp, m);
  double c = cv ? vib_cv(i, temp, m) : 0.0;
  const int nl = __ldg(m.n_level + i);
  if (nl > 0) {
    double zs = 0.0, b = 0.0, cc = 0.0;
    const double cut_t = __ldg(m.elec_cut + i) * temp;
    double th1 = 0.0;
    for (int l = 0; l < nl; ++l) {
      const double th = __ldg(m.elec_theta + i * m.max_level + l);
      if (l == 1) th1 = th;
      else if (l > 1 && th - th1 > cut_t) break;
      const double bz = __ldg(m.elec_g + i * m.max_level + l) * exp(-th / temp);
      zs += bz;
      b += bz * th;
      cc += bz * th * th;
    }
    if (zs > 0) {
      e += r * b / zs;
      if (cv) {
        const double mean = b / zs;
        c += r * (cc / zs - mean * mean) / (temp * temp);
      }
    }
  }
  if (cv) *cv = c;
  return e;
}

// Mixture e_ve (and cv_ve) at t (compute_mixture_ve_energy, src/Thermo.cu:711-723).
template <int NS>
__device__ __forceinline__ double mixture_ve_energy(double t, const double *y, const Mech &m, double *cv_ve) {
  double e = 0.0, c = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) {
    double ci;
    const double ei = ve_energy(i, t, m, cv_ve ? &ci : nullptr);
    e += y[i] * ei;
    if (cv_ve) c += y[i] * ci;
  }
  if (cv_ve) *cv_ve = c;
  return e;
}

// Mixture vibrational energy only (compute_mixture_vib_energy, src/Thermo.cu:725-737).
template <int NS>
__device__ __forceinline__ double mixture_vib_energy(double t, const double *y, const Mech &m) {
  double e = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) e += y[i] * vib_energy(i, t, m);
  return e;
}

// Translational-rotational energy e - e_ve(T) and its heat capacity (compute_mixture_tr_energy,
// src/Thermo.cu:739-761).
template <int NS>
__device__ __forceinline__ double mixture_tr_energy(double t, const double *y, const Mech &m, double &cv_tr) {
  double h[NS], cp[NS];
  species_h_cp<NS>(t, m, h, cp);
  double e = 0.0, cpm = 0.0, rm = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) {
    const double r = __ldg(m.gas_const + i);
    cpm += y[i] * cp[i];
    rm += y[i] * r;
    e += y[i] * (h[i] - r * t);
  }
  double cv_eq;
  const double eve_eq = mixture_ve_energy<NS>(t, y, m, &cv_eq);
  cv_tr = (cpm - rm) - cv_eq;
  return e - eve_eq;
}

// cv_tr, cp_tr and R of the mixture at t (the heat capacities compute_mixture_tr_energy returns,
// src/Thermo.cu:739-761).
template <int NS>
__device__ __forceinline__ void tr_heat_capacities(double t, const double *y, const Mech &m, double &cv_tr,
                                                   double &cp_tr, double &r_mix) {
  double h[NS], cp[NS];
  species_h_cp<NS>(t, m, h, cp);
  double cpm = 0.0, rm = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) {
    cpm += y[i] * cp[i];
    rm += y[i] * __ldg(m.gas_const + i);
  }
  double cv_eq;
  mixture_ve_energy<NS>(t, y, m, &cv_eq);
  cv_tr = (cpm - rm) - cv_eq;
  cp_tr = cpm - cv_eq;
  r_mix = rm;
}

// Newton inversion of T_ve from e_ve, at most 80 iterations (invert_tve_from_eve,
// src/Thermo.cu:763-779).
template <int NS>
__device__ __forceinline__ double invert_tve_from_eve(double eve_target, const double *y, double t_init,
                                                      const Mech &m) {
  double tve = fmax(t_init, 1.0);
  for (int it = 0; it < 80; ++it) {
    double cv;
    const double eve = mixture_ve_energy<NS>(tve, y, m, &cv);
    const double res = eve - eve_target;
    if (fabs(res) < 1e-8 * fmax(1.0, fabs(eve_target))) break;
    const double next = fmax(1.0, tve - res / fmax(cv, 1e-8));
    if (fabs(next - tve) < 1e-8 * fmax(1.0, tve)) {
      tve = next;
      break;
    }
    tve = next;
  }
  return tve;
}

// Millikan-White time of the pair (vibrator iv, partner ip) at (t, p) (src/Thermo.cu:800-821).
__device__ __forceinline__ double pair_mw_time(int iv, int ip, double t, double pr, const Mech &m) {
  if (pr <= 1e-16 || t <= 1.0) return 1e30;
  const double mv = 1.0 / fmax(__ldg(m.imw + iv), 1e-20);
  const double mp = 1.0 / fmax(__ldg(m.imw + ip), 1e-20);
  const double mu = mv * mp / fmax(mv + mp, 1e-20);
  double a = __ldg(m.lt_a + iv * m.n_spec + ip);
  double b = __ldg(m.lt_b + iv * m.n_spec + ip);
  if (a <= 0.0 || b <= 0.0) {
    a = 1.16e-3 * sqrt(fmax(mu, 1e-20)) * pow(fmax(__ldg(m.theta_v + iv), 0.0), 4.0 / 3.0);
    b = 0.015 * pow(fmax(mu, 1e-20), 0.25);
  }
  const double ex = a * (pow(t, -1.0 / 3.0) - b) - 18.421;
  return fmax(exp(ex) * kPatm / pr, 1e-30);
}

// Relaxation time of vibrator iv: mole-weighted Millikan-White plus Park's high-temperature
// correction (src/Thermo.cu:823-853).
template <int NS>
__device__ __forceinline__ double species_vt_time(int iv, double density, double t, double pr, const double *y,
                                                  const Mech &m) {
  double conc = 0.0, denom = 0.0;
#pragma unroll
  for (int j = 0; j < NS; ++j) {
    const double yj = fmax(y[j], 0.0);
    if (yj <= 0.0) continue;
    const double ml = yj / (1.0 / fmax(__ldg(m.imw + j), 1e-20));
    const double tau = pair_mw_time(iv, j, t, pr, m);
    conc += ml;
    denom += ml / tau;
  }
  if (conc <= 0.0 || denom <= 0.0) return 1e30;
  const double tau_mw = conc / denom;
  const double sigma = fmax(__ldg(m.park_sigma + iv), 1e-30) * (2.5e9 / fmax(t * t, 1.0));
  const double n_total = density * conc * kAvogadro;
  const double mv = 1.0 / fmax(__ldg(m.imw + iv), 1e-20);
  const double cs = sqrt(fmax(8.0 * kRu * t / (kPi * mv), 1e-30));
  const double tau_park = 1.0 / fmax(sigma * cs * n_total, 1e-30);
  return fmax(tau_mw + tau_park, 1e-30);
}

// Landau-Teller source, equilibrium e_v and effective relaxation time
// (compute_vt_relaxation_source, src/Thermo.cu:856-901).
template <int NS>
__device__ __forceinline__ double vt_relaxation_source(double density, double t, double tve, const double *y,
                                                       const Mech &m, double &eve_eq, double &tau_eff) {
  if (density <= 0.0) {
    eve_eq = 0.0;
    tau_eff = 1e30;
    return 0.0;
  }
  double rm = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) rm += fmax(y[i], 0.0) * __ldg(m.gas_const + i);
  const double pr = density * rm * fmax(t, 1.0);
  double eq_mix = 0.0, e_mix = 0.0, src = 0.0;
  for (int i = 0; i < NS; ++i) {
    if (__ldg(m.theta_v + i) <= 0.0) continue;
    const double yi = fmax(y[i], 0.0);
    if (yi <= 0.0) continue;
    const double e_eq = vib_energy(i, t, m);
    const double e_i = vib_energy(i, tve, m);
    const double d = e_eq - e_i;
    eq_mix += yi * e_eq;
    e_mix += yi * e_i;
    if (fabs(d) <= 1e-16) continue;
    const double tau = species_vt_time<NS>(i, density, t, pr, y, m);
    if (tau < 1e29) src += density * yi * d / tau;
  }
  eve_eq = eq_mix;
  const double dm = eq_mix - e_mix;
  tau_eff = (fabs(dm) > 1e-16 && fabs(src) > 1e-16) ? fmax(density * dm / src, 1e-30) : 1e30;
  return src;
}

// T_ve from e_ve, then T from the translational-rotational energy (compute_temperature_and_pressure,
// two-temperature branch, src/FieldOperation.cu:24-63) at padded index g: writes tve, bv T and p,
// and resets e_ve (sv and cv) to equilibrium at T when the T_ve inversion fails.
template <int NS>
__device__ __forceinline__ void temperature_2t(const Zone &z, const Param &p, idx_t g, double total_energy) {
  const idx_t sz = z.L.sz;
  const double density = z.bv[g];
  double y[NS], gc = 0;
#pragma unroll
  for (int l = 0; l < NS; ++l) {
    y[l] = z.sv[g + l * sz];
    gc += y[l] * __ldg(p.mech.gas_const + l);
  }
  const double u = z.bv[g + sz], v = z.bv[g + 2 * sz], w = z.bv[g + 3 * sz];
  const double e = total_energy / density - 0.5 * (u * u + v * v + w * w);
  const double t_old = z.bv[g + 5 * sz];
  double eve = fmax(z.sv[g + NS * sz], 0.0);
  double tve = z.tve[g];
  if (tve <= 0) tve = fmax(t_old, 1.0);
  tve = invert_tve_from_eve<NS>(eve, y, tve, p.mech);
  const double max_tve = fmax(1.0e7, 1000.0 * fmax(t_old, 1.0));
  if (!isfinite(eve) || !isfinite(tve) || tve <= 0.0 || tve > max_tve) {
    tve = fmax(t_old, 1.0);
    eve = mixture_ve_energy<NS>(tve, y, p.mech, nullptr);
    z.sv[g + NS * sz] = eve;
    z.cv[g + (5 + NS) * sz] = density * eve;
  }
  z.tve[g] = tve;
  double err = 1, t = fmax(t_old, 1.0);
  int iter = 0;
  while (err > 1e-5 && iter++ < 1000) {
    double cv_tr;
    const double e_tr = mixture_tr_energy<NS>(t, y, p.mech, cv_tr);
    const double t1 = fmax(1.0, t - (e_tr - (e - eve)) / fmax(cv_tr, 1e-8));
    err = fabs(1 - t1 / t);
    t = t1;
  }
  z.bv[g + 5 * sz] = t;
  z.bv[g + 4 * sz] = density * t * gc;
  if (!(t > 0) || !isfinite(t)) flag_status(p, 2u);
}

// e_ve / T_ve consistency before a conservative fill (sync_two_temperature_state_from_sv,
// src/FieldOperation.cuh:28-58).
template <int NS>
__device__ __forceinline__ void sync_two_temperature(const Zone &z, const Param &p, idx_t g) {
  const idx_t sz = z.L.sz;
  double y[NS];
#pragma unroll
  for (int l = 0; l < NS; ++l) y[l] = z.sv[g + l * sz];
  const double t = fmax(z.bv[g + 5 * sz], 1.0);
  double tve = z.tve[g];
  const double max_guess = fmax(1.0e7, 1000.0 * t);
  if (!isfinite(tve) || tve <= 0.0 || tve > max_guess) tve = t;
  double eve = z.sv[g + NS * sz];
  if (!isfinite(eve) || eve <= 0.0) {
    eve = mixture_ve_energy<NS>(tve, y, p.mech, nullptr);
  } else {
    const double tv = invert_tve_from_eve<NS>(eve, y, tve, p.mech);
    if (isfinite(tv) && tv > 0.0 && tv <= max_guess) {
      tve = tv;
    } else {
      tve = t;
      eve = mixture_ve_energy<NS>(tve, y, p.mech, nullptr);
    }
  }
  z.sv[g + NS * sz] = eve;
  z.tve[g] = tve;
}

// Total energy rho (e_tr(T) + e_ve + |V|^2/2) (compute_total_energy, two-temperature branch,
// src/FieldOperation.cuh:90-109).
template <int NS>
__device__ __forceinline__ double total_energy_2t(const Zone &z, const Param &p, idx_t g) {
  const idx_t sz = z.L.sz;
  const double u = z.bv[g + sz], v = z.bv[g + 2 * sz], w = z.bv[g + 3 * sz], t = z.bv[g + 5 * sz];
  double E = 0.5 * (u * u + v * v + w * w);
  double h[NS], cp[NS], y[NS];
  species_h_cp<NS>(t, p.mech, h, cp);
#pragma unroll
  for (int l = 0; l < NS; ++l) {
    y[l] = z.sv[g + l * sz];
    E += (h[l] - __ldg(p.mech.gas_const + l) * t) * y[l];
  }
  E -= mixture_ve_energy<NS>(t, y, p.mech, nullptr);
  E += z.sv[g + NS * sz];
  return E * z.bv[g];
}

// One node of the VT relaxation step (apply_vt_relaxation_1_point, src/FieldOperation.cuh:60-88):
// e_v relaxes exponentially towards equilibrium at T over dt_stage, then T_ve and T follow.
template <int NS>
__device__ __forceinline__ void vt_relax_point(const Zone &z, const Param &p, idx_t g, double dt_stage) {
  const idx_t sz = z.L.sz;
  const double density = z.cv[g];
  if (density <= 0.0) return;
  const double tve = z.tve[g] > 0.0 ? z.tve[g] : fmax(z.bv[g + 5 * sz], 1.0);
  double y[NS];
#pragma unroll
  for (int l = 0; l < NS; ++l) y[l] = z.sv[g + l * sz];
  double ev_eq, tau;
  vt_relaxation_source<NS>(density, z.bv[g + 5 * sz], tve, y, p.mech, ev_eq, tau);
  if (tau >= 1e29 || !isfinite(tau)) return;
  const double rev_old = fmax(z.cv[g + (5 + NS) * sz], 0.0);
  const double alpha = exp(-dt_stage / fmax(tau, 1e-30));
  const double ev_old = mixture_vib_energy<NS>(tve, y, p.mech);
  const double ev_new = ev_old * alpha + ev_eq * (1.0 - alpha);
  const double rev_new = rev_old + density * (ev_new - ev_old);
  const double rev = fmax(rev_new, 0.0);
  z.cv[g + (5 + NS) * sz] = rev;
  const double eve = rev / density;
  z.sv[g + NS * sz] = eve;
  z.tve[g] = invert_tve_from_eve<NS>(eve, y, tve, p.mech);
  temperature_2t<NS>(z, p, g, z.cv[g + 4 * sz]);
}

// Roe-state characteristic thermo of the two-temperature model (src/Thermo.cuh:49-110 with
// two_temperature on): gamma and c of the translational-rotational mode, h_tr = h - e_ve(T),
// cp_tr = cp - cv_ve(T), and (etr not null) the mixture's translational-rotational energy
// e_tr = sum Y (h_tr - R T); with alpha and ecoef not null, the species rows alpha_s and energy
// coefficients as in one temperature, and the e_ve scalar's row alpha = -(gamma - 1)/c^2 with
// energy coefficient 1.
template <int NS>
__device__ __forceinline__ void characteristic_thermo_2t(double t, const double *y, const Mech &m, double &gamma,
                                                         double &c, double *alpha, double *ecoef,
                                                         double *etr = nullptr) {
  const double te = fmax(t, 1.0);
  double h[NS], cp[NS], htr[NS];
  species_h_cp<NS>(te, m, h, cp);
  double r = 0, cpm = 0, cvm = 0, e_tr = 0;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    double cv_ve;
    const double e_ve = ve_energy(s, te, m, &cv_ve);
    const double rs = __ldg(m.gas_const + s);
    htr[s] = h[s] - e_ve;
    const double cp_tr = cp[s] - cv_ve;
    e_tr += y[s] * (htr[s] - rs * te);
    r += y[s] * rs;
    cpm += y[s] * cp_tr;
    cvm += y[s] * (cp_tr - rs);
  }
  gamma = cpm / fmax(cvm, 1e-8);
  c = sqrt(fmax(gamma * r * te, 1e-12));
  if (etr) *etr = e_tr;
  if (!alpha || !ecoef) return;
  const double gm1 = gamma - 1.0;
  const double c2 = fmax(c * c, 1e-30);
  const double inv_gm1 = 1.0 / fmax(gm1, 1e-12);
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const double a = (gamma * __ldg(m.gas_const + s) * te - gm1 * htr[s]) / c2;
    alpha[s] = a;
    ecoef[s] = -a * c2 * inv_gm1;
  }
  alpha[NS] = -gm1 / c2;
  ecoef[NS] = 1.0;
}

}  // namespace cb2
