// Finite-rate chemistry of one state: concentrations -> forward/backward rates -> rates of
// progress -> species creation and destruction (finite_rate_chemistry, generic-mechanism branch,
// src/FiniteRateChem.cu:1406-1488; forward_reaction_rate :1505-1554 with Troe :1536-1549;
// backward_reaction_rate :1560-1636; rate_of_progress :1638-1663; chemical_source :1665-1681;
// the two-temperature control temperatures reaction_temperature :1490-1503 and the e_ve
// source compute_two_temperature_chemical_source :19-31).
//
// The reaction loop is fused: each reaction's rate of progress is added to the per-species
// creation/destruction accumulators as soon as it is known, so no per-reaction arrays are
// needed; the additions happen in the reference's reaction order.  Callers that need the rates
// of progress themselves (the point-implicit Jacobian) pass arrays for them.  Arrhenius and
// Gibbs exponentials are FP64 in every precision form.
#pragma once
#include "common.cuh"
#include "thermo.cuh"
#include "thermo_2t.cuh"

namespace cb2 {

__device__ __forceinline__ double arrhenius(double t, double A, double b, double Ea) {
  return A * pow(t, b) * exp(-Ea / t);
}

// A T^b exp(-Ea/T) as one exponential, with ln T and 1/T formed once per temperature: the same
// value as the form above to a few ulp (the exponent's rounding), for a third of its cost.
struct LnT {
  double lnt, it;
  __device__ __forceinline__ explicit LnT(double t) : lnt(log(t)), it(1.0 / t) {}
};
__device__ __forceinline__ double arrhenius(const LnT &l, double A, double b, double Ea) {
  return A * exp(fma(b, l.lnt, -Ea * l.it));
}

// c^n for the small non-negative integer stoichiometric coefficients of a mechanism.
__device__ __forceinline__ double ipow(double c, int n) {
  double r = 1.0;
  for (int a = 0; a < n; ++a) r *= c;
  return r;
}

// Smoothed control temperature T^a Tve^b of a two-temperature reaction rate
// (reaction_temperature / smooth_reaction_temperature, src/FiniteRateChem.cu:1490-1503).
__device__ __forceinline__ double reaction_temperature(double t, double tve, double a, double b) {
  const double trx = pow(fmax(t, 1.0), a) * pow(fmax(tve, 1.0), b);
  constexpr double t_min = 800.0, eps = 80.0;
  return 0.5 * (trx + t_min + sqrt((trx - t_min) * (trx - t_min) + eps * eps));
}

// Forward and backward rates of progress of reaction r at t, concentrations c and
// g/(RT) of every species (used only for reactions whose backward rate follows from the
// equilibrium constant); temp_t = p_atm / (R_u T) * 1e-3.  With the mechanism's
// control-temperature model the forward rate runs at smooth(T^tcf_a Tve^tcf_b) and the backward
// rate at smooth(T^tcb_a Tve^tcb_b), its g/(RT) evaluated there (gibbs is then unused).
// The control temperatures and the backward g/(RT) of the last reaction, reused by the next one
// when its exponents are the same (the AIR5 model has two forward pairs and one backward pair):
// the same inputs give the same values, so the rates do not change.
template <int NS>
struct ParkCache {
  double fa, fb, tf, ba, bb, tb;
  LnT lf{1.0}, lb{1.0};
  bool have_g;
  double g[NS];
  __device__ __forceinline__ ParkCache() {
    const double qnan = __longlong_as_double(0x7ff8000000000000ll);
    fa = fb = ba = bb = qnan;
    tf = tb = 0;
    have_g = false;
  }
};

template <int NS>
__device__ __forceinline__ void reaction_progress(int r, double t0, double tve, const double *c,
                                                  const double *gibbs, double temp_t, const Mech &m,
                                                  double &q1_out, double &q2_out, ParkCache<NS> *pc = nullptr,
                                                  const LnT *lt0 = nullptr) {
  const int ty = __ldg(m.reac_type + r);
  const int *sf = m.stoi_f + r * NS, *sb = m.stoi_b + r * NS;
  double t = t0;
  LnT lt = m.park ? LnT(1.0) : (lt0 ? *lt0 : LnT(t0));
  if (m.park) {
    const double a = __ldg(m.tcf_a + r), b = __ldg(m.tcf_b + r);
    if (pc && pc->fa == a && pc->fb == b) {
      t = pc->tf;
      lt = pc->lf;
    } else {
      t = reaction_temperature(t0, tve, a, b);
      lt = LnT(t);
      if (pc) { pc->fa = a; pc->fb = b; pc->tf = t; pc->lf = lt; }
    }
  }
  // forward rate
  double kf = arrhenius(lt, __ldg(m.A + r), __ldg(m.b + r), __ldg(m.Ea + r));
  double cc = 0;
  if (ty > 3 || (ty != 0 && __ldg(m.rev_type + r) == 1 && ty == 4)) {
#pragma unroll
    for (int s = 0; s < NS; ++s) cc += c[s] * __ldg(m.tbc + r * NS + s);
  }
  if (ty == 3) {
    kf += arrhenius(lt, __ldg(m.A2 + r), __ldg(m.b2 + r), __ldg(m.Ea2 + r));
  } else if (ty == 4) {
    kf *= cc;
  } else if (ty > 4) {
    const double kf_low = arrhenius(lt, __ldg(m.A2 + r), __ldg(m.b2 + r), __ldg(m.Ea2 + r));
    const double kf_high = kf;
    if (kf_high < 1e-25 && kf_low < 1e-25) {
      kf = 0;
    } else {
      const double pr = kf_low * cc / kf_high;
      double F = 1.0;
      if (ty > 5) {
        const double al = __ldg(m.troe_alpha + r);
        double fc = (1 - al) * exp(-t / __ldg(m.troe_t3 + r)) + al * exp(-t / __ldg(m.troe_t1 + r));
        if (ty == 7) fc += exp(-__ldg(m.troe_t2 + r) / t);
        const double lfc = log10(fc);
        const double cq = -0.4 - 0.67 * lfc;
        const double nq = 0.75 - 1.27 * lfc;
        const double lpr = log10(pr);
        const double tmp = (lpr + cq) / (nq - 0.14 * (lpr + cq));
        F = pow(10.0, lfc / (1.0 + tmp * tmp));
      }
      kf = kf_high * pr / (1.0 + pr) * F;
    }
  }
  // backward rate
  double kb = 0;
  if (m.park) {
    if (ty != 0) {
      const double a = __ldg(m.tcb_a + r), b = __ldg(m.tcb_b + r);
      double thb;
      LnT lb(1.0);
      if (pc && pc->ba == a && pc->bb == b) {
        thb = pc->tb;
        lb = pc->lb;
      } else {
        thb = reaction_temperature(t0, tve, a, b);
        lb = LnT(thb);
        if (pc) { pc->ba = a; pc->bb = b; pc->tb = thb; pc->lb = lb; pc->have_g = false; }
      }
      if (__ldg(m.rev_type + r) == 1) {
        kb = arrhenius(lb, __ldg(m.A2 + r), __ldg(m.b2 + r), __ldg(m.Ea2 + r));
        if (ty == 4) kb *= cc;
      } else {
        double gl[NS];
        const double *g = gl;
        if (pc) {
          if (!pc->have_g) {
            species_gibbs_rt<NS>(thb, m, pc->g);
            pc->have_g = true;
          }
          g = pc->g;
        } else {
          species_gibbs_rt<NS>(thb, m, gl);
        }
        double dg = 0;
#pragma unroll
        for (int s = 0; s < NS; ++s) dg += g[s] * (__ldg(sb + s) - __ldg(sf + s));
        // (p_atm / (R_u T_b) 1e-3)^order exp(-dg) as one exponential
        const double kc = exp(fma(__ldg(m.reac_order + r), m.ln_temp_p - lb.lnt, -dg));
        kb = kf / kc;
      }
    }
  } else if (ty != 0) {
    if (__ldg(m.rev_type + r) == 1) {
      kb = arrhenius(lt, __ldg(m.A2 + r), __ldg(m.b2 + r), __ldg(m.Ea2 + r));
      if (ty == 4) kb *= cc;
    } else if (ty != 2) {
      double dg = 0;
#pragma unroll
      for (int s = 0; s < NS; ++s) dg += gibbs[s] * (__ldg(sb + s) - __ldg(sf + s));
      // temp_t^order exp(-dg), temp_t = p_atm / (R_u T) 1e-3, as one exponential
      const double kc = exp(fma(__ldg(m.reac_order + r), m.ln_temp_p - lt.lnt, -dg));
      kb = kf / kc;
    }
  }
  // rates of progress
  double q1 = 1.0, q2 = ty != 0 ? 1.0 : 0.0;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    q1 *= ipow(c[s], __ldg(sf + s));
    if (ty != 0) q2 *= ipow(c[s], __ldg(sb + s));
  }
  q1 *= kf;
  if (ty != 0) q2 *= kb;
  q1_out = q1;
  q2_out = q2;
}

// Whether any reaction takes its backward rate from the equilibrium constant.
__device__ __forceinline__ bool mech_needs_gibbs(const Mech &m) {
  for (int r = 0; r < m.n_reac; ++r) {
    const int ty = __ldg(m.reac_type + r);
    if (ty != 0 && __ldg(m.rev_type + r) != 1 && ty != 2) return true;
  }
  return false;
}

// t [K], c [mol/cm^3]; creation/destruction accumulate sum_r of q2 nu_f + q1 nu_b and
// q1 nu_f + q2 nu_b [mol/(cm^3 s)]; q1r/q2r (may be null) receive the forward and backward
// rates of progress of every reaction.
template <int NS>
__device__ __forceinline__ void chem_rates(double t, double tve, const double *c, const Mech &m, double *creation,
                                           double *destruction, double *q1r, double *q2r) {
  double gibbs[NS];
  if (!m.park && mech_needs_gibbs(m)) species_gibbs_rt<NS>(t, m, gibbs);
  constexpr double temp_p = kPatm / kRu * 1e-3;
  const double temp_t = temp_p / t;
  const LnT lt(t);
#pragma unroll
  for (int s = 0; s < NS; ++s) creation[s] = destruction[s] = 0;

  if (m.park) {
    ParkCache<NS> pc;
    for (int r = 0; r < m.n_reac; ++r) {
      double q1, q2;
      reaction_progress<NS>(r, t, tve, c, gibbs, temp_t, m, q1, q2, &pc);
      if (q1r) {
        q1r[r] = q1;
        q2r[r] = q2;
      }
      const int *sf = m.stoi_f + r * NS, *sb = m.stoi_b + r * NS;
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const double f = __ldg(sf + s), b = __ldg(sb + s);
        creation[s] += q2 * f + q1 * b;
        destruction[s] += q1 * f + q2 * b;
      }
    }
  } else {
    for (int r = 0; r < m.n_reac; ++r) {
      double q1, q2;
      reaction_progress<NS>(r, t, tve, c, gibbs, temp_t, m, q1, q2, nullptr, &lt);
      if (q1r) {
        q1r[r] = q1;
        q2r[r] = q2;
      }
      const int *sf = m.stoi_f + r * NS, *sb = m.stoi_b + r * NS;
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const double f = __ldg(sf + s), b = __ldg(sb + s);
        creation[s] += q2 * f + q1 * b;
        destruction[s] += q1 * f + q2 * b;
      }
    }
  }
}

// One node of the explicit source: dq[5+k] += J omega_k and the reaction time scale.
template <int NS>
__device__ __forceinline__ void chemistry_point(const Zone &z, const Param &p, int i, int j, int k) {
  const Mech &m = p.mech;
  const idx_t g = z.L.at(i, j, k), sz = z.L.sz;
  const double rho = z.bv[g], t = z.bv[g + 5 * sz];
  double c[NS], y[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    y[s] = z.sv[g + s * sz];
    c[s] = rho * y[s] * __ldg(m.imw + s) * 1e-3;
  }
  // two-temperature: the rates see max(T_ve, 1) (src/FiniteRateChem.cu:1450-1451)
  const bool tt = p.i_eve >= 0;
  const double tve_raw = tt ? z.tve[g] : t;
  double creation[NS], destruction[NS];
  chem_rates<NS>(t, tt ? fmax(tve_raw, 1.0) : t, c, m, creation, destruction, nullptr, nullptr);
  const double jac = z.jac[g];
  const idx_t g0 = z.L0.at(i, j, k), sz0 = z.L0.sz;
  // e_ve source sum_s omega_s e_ve,s(T_ve), T_ve replaced by max(T, 1) when not positive
  const double tve_src = tve_raw > 0.0 ? tve_raw : fmax(t, 1.0);
  double ts = 1e+6, eve_src = 0.0;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const double w = 1e+3 / __ldg(m.imw + s);
    const double od = destruction[s] * w;
    const double om = creation[s] * w - od;
    z.dq[g0 + (5 + s) * sz0] += jac * om;
    if (y[s] > 1e-25 && fabs(od) > 1e-25) ts = fmin(ts, fabs(rho * y[s] / od));
    if (tt) eve_src += om * ve_energy(s, tve_src, m, nullptr);
  }
  if (tt) z.dq[g0 + (5 + NS) * sz0] += jac * eve_src;
  if (z.rts) z.rts[g] = ts;
}

}  // namespace cb2
