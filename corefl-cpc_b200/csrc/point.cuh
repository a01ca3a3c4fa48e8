// Per-node operations shared by the block kernels and the batched (one CTA per case) kernels:
// the RK3 stage update with primitive recovery, the physical properties, the local CFL time step
// and the conservative-from-primitive fill of one node.  The block kernels call these with their
// own thread-to-node mapping, so both paths run the same arithmetic.
#pragma once
#include "common.cuh"
#include "thermo.cuh"
#include "thermo_2t.cuh"
#include "transport.cuh"

namespace cb2 {

// Newton inversion of T from the internal energy e (1T mixtures): stops at |1 - T1/T| <= 1e-5
// or after 1000 iterations, starting from the previous temperature (src/FieldOperation.cu:67-85).
template <int NS>
__device__ __forceinline__ double newton_temperature(double e, const double *y, double r_mix, double t,
                                                     const Mech &m) {
  double err = 1;
  int iter = 0;
  double h[NS], cp[NS];
  while (err > 1e-5 && iter++ < 1000) {
    species_h_cp<NS>(t, m, h, cp);
    double cpt = 0, ht = 0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      cpt += cp[s] * y[s];
      ht += h[s] * y[s];
    }
    const double et = ht - r_mix * t;
    const double cvt = cpt - r_mix;
    const double t1 = t - (et - e) / cvt;
    err = fabs(1 - t1 / t);
    t = t1;
  }
  return t;
}

// SSP-RK3 stage update of one interior node (update_cv_and_bv_rk<mix>, src/RK.cuh:277-367).
// TT: two-temperature model, rho*e_ve at cv comp 5 + NS (clipped at zero), e_ve at sv comp NS,
// T_ve and T from the two-temperature inversion.
template <int NS, bool TT = false>
__device__ __forceinline__ void stage_update_point(const Zone &z, const Param &p, double dt, int rk, int i, int j,
                                                   int k) {
  static_assert(!TT || NS > 0, "the two-temperature model needs species");
  constexpr int NV = 5 + NS + (TT ? 1 : 0);
  double a, b, c;
  ssprk3_coeff(rk, a, b, c);
  const idx_t g = z.L.at(i, j, k), sz = z.L.sz;
  const idx_t g0 = z.L0.at(i, j, k), sz0 = z.L0.sz;
  const double dtj = dt / z.jac[g];
  double q[NV];
#pragma unroll
  for (int l = 0; l < NV; ++l) q[l] = a * z.qn[g + l * sz] + b * z.cv[g + l * sz] + c * dtj * z.dq[g0 + l * sz0];
  if (z.mz == 1) q[3] = 0;
  if (!(q[0] > 0) || !isfinite(q[4])) flag_status(p, 1u);

  const double rho = q[0];
  const double dinv = 1.0 / rho;
  const double u = q[1] * dinv, v = q[2] * dinv, w = q[3] * dinv;
  const double V2 = u * u + v * v + w * w;
  z.bv[g] = rho;
  z.bv[g + sz] = u;
  z.bv[g + 2 * sz] = v;
  z.bv[g + 3 * sz] = w;
  if constexpr (NS == 0) {
    const double pr = (kGammaAir - 1) * (q[4] - 0.5 * rho * V2);
    z.bv[g + 4 * sz] = pr;
    z.bv[g + 5 * sz] = pr * kMwAir * dinv / kRu;
  } else {
    // clip negative partial densities, renormalise to sum(rho Y) = rho
    double sum = 0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      if (q[5 + s] < 0) q[5 + s] = 0;
      else sum += q[5 + s];
    }
    if constexpr (TT) q[5 + NS] = fmax(q[5 + NS], 0.0);
    sum = 1.0 / sum;
    const double scale = rho * sum;
    double y[NS], r_mix = 0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      y[s] = q[5 + s] * sum;
      q[5 + s] *= scale;
      z.sv[g + s * sz] = y[s];
    }
    if constexpr (TT) {
      z.sv[g + NS * sz] = q[5 + NS] * dinv;
#pragma unroll
      for (int l = 0; l < NV; ++l) z.cv[g + l * sz] = q[l];
      temperature_2t<NS>(z, p, g, q[4]);
      return;
    }
#pragma unroll
    for (int s = 0; s < NS; ++s) r_mix += y[s] * __ldg(p.mech.gas_const + s);
    const double e = q[4] / rho - 0.5 * V2;
    const double t = newton_temperature<NS>(e, y, r_mix, z.bv[g + 5 * sz], p.mech);
    const double pr = rho * t * r_mix;
    z.bv[g + 5 * sz] = t;
    z.bv[g + 4 * sz] = pr;
    if (!(t > 0) || !(pr > 0)) flag_status(p, 2u);
  }
#pragma unroll
  for (int l = 0; l < NV; ++l) z.cv[g + l * sz] = q[l];
}

// Physical properties of one node (update_physical_properties<mix>,
// src/FieldOperation.cuh:183-247).  transport = false skips mu, kappa and rho*D of a mixture
// (used by callers that take no viscous or diffusive term).
// F32T: the transport coefficients in FP32 (the mixed form).
template <int NS, bool F32T = false>
__device__ __forceinline__ void properties_point(const Zone &z, const Param &p, int i, int j, int k,
                                                 bool transport = true) {
  const idx_t g = z.L.at(i, j, k), sz = z.L.sz;
  const double t = z.bv[g + 5 * sz];
  const double V = norm3d(z.bv[g + sz], z.bv[g + 2 * sz], z.bv[g + 3 * sz]);
  if constexpr (NS == 0) {
    z.mul[g] = p.mu_constant > 0 ? p.mu_constant : sutherland(t);
    if (z.mach) z.mach[g] = V / sqrt(kGammaAir * kRu / kMwAir * t);
  } else {
    double cp[NS], y[NS];
    species_cp<NS>(t, p.mech, cp);
    double imw = 0, cpt = 0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      y[s] = z.sv[g + s * sz];
      imw = fma(y[s], __ldg(p.mech.imw + s), imw);
      cpt = fma(y[s], cp[s], cpt);
    }
    const double mw = 1 / fmax(imw, 1e-12);
    const double R = kRu * imw;
    const bool tt = p.i_eve >= 0;
    if (tt) {
      // two-temperature (src/FieldOperation.cuh:207-226): gamma and c of the
      // translational-rotational mode; T_ve defaults to T
      double cv_tr, cp_tr, r_mix;
      tr_heat_capacities<NS>(t, y, p.mech, cv_tr, cp_tr, r_mix);
      const double gam = cp_tr / fmax(cv_tr, 1e-8);
      z.gamma[g] = gam;
      const double a = sqrt(fmax(gam * r_mix * t, 1e-12));
      z.acoustic[g] = a;
      if (z.mach) z.mach[g] = V / a;
      if (z.tve[g] <= 0) z.tve[g] = t;
    } else {
      const double gam = cpt / (cpt - R);
      z.gamma[g] = gam;
      const double c = sqrt(gam * R * t);
      z.acoustic[g] = c;
      if (z.mach) z.mach[g] = V / c;
    }
    if (!transport) return;
    double mu, kappa, rhoD[NS];
    if constexpr (F32T) transport_properties_f32<NS>(t, mw, y, cp, p.mech, mu, kappa, rhoD);
    else transport_properties<NS>(t, z.bv[g + 4 * sz], mw, y, cp, p.mech, mu, kappa, rhoD);
    z.mul[g] = mu;
    z.kappa[g] = kappa;
#pragma unroll
    for (int s = 0; s < NS; ++s) z.rhoD[g + s * sz] = rhoD[s];
    if (tt && z.kappa_ve) {
      // kappa_ve = kappa cv_ve(T_ve) / cp
      double cv_ve;
      mixture_ve_energy<NS>(z.tve[g], y, p.mech, &cv_ve);
      z.kappa_ve[g] = kappa * cv_ve / fmax(cpt, 1e-8);
    }
  }
}

// Local CFL time step of one interior node (local_time_step<mix>, src/TimeAdvanceFunc.cuh:28-127).
template <int NS>
__device__ __forceinline__ double local_dt_point(const Zone &z, const Param &p, int i, int j, int k) {
  const idx_t g = z.L.at(i, j, k), sz = z.L.sz;
  const double *M = z.metric;
  const double gxi = norm3d(M[g], M[g + sz], M[g + 2 * sz]);
  const double geta = norm3d(M[g + 3 * sz], M[g + 4 * sz], M[g + 5 * sz]);
  const double gzeta = norm3d(M[g + 6 * sz], M[g + 7 * sz], M[g + 8 * sz]);
  const double u = z.bv[g + sz], v = z.bv[g + 2 * sz], w = z.bv[g + 3 * sz];
  const double U = u * M[g] + v * M[g + sz] + w * M[g + 2 * sz];
  const double Vc = u * M[g + 3 * sz] + v * M[g + 4 * sz] + w * M[g + 5 * sz];
  const double W = u * M[g + 6 * sz] + v * M[g + 7 * sz] + w * M[g + 8 * sz];
  double a;
  if constexpr (NS == 0) a = sqrt(kGammaAir * kRAir * z.bv[g + 5 * sz]);
  else a = z.acoustic[g];
  const bool d3 = z.mz != 1;
  double lam = fmax(fabs(U) + a * gxi, fabs(Vc) + a * geta);
  if (d3) lam = fmax(lam, fabs(W) + a * gzeta);
  if (p.viscous_order > 0) {
    double len = fmax(gxi, geta);
    if (d3) len = fmax(len, gzeta);
    const double irho = 1.0 / z.bv[g];
    double dv;
    if constexpr (NS == 0) {
      dv = fmax(kGammaAir, 4.0 / 3.0) * irho;
      dv *= z.mul[g] / p.Pr;
    } else {
      double cp[NS];
      species_cp<NS>(z.bv[g + 5 * sz], p.mech, cp);
      double cpt = 0, mrd = 0;
      for (int s = 0; s < NS; ++s) {
        cpt += cp[s] * z.sv[g + s * sz];
        mrd = fmax(mrd, z.rhoD[g + s * sz]);
      }
      dv = z.mul[g] * irho;
      dv = fmax(dv, z.kappa[g] * irho * z.gamma[g] / cpt);
      dv = fmax(dv, mrd * irho);
      if (p.i_eve >= 0 && z.kappa_ve) {
        // two-temperature: the e_ve conduction kappa_ve / (rho cv_ve) (src/TimeAdvanceFunc.cuh:95-106)
        const double tve = z.tve[g] > 0.0 ? z.tve[g] : fmax(z.bv[g + 5 * sz], 1.0);
        double y[NS], cv_ve;
#pragma unroll
        for (int s = 0; s < NS; ++s) y[s] = z.sv[g + s * sz];
        mixture_ve_energy<NS>(tve, y, p.mech, &cv_ve);
        dv = fmax(dv, z.kappa_ve[g] * irho / fmax(cv_ve, 1e-8));
      }
    }
    lam = fmax(lam, len * len * dv);
  }
  double dt = p.cfl / lam;
  if constexpr (NS > 0) {
    if (p.n_reac > 0 && z.rts) {
      const double rdt = p.cfl * z.rts[g];
      if (rdt > 1e-20 && rdt < 1e-5) dt = fmin(dt, rdt);
    }
  }
  return dt;
}

// Conservative variables of one node from its primitives (compute_cv_from_bv_1_point,
// src/FieldOperation.cuh:163).
template <int NS>
__device__ __forceinline__ void cv_point(const Zone &z, const Param &p, idx_t g) {
  const idx_t sz = z.L.sz;
  const double rho = z.bv[g], u = z.bv[g + sz], v = z.bv[g + 2 * sz], w = z.bv[g + 3 * sz];
  z.cv[g] = rho;
  z.cv[g + sz] = rho * u;
  z.cv[g + 2 * sz] = rho * v;
  z.cv[g + 3 * sz] = rho * w;
  double E = 0.5 * (u * u + v * v + w * w);
  if constexpr (NS == 0) {
    E *= rho;
    E += z.bv[g + 4 * sz] / (kGammaAir - 1);
  } else if (p.i_eve >= 0) {
    // two-temperature (src/FieldOperation.cuh:154-158, 97-109)
    sync_two_temperature<NS>(z, p, g);
#pragma unroll
    for (int s = 0; s <= NS; ++s) z.cv[g + (5 + s) * sz] = rho * z.sv[g + s * sz];
    E = total_energy_2t<NS>(z, p, g);
  } else {
    double h[NS];
    species_h<NS>(z.bv[g + 5 * sz], p.mech, h);
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const double y = z.sv[g + s * sz];
      z.cv[g + (5 + s) * sz] = rho * y;
      E += h[s] * y;
    }
    E *= rho;
    E -= z.bv[g + 4 * sz];
  }
  z.cv[g + 4 * sz] = E;
}

}  // namespace cb2
