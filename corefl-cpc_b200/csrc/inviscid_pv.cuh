// Inviscid flux from reconstructed primitive variables and an approximate Riemann solver,
// fused with the flux difference (compute_convective_term_pv_1D, src/InviscidScheme.cu:61-169;
// Roe_compute_inviscid_flux_1D, :306-395).
//
// Reconstruction of (rho,u,v,w,p,Y) at i+1/2 (reconstruction<mix>, src/InviscidScheme.cu:171-219):
//   1 first order, 2 MUSCL kappa=1/3 with minmod (src/Reconstruction.cu:14-32),
//   3 NND2 (src/Reconstruction.cu:34-45), and, added here, 5/7 = WENO5-JS / WENO7-Z weights
//   applied to the primitive point values (left state from the left-biased stencil, right
//   state from the right-biased one).
// Riemann solvers: AUSM+ (riemannSolver_ausmPlus, :397-469), HLLC with Roe-averaged wave
//   speeds (riemannSolver_hllc, :471-590), Roe with the Harten entropy fix
//   (riemannSolver_Roe + compute_half_sum_left_right_flux, :592-746; the fix delta comes from
//   compute_entropy_fix_delta, :269-304), Lax-Friedrichs for air (:748-786).
//
// Every function is templated on the arithmetic type T: double for the plain form, float for
// the mixed form (FP32 reconstruction, fluxes and flux difference; the mixture thermodynamics
// of the reconstructed states stays FP64 because it feeds the temperature; dq stays FP64).
#pragma once
#include <algorithm>
#include "common.cuh"
#include "thermo.cuh"
#include "thermo_2t.cuh"
#include "weno.cuh"
#include "sweep.cuh"
#include "stencil8.cuh"
#include "launch.h"

namespace cb2 {

// A product rounded on its own (never fused into a following add).  The reciprocal-times
// products below feed sums; pinning their rounding keeps every kernel that inlines these solvers
// (the block sweeps, the batched kernels) bitwise identical.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }


template <typename T>
__device__ __forceinline__ T sgn1(T a) { return a < 0 ? T(-1) : T(1); }
template <typename T>
__device__ __forceinline__ T minmod(T a, T b) {
  return T(0.5) * (sgn1(a) + sgn1(b)) * fmin(fabs(a), fabs(b));
}

// Per-variable WENO eps for primitive reconstruction: 1e-40 times the square of the
// variable's reference scale (rho_ref, v_ref, rho_ref v_ref^2, 1 for mass fractions).
__device__ __forceinline__ double pv_eps(const Param &p, int l) {
  double s;
  if (l == 0) s = p.rho_ref;
  else if (l <= 3) s = p.v_ref;
  else if (l == 4) s = p.rho_ref * p.v_ref * p.v_ref;
  else s = 1.0;
  return kWenoEps * s * s;
}

// Node slots: PV[v] (v < NV), then 3 metric comps, J, and (Roe) the entropy-fix delta.
// Reconstructs, from the stencil around node n (slot c, stride st along the sweep), the left
// state at n+1/2 (pl) and the right state at n-1/2 (pr).  Node n+1 supplies the right state of
// the interface n+1/2, so each interface is formed by the thread of its left node.
template <int NS, int REC, typename T>
__device__ __forceinline__ void reconstruct_node(const T *sN, int NN, int c, int st, const Param &p, T *pl,
                                                 T *pr) {
  constexpr int NV = 5 + NS;
#define PV(v, m) sN[(v) * NN + c + (m) * st]
#pragma unroll
  for (int l = 0; l < NV; ++l) {
    if constexpr (REC == 1) {
      pl[l] = pr[l] = PV(l, 0);
    } else if constexpr (REC == 2 || REC == 3) {
      const T v0 = PV(l, 0);
      const T a = v0 - PV(l, -1), b = PV(l, 1) - v0;
      if constexpr (REC == 2) {
        // MUSCL kappa = 1/3 with minmod; minmod is symmetric, so both faces use one slope pair
        const T kappa = T(1.0 / 3.0);
        const T m = minmod(a, b);
        const T d = T(0.25) * ((1 - kappa) * m + (1 + kappa) * m);
        pl[l] = v0 + d;
        pr[l] = v0 - d;
      } else {
        const T d = T(0.5) * minmod(a, b);
        pl[l] = v0 + d;
        pr[l] = v0 - d;
      }
    } else {
      constexpr int W = REC;  // stencil width, node n in the middle
      T v[W];
#pragma unroll
      for (int m = 0; m < W; ++m) v[m] = PV(l, m - W / 2);
      // FP32: eps is raised to 1e-18 times the squared scale so that (eps + beta)^2 of uniform
      // data is a normal FP32 number; like the FP64 eps it only matters where beta ~ 0, where
      // both give the linear weights
      const T eps = sizeof(T) == 4 ? T(pv_eps(p, l) * 1e22) : T(pv_eps(p, l));
      if constexpr (sizeof(T) == 4) {
        if constexpr (REC == 5) weno5_node_x2(v, eps, pl[l], pr[l]);
        else weno7_node_x2(v, eps, pl[l], pr[l]);
      } else if constexpr (REC == 5) {
        weno5_node(v, eps, pl[l], pr[l]);
      } else {
        weno7_node(v, eps, pl[l], pr[l]);
      }
    }
  }
#undef PV
}

// Total energy (index NV) and gamma (index NV+1) of a reconstructed state.  NS counts the
// scalars; with TT (two temperatures) the last one is e_ve: the energy is
// rho (e_k + e_tr(T) + max(e_ve, 0)) and gamma the translational-rotational one
// (src/InviscidScheme.cu:184-211).
template <int NS, typename T, bool TT = false>
__device__ __forceinline__ void state_energy(T *pv, const Mech &m) {
  constexpr int NV = 5 + NS;
  const T ek = T(0.5) * (pv[1] * pv[1] + pv[2] * pv[2] + pv[3] * pv[3]);
  if constexpr (TT) {
    constexpr int NSP = NS - 1;  // species
    double y[NSP], r = 0;
#pragma unroll
    for (int s = 0; s < NSP; ++s) {
      y[s] = double(pv[5 + s]);
      r += y[s] * __ldg(m.gas_const + s);
    }
    const double t = double(pv[4]) / fmax(double(pv[0]) * r, 1e-12);
    double gam, c, etr;
    characteristic_thermo_2t<NSP>(t, y, m, gam, c, nullptr, nullptr, &etr);
    const double eve = fmax(double(pv[5 + NSP]), 0.0);
    pv[NV] = T(double(pv[0]) * (double(ek) + etr + eve));
    pv[NV + 1] = T(gam);
  } else if constexpr (NS == 0) {
    pv[NV] = ek * pv[0] + mul_rn(pv[4], T(1.0 / (kGammaAir - 1)));
    pv[NV + 1] = T(kGammaAir);
  } else if (sizeof(T) == 4 && !m.nasa9) {
    // mixed form: the state's thermodynamics in FP32 (NASA7)
    float y[NS], r = 0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      y[s] = float(pv[5 + s]);
      r += y[s] * float(__ldg(m.gas_const + s));
    }
    const float t = float(pv[4]) / fmaxf(float(pv[0]) * r, 1e-12f);
    float gam, c, etr;
    characteristic_thermo_f32<NS>(t, y, m, gam, c, nullptr, nullptr, &etr);
    pv[NV] = T(float(pv[0]) * (float(ek) + etr));
    pv[NV + 1] = T(gam);
  } else {
    double y[NS], r = 0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      y[s] = double(pv[5 + s]);
      r += y[s] * __ldg(m.gas_const + s);
    }
    const double t = double(pv[4]) / fmax(double(pv[0]) * r, 1e-12);
    double gam, c, etr;
    characteristic_thermo<NS>(t, y, m, gam, c, nullptr, nullptr, &etr);
    pv[NV] = T(double(pv[0]) * (double(ek) + etr));
    pv[NV + 1] = T(gam);
  }
}

template <int NS, typename T>
__device__ __forceinline__ void ausm_plus(const T *pl, const T *pr, const T *ml, const T *mr, T jl, T jr, T *fc) {
  constexpr int NV = 5 + NS;
  const T half = T(0.5);
  const T k1 = half * (jl * ml[0] + jr * mr[0]);
  const T k2 = half * (jl * ml[1] + jr * mr[1]);
  const T k3 = half * (jl * ml[2] + jr * mr[2]);
  const T gk = sqrt(k1 * k1 + k2 * k2 + k3 * k3);
  // one reciprocal each for |grad xi| and c instead of two divisions
  const T igk = T(1) / gk;
  const T ul = mul_rn(k1 * pl[1] + k2 * pl[2] + k3 * pl[3], igk);
  const T ur = mul_rn(k1 * pr[1] + k2 * pr[2] + k3 * pr[3], igk);
  const T c = half * (sqrt(pl[NV + 1] * pl[4] / pl[0]) + sqrt(pr[NV + 1] * pr[4] / pr[0]));
  const T ic = T(1) / c;
  const T Ml = mul_rn(ul, ic), Mr = mul_rn(ur, ic);
  const T alpha = T(3 / 16.0);
  T mlp, plp, mrn, prn;
  // supersonic: M+ = (M + |M|)/2 and P+ = M+/M, which is exactly 1 (M > 1) or 0 (M < -1)
  if (fabs(Ml) > 1) {
    mlp = half * (Ml + fabs(Ml));
    plp = Ml > 0 ? T(1) : T(0);
  } else {
    const T a = (Ml + 1) * (Ml + 1) * T(0.25), b = (Ml * Ml - 1) * (Ml * Ml - 1);
    mlp = a + T(0.125) * b;
    plp = a * (2 - Ml) + alpha * Ml * b;
  }
  if (fabs(Mr) > 1) {
    mrn = half * (Mr - fabs(Mr));
    prn = Mr < 0 ? T(1) : T(0);
  } else {
    const T a = (Mr - 1) * (Mr - 1) * T(0.25), b = (Mr * Mr - 1) * (Mr * Mr - 1);
    mrn = -a - T(0.125) * b;
    prn = a * (2 + Mr) - alpha * Mr * b;
  }
  const T pc = plp * pl[4] + prn * pr[4];
  const T mh = mlp + mrn;
  const T mflux = c * (pl[0] * half * (mh + fabs(mh)) + pr[0] * half * (mh - fabs(mh)));
  const T coeff = mflux * gk;
  const T *pu = mflux >= 0 ? pl : pr;
  fc[0] = coeff;
  fc[1] = coeff * pu[1] + pc * k1;
  fc[2] = coeff * pu[2] + pc * k2;
  fc[3] = coeff * pu[3] + pc * k3;
  fc[4] = coeff * (pu[NV] + pu[4]) / pu[0];
#pragma unroll
  for (int l = 5; l < NV; ++l) fc[l] = coeff * pu[l];
}

template <int NS, typename T, bool TT = false>
__device__ __forceinline__ void hllc(const T *pl, const T *pr, const T *ml, const T *mr, T jl, T jr,
                                     const Mech &mech, T *fc) {
  constexpr int NV = 5 + NS;
  const T half = T(0.5);
  const T sl0 = sqrt(pl[0]), sr0 = sqrt(pr[0]);
  const T isum = T(1) / (sl0 + sr0);
  const T rlc = mul_rn(sl0, isum), rrc = mul_rn(sr0, isum);
  const T ut = pl[1] * rlc + pr[1] * rrc, vt = pl[2] * rlc + pr[2] * rrc, wt = pl[3] * rlc + pr[3] * rrc;
  T ct;
  if constexpr (NS == 0) {
    const T hl = (pl[NV] + pl[4]) / pl[0], hr = (pr[NV] + pr[4]) / pr[0];
    const T ht = hl * rlc + hr * rrc;
    const T ekt = half * (ut * ut + vt * vt + wt * wt);
    ct = sqrt(T(kGammaAir - 1) * (ht - ekt));
  } else if constexpr (TT) {
    // two temperatures: the Roe state's translational-rotational sound speed
    constexpr int NSP = NS - 1;
    double svm[NSP], r = 0;
#pragma unroll
    for (int s = 0; s < NSP; ++s) {
      svm[s] = double(rlc * pl[5 + s] + rrc * pr[5 + s]);
      r += svm[s] * __ldg(mech.gas_const + s);
    }
    const double t = double(rlc * (pl[4] / pl[0]) + rrc * (pr[4] / pr[0])) / fmax(r, 1e-12);
    double gam, c64;
    characteristic_thermo_2t<NSP>(t, svm, mech, gam, c64, nullptr, nullptr);
    ct = T(c64);
  } else if (sizeof(T) == 4 && !mech.nasa9) {
    // mixed form: the Roe state's sound speed in FP32 (NASA7)
    float svm[NS], r = 0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      svm[s] = float(rlc * pl[5 + s] + rrc * pr[5 + s]);
      r += svm[s] * float(__ldg(mech.gas_const + s));
    }
    const float t = float(rlc * (pl[4] / pl[0]) + rrc * (pr[4] / pr[0])) / fmaxf(r, 1e-12f);
    float gam, c32;
    characteristic_thermo_f32<NS>(t, svm, mech, gam, c32, nullptr, nullptr, nullptr);
    ct = T(c32);
  } else {
    double svm[NS], r = 0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      svm[s] = double(rlc * pl[5 + s] + rrc * pr[5 + s]);
      r += svm[s] * __ldg(mech.gas_const + s);
    }
    const double t = double(rlc * (pl[4] / pl[0]) + rrc * (pr[4] / pr[0])) / fmax(r, 1e-12);
    double gam, c64;
    characteristic_thermo<NS>(t, svm, mech, gam, c64, nullptr, nullptr, nullptr);
    ct = T(c64);
  }
  const T kx = half * (ml[0] + mr[0]), ky = half * (ml[1] + mr[1]), kz = half * (ml[2] + mr[2]);
  const T gk = sqrt(kx * kx + ky * ky + kz * kz);
  const T igk = T(1) / gk;
  const T Ut = mul_rn(kx * ut + ky * vt + kz * wt, igk);
  const T ja = half * (jl + jr);
  const T Ul = kx * pl[1] + ky * pl[2] + kz * pl[3];
  const T cl = sqrt(pl[NV + 1] * pl[4] / pl[0]);
  const T Uln = mul_rn(Ul, igk);  // normal velocities
  const T sl = fmin(Uln - cl, Ut - ct);
  if (sl >= 0) {
    const T rU = pl[0] * Ul;
    fc[0] = ja * rU;
    fc[1] = ja * (rU * pl[1] + pl[4] * kx);
    fc[2] = ja * (rU * pl[2] + pl[4] * ky);
    fc[3] = ja * (rU * pl[3] + pl[4] * kz);
    fc[4] = ja * ((pl[NV] + pl[4]) * Ul);
#pragma unroll
    for (int l = 5; l < NV; ++l) fc[l] = ja * rU * pl[l];
    return;
  }
  const T Ur = kx * pr[1] + ky * pr[2] + kz * pr[3];
  const T cr = sqrt(pr[NV + 1] * pr[4] / pr[0]);
  const T Urn = mul_rn(Ur, igk);
  const T sr = fmax(Urn + cr, Ut + ct);
  if (sr < 0) {
    const T rU = pr[0] * Ur;
    fc[0] = ja * rU;
    fc[1] = ja * (rU * pr[1] + pr[4] * kx);
    fc[2] = ja * (rU * pr[2] + pr[4] * ky);
    fc[3] = ja * (rU * pr[3] + pr[4] * kz);
    fc[4] = ja * ((pr[NV] + pr[4]) * Ur);
#pragma unroll
    for (int l = 5; l < NV; ++l) fc[l] = ja * rU * pr[l];
    return;
  }
  const T sm = (mul_rn(pr[0] * Ur * (sr - Urn) - pl[0] * Ul * (sl - Uln), igk) + pl[4] - pr[4]) /
               (pr[0] * (sr - Urn) - pl[0] * (sl - Uln));
  const T pm = pl[0] * (sl - Uln) * (sm - Uln) + pl[4];
  const bool left = sm >= 0;
  const T *ps = left ? pl : pr;
  const T ss = left ? sl : sr, Us = left ? Ul : Ur;
  const T pco = T(1) / (ss - sm);
  const T qco = ja * pco * sm * (ss * gk - Us) * ps[0];
  fc[0] = qco;
  const T dP = (ss * pm - sm * ps[4]) * pco * ja;
  fc[1] = qco * ps[1] + dP * kx;
  fc[2] = qco * ps[2] + dP * ky;
  fc[3] = qco * ps[3] + dP * kz;
  fc[4] = qco * ps[NV] / ps[0] + pco * ja * (ss * pm * sm * gk - sm * ps[4] * Us);
#pragma unroll
  for (int l = 5; l < NV; ++l) fc[l] = qco * ps[l];
}

template <int NS, typename T>
__device__ __forceinline__ void roe_flux(const T *pl, const T *pr, const T *ml, const T *mr, T jl, T jr, T efl,
                                         T efr, const Param &p, T *fc) {
  constexpr int NV = 5 + NS;
  const T half = T(0.5);
  // half sum of the left and right physical fluxes
  {
    T JKx = jl * ml[0], JKy = jl * ml[1], JKz = jl * ml[2];
    T Uk = pl[1] * JKx + pl[2] * JKy + pl[3] * JKz;
    T co = Uk * pl[0];
    fc[0] = half * co;
    fc[1] = half * (co * pl[1] + pl[4] * JKx);
    fc[2] = half * (co * pl[2] + pl[4] * JKy);
    fc[3] = half * (co * pl[3] + pl[4] * JKz);
    fc[4] = half * Uk * (pl[4] + pl[NV]);
#pragma unroll
    for (int l = 5; l < NV; ++l) fc[l] = half * co * pl[l];
    JKx = jr * mr[0]; JKy = jr * mr[1]; JKz = jr * mr[2];
    Uk = pr[1] * JKx + pr[2] * JKy + pr[3] * JKz;
    co = Uk * pr[0];
    fc[0] += half * co;
    fc[1] += half * (co * pr[1] + pr[4] * JKx);
    fc[2] += half * (co * pr[2] + pr[4] * JKy);
    fc[3] += half * (co * pr[3] + pr[4] * JKz);
    fc[4] += half * Uk * (pr[4] + pr[NV]);
#pragma unroll
    for (int l = 5; l < NV; ++l) fc[l] += half * co * pr[l];
  }
  const T dl = sqrt(pl[0]), dr = sqrt(pr[0]);
  const T idn = T(1) / (dl + dr);
  const T u = (dl * pl[1] + dr * pr[1]) * idn, v = (dl * pl[2] + dr * pr[2]) * idn,
          w = (dl * pl[3] + dr * pr[3]) * idn;
  const T ek = half * (u * u + v * v + w * w);
  const T hl = (pl[NV] + pl[4]) / pl[0], hr = (pr[NV] + pr[4]) / pr[0];
  const T h = (dl * hl + dr * hr) * idn;
  T gamma = T(kGammaAir);
  T c = sqrt((gamma - 1) * (h - ek));
  T svm[NS > 0 ? NS : 1], alpha[NS > 0 ? NS : 1], ecoef[NS > 0 ? NS : 1];
  if constexpr (NS > 0) {
    double sv64[NS], r = 0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      svm[s] = (dl * pl[5 + s] + dr * pr[5 + s]) * idn;
      sv64[s] = double(svm[s]);
      r += sv64[s] * __ldg(p.mech.gas_const + s);
    }
    const double t = double((dl * (pl[4] / pl[0]) + dr * (pr[4] / pr[0])) * idn) / fmax(r, 1e-12);
    double g64, c64, a64[NS], e64[NS];
    characteristic_thermo<NS>(t, sv64, p.mech, g64, c64, a64, e64, nullptr);
    gamma = T(g64);
    c = T(c64);
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      alpha[s] = T(a64[s]);
      ecoef[s] = T(e64[s]);
    }
  }
  T kx = half * (ml[0] + mr[0]), ky = half * (ml[1] + mr[1]), kz = half * (ml[2] + mr[2]);
  const T gk = sqrt(kx * kx + ky * ky + kz * kz);
  T Uk = kx * u + ky * v + kz * w;
  T ch[3] = {Uk - gk * c, Uk, Uk + gk * c};
  const T efd = half * (efl + efr);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    ch[a] = fabs(ch[a]);
    if (ch[a] < efd) ch[a] = half * (ch[a] * ch[a] / efd + efd);
  }
  kx /= gk; ky /= gk; kz /= gk; Uk /= gk;
  const T ja = half * (jl + jr);
  T dq[NV];
  dq[0] = ja * (pr[0] - pl[0]);
#pragma unroll
  for (int l = 1; l < NV; ++l) dq[l] = ja * (pr[0] * pr[l] - pl[0] * pl[l]);
  dq[4] = ja * (pr[NV] - pl[NV]);
  T c1 = (gamma - 1) * (ek * dq[0] - u * dq[1] - v * dq[2] - w * dq[3] + dq[4]) / (c * c);
  T c2 = (kx * dq[1] + ky * dq[2] + kz * dq[3] - Uk * dq[0]) / c;
  if constexpr (NS > 0) {
#pragma unroll
    for (int s = 0; s < NS; ++s) c1 += alpha[s] * dq[s + 5];
  }
  T c3 = dq[0] - c1;
  T b[NV];
  {
    T L[NV];
    L[0] = half * (c1 - c2);
    L[1] = kx * c3 - ((kz * v - ky * w) * dq[0] - kz * dq[2] + ky * dq[3]) / c;
    L[2] = ky * c3 - ((kx * w - kz * u) * dq[0] - kx * dq[3] + kz * dq[1]) / c;
    L[3] = kz * c3 - ((ky * u - kx * v) * dq[0] - ky * dq[1] + kx * dq[2]) / c;
    L[4] = half * (c1 + c2);
    if constexpr (NS > 0) {
#pragma unroll
      for (int s = 0; s < NS; ++s) L[s + 5] = dq[s + 5] - svm[s] * dq[0];
    }
    b[0] = -ch[0] * L[0];
#pragma unroll
    for (int l = 1; l < NV; ++l) b[l] = -ch[1] * L[l];
    b[4] = -ch[2] * L[4];
  }
  const T c0 = kx * b[1] + ky * b[2] + kz * b[3];
  c1 = c0 + b[0] + b[4];
  c2 = c * (b[4] - b[0]);
  c3 = 0;
  if constexpr (NS > 0) {
#pragma unroll
    for (int s = 0; s < NS; ++s) c3 += ecoef[s] * b[s + 5];
  }
  fc[0] += half * c1;
  fc[1] += half * (u * c1 + kx * c2 - c * (kz * b[2] - ky * b[3]));
  fc[2] += half * (v * c1 + ky * c2 - c * (kx * b[3] - kz * b[1]));
  fc[3] += half * (w * c1 + kz * c2 - c * (ky * b[1] - kx * b[2]));
  fc[4] += half * (h * c1 + Uk * c2 - c * c * c0 / (gamma - 1) +
                   c * ((kz * v - ky * w) * b[1] + (kx * w - kz * u) * b[2] + (ky * u - kx * v) * b[3]) + c3);
  if constexpr (NS > 0) {
#pragma unroll
    for (int s = 0; s < NS; ++s) fc[5 + s] += half * (b[s + 5] + svm[s] * c1);
  }
}

template <typename T>
__device__ __forceinline__ void lax_friedrichs_air(const T *pl, const T *pr, const T *ml, const T *mr, T jl, T jr,
                                                   T *fc) {
  constexpr int NV = 5;
  const T half = T(0.5);
  const T kx = half * (ml[0] + mr[0]), ky = half * (ml[1] + mr[1]), kz = half * (ml[2] + mr[2]);
  const T gk = sqrt(kx * kx + ky * ky + kz * kz);
  const T Ukl = pl[1] * kx + pl[2] * ky + pl[3] * kz, Ukr = pr[1] * kx + pr[2] * ky + pr[3] * kz;
  const T cl = sqrt(T(kGammaAir) * pl[4] / pl[0]), cr = sqrt(T(kGammaAir) * pr[4] / pr[0]);
  const T sr = fmax(fabs(Ukl) + cl * gk, fabs(Ukr) + cr * gk);
  const T hj = half * half * (jl + jr);
  const T rUl = pl[0] * Ukl, rUr = pr[0] * Ukr;
  fc[0] = (rUl + rUr - sr * (pr[0] - pl[0])) * hj;
  fc[1] = (rUl * pl[1] + rUr * pr[1] + kx * (pl[4] + pr[4]) - sr * (pr[1] * pr[0] - pl[1] * pl[0])) * hj;
  fc[2] = (rUl * pl[2] + rUr * pr[2] + ky * (pl[4] + pr[4]) - sr * (pr[2] * pr[0] - pl[2] * pl[0])) * hj;
  fc[3] = (rUl * pl[3] + rUr * pr[3] + kz * (pl[4] + pr[4]) - sr * (pr[3] * pr[0] - pl[3] * pl[0])) * hj;
  fc[4] = ((pl[NV] + pl[4]) * Ukl + (pr[NV] + pr[4]) * Ukr - sr * (pr[NV] - pl[NV])) * hj;
}

// Half-width of the node-centred reconstruction stencil.
template <int REC>
__host__ __device__ constexpr int pv_half_width() { return REC == 1 ? 0 : (REC <= 3 ? 1 : REC / 2); }

// Shared-memory bytes of one sweep tile.
// VF: the tile also holds the node flux comps 1-4 of the 8th-order viscous terms along the sweep.
template <typename T, int NS, int REC, int SOLVER, bool VF = false>
__host__ __device__ constexpr size_t pv_tile_smem(int dir, int ni = kNI) {
  return sizeof(T) * ((size_t)(5 + NS + 4 + (SOLVER == CB2_INV_ROE ? 1 : 0) + (VF ? 4 : 0)) *
                          (dir == 0 ? (kSweepThreads + 2 * pv_half_width<REC>())
                                    : ni * (kSweepThreads / ni + 2 * pv_half_width<REC>())) +
                      (size_t)(2 * (5 + NS) + 2) * kSweepThreads);
}

// One tile of the sweep: tile (bx, by, bz) of the grid that node_sweep_grid describes, run by a
// CTA of kSweepThreads threads; sN holds the node data [NSLOT][NN], sR the right states
// [NV+2][kSweepThreads], sF the interface fluxes [NV][kSweepThreads].  The tile ends with the
// whole CTA in step, so a CTA may run several tiles back to back.
// VF (air, WENO7): the 8th-order viscous divergence along this direction is taken here too
// (compute_viscous_flux_derivative<8>, src/ViscousScheme.cu:790-834, one direction of it): the
// tile also stages comps 1-4 of this direction's node flux (fFlux / gFlux / hFlux after their
// periodic exchange), and every updated node adds J d8(F) before subtracting its inviscid flux
// difference.  The WENO7 tile's halo of 3 nodes plus the neighbour node covers the +-4 stencil
// of every updated node.
template <typename T, int NS, int DIR, int REC, int SOLVER, int NI = kNI, bool VF = false, bool TT = false>
__device__ __forceinline__ void pv_tile_body(const Zone &z, const Param &p, idx_t run, int bx, int by, int bz,
                                             T *sN, T *sR, T *sF) {
  static_assert(!VF || (REC == 7 && NS == 0 && sizeof(T) == 4),
                "the fused viscous divergence is built for the mixed form's WENO7 air tile");
  constexpr int NV = 5 + NS;
  constexpr int RH = pv_half_width<REC>();
  constexpr int NSW = kSweepThreads / NI;  // y/z tile: nodes along the sweep
  constexpr int NN = DIR == 0 ? (kSweepThreads + 2 * RH) : NI * (NSW + 2 * RH);
  const int tid = threadIdx.x;
  const int g = z.ngg;
  const Layout &L = z.L;
  const idx_t sz = L.sz;

  constexpr int NSB = NV + 4 + (SOLVER == CB2_INV_ROE ? 1 : 0);  // first node-flux slot (VF)
  auto put = [&](int idx, const double *src) { sN[idx] = T(*src); };
  auto load = [&](idx_t gi, int slot, int i, int j, int k) {
    if constexpr (VF) {
      if constexpr (sizeof(T) == 4) {
        const float *FL = DIR == 0 ? z.fF32 : (DIR == 1 ? z.gF32 : z.hF32);
#pragma unroll
        for (int c = 0; c < 4; ++c) sN[(NSB + c) * NN + slot] = FL[gi + (c + 1) * sz];
      } else {
        const double *FL = DIR == 0 ? z.fF : (DIR == 1 ? z.gF : z.hF);
#pragma unroll
        for (int c = 0; c < 4; ++c) sN[(NSB + c) * NN + slot] = FL[gi + (c + 1) * sz];
      }
    }
    if constexpr (sizeof(T) == 4) {
      // mixed form: the FP32 copies of bv, the metric and J
#pragma unroll
      for (int l = 0; l < 5; ++l) sN[l * NN + slot] = z.bv32[gi + l * sz];
#pragma unroll
      for (int c = 0; c < 3; ++c) sN[(NV + c) * NN + slot] = z.met32[gi + (3 * DIR + c) * sz];
      sN[(NV + 3) * NN + slot] = z.met32[gi + 9 * sz];
    } else {
#pragma unroll
      for (int l = 0; l < 5; ++l) put(l * NN + slot, z.bv + gi + l * sz);
#pragma unroll
      for (int c = 0; c < 3; ++c) put((NV + c) * NN + slot, z.metric + gi + (3 * DIR + c) * sz);
      put((NV + 3) * NN + slot, z.jac + gi);
    }
#pragma unroll
    for (int s = 0; s < NS; ++s) put((5 + s) * NN + slot, z.sv + gi + s * sz);
    if constexpr (SOLVER == CB2_INV_ROE) {
      // entropy-fix delta exists on [-1, m] only (ghost width 1)
      const bool in1 = i >= -1 && i <= z.mx && j >= -1 && j <= z.my && k >= -1 && k <= z.mz;
      if (in1) put((NV + 4) * NN + slot, z.efd + z.L1.at(i, j, k));
      else sN[(NV + 4) * NN + slot] = T(0);
    }
  };

  // Thread tid owns node n.  rec: n lies in [-1, m] along the sweep (both of its faces are
  // needed); face: the interface n+1/2 is an interior face, i.e. n in [-1, m-1], and node n+1
  // belongs to this CTA; upd: n in [0, m-1] is updated from the faces n-1/2 and n+1/2.
  int i, j, k, n, ms, tpos;
  bool inside;
  int c, st;
  if constexpr (DIR == 0) {
    // positions along the run of one k plane (q = j disp2 + i + g) fit in 32 bits: a plane
    // holds far fewer than 2^31 nodes, and 32-bit division is several times cheaper
    k = bz;
    const int d2 = (int)L.disp2;
    const int q0 = bx * (kSweepThreads - 2) - 1;
    const idx_t base = (idx_t)k * L.disp1 + L.dispt - g;
    const int qlo = q0 - RH;
    const int qmin = -L.gj * d2, qmax = (L.my + L.gj) * d2;
    for (int s = tid; s < NN; s += kSweepThreads) {
      const int q = qlo + s;
      if (q >= qmin && q < qmax) {
        const int jj = q >= 0 ? q / d2 : -((-q + d2 - 1) / d2);
        load(base + q, s, q - jj * d2 - g, jj, k);
      }
    }
    const int q = q0 + tid;
    const int jj = q >= 0 ? q / d2 : -1;
    i = q - jj * d2 - g;
    j = jj;
    n = i;
    ms = L.mx;
    inside = q >= 0 && q < run;
    tpos = tid;
    c = tid + RH;
    st = 1;
  } else {
    const int ti = tid % NI, ts = tid / NI;
    i = bx * NI + ti;
    const int s0 = by * (NSW - 2) - 1;
    ms = DIR == 1 ? L.my : L.mz;
    if (DIR == 1) k = bz; else j = bz;
    for (int s = ts; s < NSW + 2 * RH; s += NSW) {
      const int nn = s0 - RH + s;
      if (i < L.mx && nn < ms + g) {
        if (DIR == 1) load(L.at(i, nn, k), s * NI + ti, i, nn, k);
        else load(L.at(i, j, nn), s * NI + ti, i, j, nn);
      }
    }
    n = s0 + ts;
    if (DIR == 1) j = n; else k = n;
    inside = i < L.mx;
    tpos = ts;
    c = (ts + RH) * NI + ti;
    st = NI;
  }
  const bool rec = inside && n >= -1 && n <= ms;
  const bool face = rec && n <= ms - 1 && tpos < (DIR == 0 ? kSweepThreads : NSW) - 1;
  const bool upd = face && n >= 0 && tpos >= 1;
  __syncthreads();

  T pl[NV + 2];
  if (rec) {
    T pr[NV + 2];
    reconstruct_node<NS, REC>(sN, NN, c, st, p, pl, pr);
    state_energy<NS, T, TT>(pl, p.mech);
    state_energy<NS, T, TT>(pr, p.mech);
#pragma unroll
    for (int v = 0; v < NV + 2; ++v) sR[v * kSweepThreads + tid] = pr[v];
  }
  __syncthreads();

  if (face) {
    const int tn = tid + st;  // the thread of node n+1 (st is 1 or NI, as the thread layout)
    T pr[NV + 2];
#pragma unroll
    for (int v = 0; v < NV + 2; ++v) pr[v] = sR[v * kSweepThreads + tn];
    const T ml[3] = {sN[NV * NN + c], sN[(NV + 1) * NN + c], sN[(NV + 2) * NN + c]};
    const T mr[3] = {sN[NV * NN + c + st], sN[(NV + 1) * NN + c + st], sN[(NV + 2) * NN + c + st]};
    const T jl = sN[(NV + 3) * NN + c], jr = sN[(NV + 3) * NN + c + st];
    T fc[NV];
    if constexpr (SOLVER == CB2_INV_AUSMP) ausm_plus<NS>(pl, pr, ml, mr, jl, jr, fc);
    else if constexpr (SOLVER == CB2_INV_HLLC) hllc<NS, T, TT>(pl, pr, ml, mr, jl, jr, p.mech, fc);
    else if constexpr (SOLVER == CB2_INV_ROE)
      roe_flux<NS>(pl, pr, ml, mr, jl, jr, sN[(NV + 4) * NN + c], sN[(NV + 4) * NN + c + st], p, fc);
    else lax_friedrichs_air(pl, pr, ml, mr, jl, jr, fc);
#pragma unroll
    for (int v = 0; v < NV; ++v) sF[v * kSweepThreads + tid] = fc[v];
  }
  __syncthreads();

  if (upd) {
    const int tprev = tid - st;
    const idx_t gd = z.L0.at(i, j, k);
    const idx_t sz0 = z.L0.sz;
    if constexpr (VF) {
      // physical-boundary closures of the stencil along this direction
      bool bl, br;
      if (DIR == 0) {
        bl = z.bt.il[j + k * z.my] != 0;
        br = z.bt.ir[j + k * z.my] != 0;
      } else if (DIR == 1) {
        bl = z.bt.jl[i + k * z.mx] != 0;
        br = z.bt.jr[i + k * z.mx] != 0;
      } else {
        bl = z.bt.kl[i + j * z.mx] != 0;
        br = z.bt.kr[i + j * z.mx] != 0;
      }
      const T jac = sN[(NV + 3) * NN + c];
      const bool first = DIR == 0 && p.visc8_fused == 2;
      const double d0 = double(sF[tid] - sF[tprev]);
      if (first) z.dq[gd] = -d0;
      else z.dq[gd] -= d0;
#pragma unroll
      for (int v = 1; v < 5; ++v) {
        const T *Fv = sN + (NSB + v - 1) * NN + c;
        const T dv = d8<T>([&](int m) { return Fv[m * st]; }, n, ms, bl, br);
        const double inv = double(sF[v * kSweepThreads + tid] - sF[v * kSweepThreads + tprev]);
        const double vis = double(dv * jac);
        if (first) z.dq[gd + v * sz0] = vis - inv;
        else z.dq[gd + v * sz0] = (z.dq[gd + v * sz0] + vis) - inv;
      }
    } else {
#pragma unroll
      for (int v = 0; v < NV; ++v)
        z.dq[gd + v * sz0] -= double(sF[v * kSweepThreads + tid] - sF[v * kSweepThreads + tprev]);
    }
  }
  __syncthreads();
}

// One whole tile with pv_tile_smem bytes at pv_smem.
template <typename T, int NS, int DIR, int REC, int SOLVER, int NI = kNI, bool VF = false, bool TT = false>
__device__ __forceinline__ void pv_tile(const Zone &z, const Param &p, idx_t run, int bx, int by, int bz,
                                        unsigned char *pv_smem) {
  constexpr int NV = 5 + NS;
  constexpr int RH = pv_half_width<REC>();
  constexpr int NN = DIR == 0 ? (kSweepThreads + 2 * RH) : NI * (kSweepThreads / NI + 2 * RH);
  constexpr int NSLOT = NV + 4 + (SOLVER == CB2_INV_ROE ? 1 : 0) + (VF ? 4 : 0);
  T *sN = reinterpret_cast<T *>(pv_smem);
  T *sR = sN + NSLOT * NN;
  T *sF = sR + (NV + 2) * kSweepThreads;
  pv_tile_body<T, NS, DIR, REC, SOLVER, NI, VF, TT>(z, p, run, bx, by, bz, sN, sR, sF);
}

template <typename T, int NS, int DIR, int REC, int SOLVER, int NI = kNI, bool VF = false, bool TT = false>
__global__ void __launch_bounds__(kSweepThreads) k_inviscid_pv(Zone z, Param p, idx_t run) {
  extern __shared__ __align__(16) unsigned char pv_smem[];
  pv_tile<T, NS, DIR, REC, SOLVER, NI, VF, TT>(z, p, run, blockIdx.x, blockIdx.y, blockIdx.z, pv_smem);
}

// The mixed form's mixture sweeps, held to 128 registers (two CTAs per SM): with the FP32 state
// thermodynamics the y/z tiles would otherwise take 170 and run one CTA per SM.
template <typename T, int NS, int DIR, int REC, int SOLVER, int NI = kNI, bool VF = false>
__global__ void __launch_bounds__(kSweepThreads, 2) k_inviscid_pv_mb2(Zone z, Param p, idx_t run) {
  extern __shared__ __align__(16) unsigned char pv_smem[];
  pv_tile<T, NS, DIR, REC, SOLVER, NI, VF>(z, p, run, blockIdx.x, blockIdx.y, blockIdx.z, pv_smem);
}

template <typename T, int NS, int DIR, int REC, int SOLVER, int NI, bool VF, bool TT = false>
constexpr auto pv_kernel() {
  if constexpr (sizeof(T) == 4 && NS > 0) return k_inviscid_pv_mb2<T, NS, DIR, REC, SOLVER, NI, VF>;
  else return k_inviscid_pv<T, NS, DIR, REC, SOLVER, NI, VF, TT>;
}

// Entropy-fix delta of the Roe scheme on [-1, m] in every direction (ghost width 1), FP64.
template <int NS>
__global__ void k_entropy_fix_delta(Zone z, Param p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x - 1, j = blockIdx.y - 1, k = blockIdx.z - 1;
  if (i > z.mx) return;
  const idx_t g = z.L.at(i, j, k), sz = z.L.sz;
  const double *M = z.metric + g;
  const double u = z.bv[g + sz], v = z.bv[g + 2 * sz], w = z.bv[g + 3 * sz];
  const double U = fabs(u * M[0] + v * M[sz] + w * M[2 * sz]);
  const double V = fabs(u * M[3 * sz] + v * M[4 * sz] + w * M[5 * sz]);
  const double W = fabs(u * M[6 * sz] + v * M[7 * sz] + w * M[8 * sz]);
  const double kx = norm3d(M[0], M[sz], M[2 * sz]);
  const double ky = norm3d(M[3 * sz], M[4 * sz], M[5 * sz]);
  const double kz = norm3d(M[6 * sz], M[7 * sz], M[8 * sz]);
  double a;
  if constexpr (NS == 0) a = sqrt(kGammaAir * z.bv[g + 4 * sz] / z.bv[g]);
  else a = z.acoustic[g];
  double d;
  if (p.dim == 2) d = p.entropy_fix_factor * (U + V + a * 0.5 * (kx + ky));
  else d = p.entropy_fix_factor * (U + V + W + a * (kx + ky + kz) / 3.0);
  z.efd[z.L1.at(i, j, k)] = d;
}

template <typename T, int NS, int DIR, int REC, int SOLVER, int NI, bool VF = false, bool TT = false>
static int launch_pv_yz(const Zone &z, const Param &p, cudaStream_t s) {
  SweepGeom geo;
  const dim3 grid = node_sweep_grid(DIR, z.L, geo, NI);
  const size_t smem = pv_tile_smem<T, NS, REC, SOLVER, VF>(DIR, NI);
  auto kern = pv_kernel<T, NS, DIR, REC, SOLVER, NI, VF, TT>();
  CB2_TRY(prepare_smem(kern, smem));
  kern<<<grid, kSweepThreads, smem, s>>>(z, p, 0);
  return check_launch();
}

// y/z sweep with the block's tile width: the autotuned widths exist for the WENO5/7 air sweeps
// (the bench's kernels); every other combination uses kNI.
template <typename T, int NS, int DIR, int REC, int SOLVER, bool VF = false, bool TT = false>
static int launch_pv_yz_ni(const Zone &z, const Param &p, cudaStream_t s) {
  if constexpr ((REC == 5 || REC == 7) && NS == 0) {
    const int ni = z.tile_ni[DIR];
    if (ni == 4) return launch_pv_yz<T, NS, DIR, REC, SOLVER, 4, VF>(z, p, s);
    if (ni == 16) return launch_pv_yz<T, NS, DIR, REC, SOLVER, 16, VF>(z, p, s);
  }
  return launch_pv_yz<T, NS, DIR, REC, SOLVER, kNI, VF, TT>(z, p, s);
}

template <typename T, int NS, int REC, int SOLVER, bool VF, bool TT = false>
static int launch_pv_dir(int d, const Zone &z, const Param &p, cudaStream_t s) {
  if (d == 0) {
    SweepGeom geo;
    const dim3 grid = node_sweep_grid(0, z.L, geo);
    const size_t smem = pv_tile_smem<T, NS, REC, SOLVER, VF>(0);
    auto kern = pv_kernel<T, NS, 0, REC, SOLVER, kNI, VF, TT>();
    CB2_TRY(prepare_smem(kern, smem));
    kern<<<grid, kSweepThreads, smem, s>>>(z, p, geo.run);
    return check_launch();
  }
  if (d == 1) return launch_pv_yz_ni<T, NS, 1, REC, SOLVER, VF, TT>(z, p, s);
  return launch_pv_yz_ni<T, NS, 2, REC, SOLVER, VF, TT>(z, p, s);
}

// NS counts the scalars of sv; TT: two temperatures (the last scalar is e_ve)
template <typename T, int NS, int REC, int SOLVER, bool TT = false>
static int launch_pv_dirs(const Zone &z, const Param &p, cudaStream_t s, int &nl) {
  if (SOLVER == CB2_INV_ROE) {
    dim3 grid((z.mx + 2 + 127) / 128, z.my + 2, z.mz + 2);
    ProfScope prof("entropy_fix_delta", s);
    k_entropy_fix_delta<NS><<<grid, 128, 0, s>>>(z, p);
    ++nl;
    CB2_TRY(check_launch());
  }
  const int ndir = z.mz > 1 ? 3 : 2;
  for (int d = 0; d < ndir; ++d) {
    if (z.sweep_mask && !(z.sweep_mask & (1u << d))) continue;
    static const char *names[3] = {"pv_flux_x", "pv_flux_y", "pv_flux_z"};
    ProfScope prof(names[d], s);
    if constexpr (REC == 7 && NS == 0 && sizeof(T) == 4) {
      if (p.visc8_fused) CB2_TRY((launch_pv_dir<T, NS, REC, SOLVER, true>(d, z, p, s)));
      else CB2_TRY((launch_pv_dir<T, NS, REC, SOLVER, false>(d, z, p, s)));
    } else {
      if (p.visc8_fused) return CB2_ERR_UNSUPPORTED;
      CB2_TRY((launch_pv_dir<T, NS, REC, SOLVER, false, TT>(d, z, p, s)));
    }
    ++nl;
  }
  return CB2_OK;
}

}  // namespace cb2
