// SSP-RK3 stage update with primitive recovery (update_cv_and_bv_rk<mix>,
// src/RK.cuh:277-367; compute_temperature_and_pressure, src/FieldOperation.cu:4-94) and the
// conservative-from-primitive fill (compute_cv_from_bv<mix>, src/FieldOperation.cuh:90-161).
//
// One thread per node, i fastest, so every array access of a warp is one contiguous run.
#include "common.cuh"
#include "thermo.cuh"
#include "launch.h"

namespace cb2 {

constexpr int kPtThreads = 128;

// Newton inversion of T from the internal energy e (1T mixtures): stops at |1 - T1/T| <= 1e-5
// or after 1000 iterations, starting from the previous temperature (src/FieldOperation.cu:67-85).
template <int NS>
__device__ __forceinline__ double newton_temperature(double e, const double *y, double r_mix, double t,
                                                     const Mech &m) {
  double err = 1;
  int iter = 0;
  double h[NS], cp[NS];
  while (err > 1e-5 && iter++ < 1000) {
    nasa7_h_cp<NS>(t, m, h, cp);
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

template <int NS>
__global__ void __launch_bounds__(kPtThreads) k_stage_update(Zone z, Param p, double dt, int rk) {
  const int i = blockIdx.x * kPtThreads + threadIdx.x;
  const int j = blockIdx.y, k = blockIdx.z;
  if (i >= z.mx) return;
  constexpr int NV = 5 + NS;
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
    sum = 1.0 / sum;
    const double scale = rho * sum;
    double y[NS], r_mix = 0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      y[s] = q[5 + s] * sum;
      q[5 + s] *= scale;
      z.sv[g + s * sz] = y[s];
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

template <int NS>
__global__ void __launch_bounds__(kPtThreads) k_cv_from_bv(Zone z, Param p) {
  const int g_ = z.ngg;
  const int i = blockIdx.x * kPtThreads + threadIdx.x - g_;
  const int j = blockIdx.y - g_, k = blockIdx.z - g_;
  if (i >= z.mx + g_) return;
  const idx_t g = z.L.at(i, j, k), sz = z.L.sz;
  const double rho = z.bv[g], u = z.bv[g + sz], v = z.bv[g + 2 * sz], w = z.bv[g + 3 * sz];
  const double pr = z.bv[g + 4 * sz];
  z.cv[g] = rho;
  z.cv[g + sz] = rho * u;
  z.cv[g + 2 * sz] = rho * v;
  z.cv[g + 3 * sz] = rho * w;
  double E = 0.5 * (u * u + v * v + w * w);
  if constexpr (NS == 0) {
    E *= rho;
    E += pr / (kGammaAir - 1);
  } else {
    double h[NS];
    nasa7_h<NS>(z.bv[g + 5 * sz], p.mech, h);
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const double y = z.sv[g + s * sz];
      z.cv[g + (5 + s) * sz] = rho * y;
      E += h[s] * y;
    }
    E *= rho;
    E -= pr;
  }
  z.cv[g + 4 * sz] = E;
}

template <int NS>
static int launch_update_ns(const Zone &z, const Param &p, double dt, int rk, cudaStream_t s) {
  dim3 grid((z.mx + kPtThreads - 1) / kPtThreads, z.my, z.mz);
  ProfScope prof("stage_update", s);
  k_stage_update<NS><<<grid, kPtThreads, 0, s>>>(z, p, dt, rk);
  return check_launch();
}

int launch_stage_update(const Zone &z, const Param &p, double dt, int rk, cudaStream_t s, int &n_launch) {
  ++n_launch;
  switch (p.n_spec) {
    case 0: return launch_update_ns<0>(z, p, dt, rk, s);
    case 5: return launch_update_ns<5>(z, p, dt, rk, s);
    case 9: return launch_update_ns<9>(z, p, dt, rk, s);
    default: return CB2_ERR_UNSUPPORTED;
  }
}

int launch_cv_from_bv(const Zone &z, const Param &p, cudaStream_t s, int &n_launch) {
  ++n_launch;
  const int g = z.ngg;
  dim3 grid((z.mx + 2 * g + kPtThreads - 1) / kPtThreads, z.my + 2 * g, z.mz + 2 * g);
  ProfScope prof("cv_from_bv", s);
  switch (p.n_spec) {
    case 0: k_cv_from_bv<0><<<grid, kPtThreads, 0, s>>>(z, p); break;
    case 5: k_cv_from_bv<5><<<grid, kPtThreads, 0, s>>>(z, p); break;
    case 9: k_cv_from_bv<9><<<grid, kPtThreads, 0, s>>>(z, p); break;
    default: return CB2_ERR_UNSUPPORTED;
  }
  return check_launch();
}

}  // namespace cb2
