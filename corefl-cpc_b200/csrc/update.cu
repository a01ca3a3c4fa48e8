// SSP-RK3 stage update with primitive recovery (update_cv_and_bv_rk<mix>,
// src/RK.cuh:277-367; compute_temperature_and_pressure, src/FieldOperation.cu:4-94) and the
// conservative-from-primitive fill (compute_cv_from_bv<mix>, src/FieldOperation.cuh:90-161).
//
// One thread per node, i fastest, so every array access of a warp is one contiguous run.
#include "point.cuh"
#include "launch.h"

namespace cb2 {

constexpr int kPtThreads = 128;

template <int NS>
__global__ void __launch_bounds__(kPtThreads) k_stage_update(Zone z, Param p, double dt, int rk) {
  const int i = blockIdx.x * kPtThreads + threadIdx.x;
  const int j = blockIdx.y, k = blockIdx.z;
  if (i >= z.mx) return;
  stage_update_point<NS>(z, p, dt, rk, i, j, k);
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
