// SSP-RK3 stage update with primitive recovery (update_cv_and_bv_rk<mix>,
// src/RK.cuh:277-367; compute_temperature_and_pressure, src/FieldOperation.cu:4-94) and the
// conservative-from-primitive fill (compute_cv_from_bv<mix>, src/FieldOperation.cuh:90-161).
//
// One thread per node, i fastest, so every array access of a warp is one contiguous run.
#include "point.cuh"
#include "launch.h"

namespace cb2 {

constexpr int kPtThreads = 128;

template <int NS, bool TT>
__global__ void __launch_bounds__(kPtThreads) k_stage_update(Zone z, Param p, double dt, int rk) {
  const int i = blockIdx.x * kPtThreads + threadIdx.x;
  const int j = blockIdx.y, k = blockIdx.z;
  if (i >= z.mx) return;
  stage_update_point<NS, TT>(z, p, step_dt(p, dt), rk, i, j, k);
}

// VT relaxation of every interior node over dt_scale x the step's dt (apply_vt_relaxation_rk,
// src/RK.cuh:20-28; dt_stage = rk_stage_dt_scale[rk] * dt, :91, 202).
template <int NS>
__global__ void __launch_bounds__(kPtThreads) k_vt_relaxation(Zone z, Param p, double dt, double dt_scale) {
  const int i = blockIdx.x * kPtThreads + threadIdx.x;
  const int j = blockIdx.y, k = blockIdx.z;
  if (i >= z.mx) return;
  vt_relax_point<NS>(z, p, z.L.at(i, j, k), dt_scale * step_dt(p, dt));
}

template <int NS>
__global__ void __launch_bounds__(kPtThreads) k_cv_from_bv(Zone z, Param p) {
  const int g_ = z.ngg;
  const int i = blockIdx.x * kPtThreads + threadIdx.x - g_;
  const int j = blockIdx.y - g_, k = blockIdx.z - g_;
  if (i >= z.mx + g_) return;
  cv_point<NS>(z, p, z.L.at(i, j, k));
}

// ---- limit_flow (src/TimeAdvanceFunc.cuh:129-232) --------------------------------------------
// A node is bad when one of rho, u, v, w, p is NaN or outside its bounds; a bad node takes the
// mean of the good nodes of its 3x3x3 neighbourhood inside the block (its own clamped values if
// there are none), then T from the gas law and cv.  The reference does this in place in one
// kernel, where a neighbour already replaced by another thread may or may not count as good;
// here pass 1 reads only the values left by the stage update and parks the means in dq (free
// until the next right-hand side), and pass 2 writes them, so the result does not depend on
// thread timing.
__device__ __forceinline__ bool lf_bad(const Zone &z, const Param &p, idx_t g) {
  const idx_t sz = z.L.sz;
#pragma unroll
  for (int l = 0; l < 5; ++l) {
    const double v = z.bv[g + l * sz];
    if (isnan(v) || v < p.lf_ll[l] || v > p.lf_ul[l]) return true;
  }
  return false;
}

__global__ void __launch_bounds__(kPtThreads) k_limit_flow_mean(Zone z, Param p) {
  const int i = blockIdx.x * kPtThreads + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  if (i >= z.mx) return;
  const idx_t g = z.L.at(i, j, k), sz = z.L.sz;
  if (!lf_bad(z, p, g)) return;
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
        const idx_t gn = z.L.at(i1, j1, k1);
        if (lf_bad(z, p, gn)) continue;
#pragma unroll
        for (int l = 0; l < 5; ++l) v[l] += z.bv[gn + l * sz];
        ++kn;
      }
    }
  }
  if (kn > 0) {
    const double inv = 1.0 / kn;
#pragma unroll
    for (int l = 0; l < 5; ++l) v[l] *= inv;
  } else {
#pragma unroll
    for (int l = 0; l < 5; ++l) v[l] = fmin(fmax(z.bv[g + l * sz], p.lf_ll[l]), p.lf_ul[l]);
  }
  const idx_t g0 = z.L0.at(i, j, k), sz0 = z.L0.sz;
#pragma unroll
  for (int l = 0; l < 5; ++l) z.dq[g0 + l * sz0] = v[l];
}

template <int NS>
__global__ void __launch_bounds__(kPtThreads) k_limit_flow_apply(Zone z, Param p) {
  const int i = blockIdx.x * kPtThreads + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  if (i >= z.mx) return;
  const idx_t g = z.L.at(i, j, k), sz = z.L.sz;
  if (!lf_bad(z, p, g)) return;
  const idx_t g0 = z.L0.at(i, j, k), sz0 = z.L0.sz;
#pragma unroll
  for (int l = 0; l < 5; ++l) z.bv[g + l * sz] = z.dq[g0 + l * sz0];
  const double rho = z.bv[g], pr = z.bv[g + 4 * sz];
  if constexpr (NS == 0) {
    z.bv[g + 5 * sz] = pr * kMwAir / (rho * kRu);
  } else {
    double r = 0;
#pragma unroll
    for (int s = 0; s < NS; ++s) r += z.sv[g + s * sz] * __ldg(p.mech.gas_const + s);
    z.bv[g + 5 * sz] = pr / (rho * r);
  }
  cv_point<NS>(z, p, g);
}

template <int NS>
static int launch_vt_ns(const Zone &z, const Param &p, double dt, double dt_scale, cudaStream_t s, int &nl) {
  if (!p.mech.enable_vt) return CB2_OK;
  dim3 grid((z.mx + kPtThreads - 1) / kPtThreads, z.my, z.mz);
  ProfScope prof("vt_relaxation", s);
  k_vt_relaxation<NS><<<grid, kPtThreads, 0, s>>>(z, p, dt, dt_scale);
  ++nl;
  return check_launch();
}

template <int NS>
static int launch_update_ns(const Zone &z, const Param &p, double dt, int rk, cudaStream_t s, int &nl) {
  dim3 grid((z.mx + kPtThreads - 1) / kPtThreads, z.my, z.mz);
  const bool tt = p.i_eve >= 0;
  {
    ProfScope prof("stage_update", s);
    if constexpr (NS > 0) {
      if (tt) k_stage_update<NS, true><<<grid, kPtThreads, 0, s>>>(z, p, dt, rk);
      else k_stage_update<NS, false><<<grid, kPtThreads, 0, s>>>(z, p, dt, rk);
    } else {
      k_stage_update<NS, false><<<grid, kPtThreads, 0, s>>>(z, p, dt, rk);
    }
  }
  CB2_TRY(check_launch());
  if constexpr (NS > 0) {
    // the stage's VT relaxation follows its update and precedes limit_flow (src/RK.cuh:198-207)
    if (tt) {
      double a, b, c;
      ssprk3_coeff(rk, a, b, c);
      CB2_TRY(launch_vt_ns<NS>(z, p, dt, c, s, nl));
    }
  }
  if (p.limit_flow) {
    ProfScope prof("limit_flow", s);
    k_limit_flow_mean<<<grid, kPtThreads, 0, s>>>(z, p);
    k_limit_flow_apply<NS><<<grid, kPtThreads, 0, s>>>(z, p);
    nl += 2;
    CB2_TRY(check_launch());
  }
  return CB2_OK;
}

int launch_stage_update(const Zone &z, const Param &p, double dt, int rk, cudaStream_t s, int &n_launch) {
  ++n_launch;
  switch (p.n_spec) {
    case 0: return launch_update_ns<0>(z, p, dt, rk, s, n_launch);
    case 5: return launch_update_ns<5>(z, p, dt, rk, s, n_launch);
    case 9: return launch_update_ns<9>(z, p, dt, rk, s, n_launch);
    default: return CB2_ERR_UNSUPPORTED;
  }
}

int launch_vt_relaxation(const Zone &z, const Param &p, double dt_stage, cudaStream_t s, int &n_launch) {
  if (p.i_eve < 0) return CB2_ERR_UNSUPPORTED;
  switch (p.n_spec) {
    case 5: return launch_vt_ns<5>(z, p, dt_stage, 1.0, s, n_launch);
    case 9: return launch_vt_ns<9>(z, p, dt_stage, 1.0, s, n_launch);
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
