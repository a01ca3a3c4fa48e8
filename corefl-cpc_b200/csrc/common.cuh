// Device-side data model shared by all kernels of the library.
//
// The field arrays are the caller's: padded SoA FP64 arrays in the layout of
// ggxl::VectorField3D<real> (src/gxl_lib/Array.cuh:307-328).  A `Layout` holds the
// displacements of one ghost width; `Zone` is passed to every kernel by value.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include "cb200.h"

namespace cb2 {

// Physical constants (src/Constants.h:11-36).
constexpr double kRu = 8314.462618;       // J/(kmol K)
constexpr double kRc = 1.98720425864083;  // cal/(mol K)
constexpr double kGammaAir = 1.4;
constexpr double kMwAir = 28.9647;
constexpr double kRAir = kRu / kMwAir;
constexpr double kPatm = 101325.0;
constexpr double kWenoEps = 1e-40;         // src/WENO.cu:8

constexpr int kMaxSpec = 9;   // MAX_SPEC_NUMBER of the reference build (CMakeLists.txt:17)
constexpr int kMaxReac = 20;
constexpr int kMaxVar = 5 + kMaxSpec + 1;

typedef long long idx_t;

struct Layout {
  int mx, my, mz, g;
  int gj;  // ghost layers stored along j (g for a block layout, 0 for a compact 1-D case)
  idx_t disp2, disp1, dispt, sz;
  __host__ __device__ __forceinline__ idx_t at(int i, int j, int k) const {
    return (idx_t)k * disp1 + (idx_t)j * disp2 + i + dispt;
  }
};

inline Layout make_layout(int mx, int my, int mz, int g) {
  Layout L;
  L.mx = mx; L.my = my; L.mz = mz; L.g = g; L.gj = g;
  L.disp2 = mx + 2 * g;
  L.disp1 = (idx_t)(my + 2 * g) * L.disp2;
  L.dispt = (L.disp1 + L.disp2 + 1) * g;
  L.sz = (idx_t)(mx + 2 * g) * (my + 2 * g) * (mz + 2 * g);
  return L;
}

// A 1-D case stored without ghost rows or planes: only the g ghost nodes at each end of the
// single i-line (the batched cases use it; at(i, 0, 0) = i + g).
inline Layout make_layout_1d(int mx, int g) {
  Layout L;
  L.mx = mx; L.my = 1; L.mz = 1; L.g = g; L.gj = 0;
  L.disp2 = mx + 2 * g;
  L.disp1 = L.disp2;
  L.dispt = g;
  L.sz = L.disp2;
  return L;
}

// Per-face physical-boundary flags, one int per face node (bType_il..kr of DZone,
// src/Field.h:20, filled as src/Mesh.cpp:855-900 does): 0 = inner or periodic.
struct BTypes {
  const int *il, *ir, *jl, *jr, *kl, *kr;  // (my,mz), (my,mz), (mx,mz), (mx,mz), (mx,my), (mx,my)
};

struct Zone {
  int mx, my, mz, ngg;
  Layout L;   // ghost ngg
  Layout L0;  // ghost 0 (dq, dt_local)
  Layout L1;  // ghost 1 (vis_flux, entropy_fix_delta)
  double *cv, *bv, *sv, *qn, *dq, *metric, *jac, *mul, *kappa, *rhoD, *acoustic, *gamma, *mach;
  double *fF, *gF, *hF, *visf, *shock, *dtl, *rts, *efd;
  double *tve;  // two-temperature: T_ve, ghost ngg
  double *kappa_ve;  // two-temperature: vibrational-electronic conductivity, ghost ngg
  // mixed form: FP32 copies the FP32 kernels read instead of the FP64 arrays (private scratch,
  // same padded layout): bv (6 comps, refreshed at the start of every residual) and the
  // metric (9 comps) followed by J, taken when the block is bound
  float *bv32, *met32;
  float *fF32, *gF32, *hF32;  // mixed form: 8th-order viscous node fluxes (n_var comps, ghost ngg)
  BTypes bt;
  int tile_ni[3];       // i-columns of the y/z sweep tiles (0: the default), set by the autotuner
  unsigned sweep_mask;  // primitive sweeps to run (bit d: direction d; 0: all)
};

// Mechanism tables in device memory (copied from cb2_mechanism by cb2_init).
struct Mech {
  int n_spec, n_reac;
  const double *imw, *gas_const, *mw;
  const double *lo, *hi;         // [n_spec*7]
  const double *t_low, *t_mid, *t_high;
  const double *geometry, *lj_inv, *vis_coeff;
  const double *wjwi14, *sqwiwj8, *bdc, *kbe;  // [n_spec*n_spec]
  const double *ln_kbe, *ln_lj_inv;            // ln of kbe and lj_inv (transport_ln = 1)
  int transport_ln;
  double ln_temp_p;  // ln(p_atm / R_u * 1e-3): the equilibrium constant's (p_atm / (R_u T))^order
  const double *zrot;
  const int *reac_type, *rev_type, *stoi_f, *stoi_b, *reac_order;
  const double *A, *b, *Ea, *A2, *b2, *Ea2, *tbc, *troe_alpha, *troe_t3, *troe_t1, *troe_t2;
  // NASA9 multi-range thermo (nasa9 = 1): cuts [n_spec][max_range+1], coefficients
  // [n_spec][max_range][9] (a0..a6, b1, b2)
  int nasa9, max_range;
  const int *n_range;
  const double *t_cut, *poly9;
  // control temperatures of the two-temperature reaction rates (park = 1)
  int park;
  const double *tcf_a, *tcf_b, *tcb_a, *tcb_b;
  // two-temperature data (null / 0 for one temperature)
  int max_level, enable_vt;
  const double *theta_v, *elec_theta, *elec_g, *lt_a, *lt_b, *park_sigma;
  const int *n_level;
  const double *elec_cut;  // [n_spec] truncation constant A of the electronic sums (ve_energy)
};

// Scalar settings passed by value to kernels.
struct Param {
  int dim, n_var, n_spec, n_scalar, n_scalar_transported, n_reac;
  int i_eve;  // two-temperature: e_ve's index in sv (= n_spec); -1 for one temperature
  int inviscid_scheme, reconstruction, limiter, viscous_order, positive_preserving;
  int gradP, reaction, shock_sensor;
  double sensor_eps, sensor_threshold, entropy_fix_factor, Pr, cfl;
  double rho_ref, v_ref, weno_eps_scale, mu_constant;
  int precision;
  // air with 8th-order viscous terms and WENO7 primitive sweeps: each sweep also adds
  // J d(node flux)/d(its direction) (the viscous divergence), and the x sweep, the first writer
  // of the residual, assigns dq instead of adding to it
  int visc8_fused;
  int limit_flow;
  double lf_ll[5], lf_ul[5];  // limit_flow bounds of rho, u, v, w, p
  double dt;                  // the current step's time step (positivity limiter)
  const double *dt_dev;       // non-null: the step's time step lives on the device (graph runs)
  long long step;             // the step number the face conditions see (the blowing wall)
  unsigned *status;  // device status word
  Mech mech;
};

__device__ __forceinline__ void flag_status(const Param &p, unsigned bits) {
  if (p.status) atomicOr(p.status, bits);
}

// The step's time step: the device copy when the step runs inside a device-driven graph,
// otherwise the value the launch carries.
__device__ __forceinline__ double step_dt(const Param &p, double dt) { return p.dt_dev ? *p.dt_dev : dt; }

// SSP-RK3 Shu-Osher coefficients (src/RK.cuh:12-16).
__host__ __device__ __forceinline__ void ssprk3_coeff(int rk, double &a, double &b, double &c) {
  if (rk == 0) { a = 1.0; b = 0.0; c = 1.0; }
  else if (rk == 1) { a = 0.75; b = 0.25; c = 0.25; }
  else { a = 1.0 / 3.0; b = 2.0 / 3.0; c = 2.0 / 3.0; }
}

__host__ __device__ __forceinline__ double sutherland(double t) {
  // src/Transport.cu:7-9
  return 1.7894e-5 * pow(t / 288.16, 1.5) * (288.16 + 110) / (t + 110);
}

}  // namespace cb2
