// FP64 host oracle of COREFL's explicit residual-and-update path.
//
// TEST INFRASTRUCTURE ONLY: this restatement of the reference algorithm is the checker the
// parity tests, smoke() and the bench's CPU-baseline leg compare the CUDA library against.
// The product (libcb200) never links, loads or calls it.
//
// Every routine restates one reference kernel as a plain loop over nodes, in the same
// arithmetic order as the reference source (cited per function, paths relative to the
// COREFL-CPC source tree).  Arrays use the reference's padded SoA layout
// (ggxl::VectorField3D, src/gxl_lib/Array.cuh:307-328), so the same buffers can be handed
// to the oracle and (after a host->device copy) to the library.
#pragma once
#include <cmath>
#include <cstdint>
#include <vector>
#include <algorithm>
#include "cb200.h"

namespace oracle {

constexpr double R_u = 8314.462618;   // src/Constants.h:15
constexpr double R_c = 1.98720425864083;
constexpr double gamma_air = 1.4;     // src/Constants.h:19
constexpr double mw_air = 28.9647;    // src/Constants.h:25
constexpr double R_air = R_u / mw_air;
constexpr double p_atm = 101325;
constexpr double eps_weno = 1e-40;    // src/WENO.cu:8
constexpr double pi = 3.141592653589793;

// A padded array view with g ghost layers: element (i,j,k,l) at
// k*d1 + j*d2 + i + dt + l*sz (src/gxl_lib/Array.cuh:315-324).
struct Arr {
  double *p = nullptr;
  long long d2 = 0, d1 = 0, dt = 0, sz = 0;
  Arr() = default;
  Arr(double *ptr, int mx, int my, int mz, int g) : p(ptr) {
    d2 = mx + 2 * g;
    d1 = (long long)(my + 2 * g) * d2;
    dt = (d1 + d2 + 1) * g;
    sz = (long long)(mx + 2 * g) * (my + 2 * g) * (mz + 2 * g);
  }
  double &operator()(int i, int j, int k, int l = 0) const { return p[k * d1 + j * d2 + i + dt + l * sz]; }
  explicit operator bool() const { return p != nullptr; }
};

struct Mechanism {
  int n_spec = 0, n_reac = 0;
  std::vector<double> imw, gas_const, mw;
  std::vector<double> lo, hi, t_low, t_mid, t_high;
  std::vector<double> geometry, lj_inv, vis_coeff, wjwi14, sqwiwj8, bdc, kbe, zrot;
  std::vector<int> reac_type, rev_type, stoi_f, stoi_b, reac_order;
  std::vector<double> A, b, Ea, A2, b2, Ea2, tbc, troe_alpha, troe_t3, troe_t1, troe_t2;
  // NASA9 multi-range thermo (nasa == 9): cuts [n_spec][max_range+1], coefficients
  // [n_spec][max_range][9]
  int nasa = 7, max_range = 0;
  std::vector<int> n_range;
  std::vector<double> t_cut, poly9;
  // two-temperature control temperatures of the reaction rates
  bool park = false;
  std::vector<double> tcf_a, tcf_b, tcb_a, tcb_b;
};

// Vibrational-electronic data of the two-temperature model (cfd::Species::read_two_temperature,
// src/ChemData.cpp:130-233; DParameter copies, src/DParameter.cu:150-200)
struct TwoTemperature {
  bool on = false;
  bool enable_vt = true;
  int max_level = 1;
  std::vector<double> theta_v, elec_theta, elec_g, lt_a, lt_b, park_sigma;
  std::vector<int> n_level;
};

struct Param {
  int dim = 3, n_var = 5, n_spec = 0, n_scalar = 0, n_scalar_transported = 0, n_reac = 0;
  int i_eve = -1;  // index of e_ve in sv (two-temperature), -1 otherwise
  int inviscid_scheme = 52, reconstruction = 2, limiter = 0, viscous_order = 0;
  int positive_preserving = 0, gradP = 0, reaction = 0, shock_sensor = 0;
  double sensor_eps = 0, sensor_threshold = 0, entropy_fix_factor = 0.125, Pr = 0.72, cfl = 0.5;
  double rho_ref = 1, v_ref = 1, weno_eps_scale = 1, mu_constant = 0;
  int limit_flow = 0;
  double dt = 0;  // the step's time step (positivity limiter)
  long long step = 0;  // the step number the face conditions see (the blowing wall)
  double lf_ll[5] = {0, 0, 0, 0, 0}, lf_ul[5] = {0, 0, 0, 0, 0};
  Mechanism mech;
  TwoTemperature tt;
};

struct FaceBC {
  int type = 0, face = 0, direction = 1;
  bool nonreflecting = false;  // outflow with the non-reflecting dq correction
  int start[3] = {0, 0, 0}, end[3] = {0, 0, 0};
  double rho = 0, u = 0, v = 0, w = 0, p = 0, T = 0, wall_T = 0, wall_Tve = 0;
  std::vector<double> sv;  // inflow scalars
  bool blow = false;        // blowing wall (cb2_face_bc::blow_*)
  int blow_start = 0, blow_end = 0;
  double blow_coef = 0;
};

struct Zone {
  int mx = 0, my = 0, mz = 0, ngg = 0;
  Arr cv, bv, sv, qn, dq, metric, jac, mul, kappa, rhoD, acoustic, gamma, mach, fF, gF, hF, visf, shock, dtl, rts,
      efd, tve, kappa_ve;
  std::vector<int> il, ir, jl, jr, kl, kr;  // physical-boundary flags per face node
  std::vector<FaceBC> faces;
  std::vector<cb2_inner_face> inner;  // inner faces of a multi-block grid
};

Param make_param(const cb2_param_view &pv);
// the step number make_param gives the face conditions (the library's cb2_set_step); rk3_step
// counts one before its stages and leaves it there
void set_step(long long step);
Zone make_zone(const cb2_zone_view &v, const cb2_face_bc *faces, int n_faces, const Param &p);

void update_cv_and_bv_rk(Zone &z, const Param &p, double dt, int rk);
void inner_exchange(std::vector<Zone> &zones, const Param &p);
void limit_flow(Zone &z, const Param &p);
void compute_cv_from_bv(Zone &z, const Param &p);
void compute_inviscid_flux(Zone &z, const Param &p);
void outflow_nonreflecting(Zone &z, const Param &p);
void compute_viscous_flux(Zone &z, const Param &p, int phase = 0);
void inner_flux_exchange(std::vector<Zone> &zones, const Param &p);
void viscous_all(std::vector<Zone> &zones, const Param &p);
void compute_chemistry(Zone &z, const Param &p);
void chemistry_source(const Mechanism &m, double rho, double t, const double *y, double *omega, double *omega_d);
// g_k/(R_k T) of every species (compute_gibbs_div_rt)
void species_gibbs_rt(double t, const Mechanism &m, double *g);
// the same at (T, Tve): the control temperatures of the two-temperature reaction rates
void chemistry_source_2t(const Mechanism &m, double rho, double t, double tve, const double *y, double *omega,
                         double *omega_d);
void update_physical_properties(Zone &z, const Param &p);
void compute_shock_sensor(Zone &z, const Param &p);
void apply_boundary_conditions(Zone &z, const Param &p);
double local_time_step_min(Zone &z, const Param &p);
void rk3_step(std::vector<Zone> &zones, const Param &p, double &dt, bool fixed_dt);

// thermodynamics used by the tests directly
void nasa7_h_cp(double t, const Mechanism &m, double *h, double *cp);

// forward/backward rates of progress [mol/(cm^3 s)] of every reaction at t and c [mol/cm^3]
void reaction_rates(const Mechanism &m, double t, const double *c, double *q1, double *q2);

// two-temperature model (two_temp.cpp)
double ve_energy(const Param &p, int i, double t);
double ve_cv(const Param &p, int i, double t);
double mixture_ve_energy(const Param &p, double t, const double *y, double *cv_ve);
void characteristic_thermo_2t(const Param &p, double t, const double *y, double *gamma, double *c, double *alpha,
                              double *ecoef, double *e_tr_out = nullptr);
// cv_tr, cp_tr and R of the mixture at t (compute_mixture_tr_energy's heat capacities)
void tr_heat_capacities(const Param &p, double t, const double *y, double &cv_tr, double &cp_tr, double &r_mix);
double invert_tve_from_eve(const Param &p, double eve_target, const double *y, double t_init);
double vt_relaxation_source(const Param &p, double density, double t, double tve, const double *y, double *eve_eq,
                            double *tau_eff);
void temperature_2t(Zone &z, const Param &p, int i, int j, int k, double total_energy);
void sync_two_temperature(Zone &z, const Param &p, int i, int j, int k);
double total_energy_2t(Zone &z, const Param &p, int i, int j, int k);
void apply_vt_relaxation(Zone &z, const Param &p, double dt_stage);

// 0-D constant-volume reactor (reactor.cpp)
struct ReactorState {
  std::vector<double> rhoY;
  double rho = 0, E = 0, T = 0, p = 0, time = 0, t_end = 0, h = 0, err_last = 0;
  int step = 0, n_reject = 0, status = 0;
};
void reactor_setup(const Mechanism &m, double T0, double p0, const double *Y, double t_end, double h0,
                   ReactorState &st);
void reactor_advance(const Mechanism &m, ReactorState &st, int max_attempts, double rtol, double atol,
                     bool krylov = false);
void reactor_advance_fixed(const Mechanism &m, ReactorState &st, int max_steps, int scheme, bool conserve);

}  // namespace oracle
