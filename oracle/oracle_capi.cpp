// C ABI of the FP64 host oracle (loaded by the tests through ctypes).
// TEST INFRASTRUCTURE ONLY: never linked into or called by libcb200.
//
// The oracle takes the same cb2_param_view / cb2_zone_view / cb2_face_bc structs as the
// library, with HOST pointers in the zone view.
#include "oracle.hpp"
#include "cb200_serve.h"
#include <cstring>
#ifdef _OPENMP
#include <omp.h>
#endif

using namespace oracle;

extern "C" {

void oracle_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

int oracle_stage_update(const cb2_param_view *pv, const cb2_zone_view *zv, double dt, int rk) {
  Param p = make_param(*pv);
  Zone z = make_zone(*zv, nullptr, 0, p);
  update_cv_and_bv_rk(z, p, dt, rk);
  return 0;
}

int oracle_vt_relaxation(const cb2_param_view *pv, const cb2_zone_view *zv, double dt_stage) {
  Param p = make_param(*pv);
  Zone z = make_zone(*zv, nullptr, 0, p);
  apply_vt_relaxation(z, p, dt_stage);
  return 0;
}

// Two-temperature functions at one state (for the golden-fixture checks): out[0..3] = mixture
// e_ve(T), cv_ve(T), e_ve(Tve), cv_ve(Tve); out[4] = T_ve inverted from e_ve(Tve) starting at T;
// out[5..7] = VT source, e_ve equilibrium, effective relaxation time.
void oracle_two_temperature_state(const cb2_param_view *pv, double rho, double t, double tve, const double *y,
                                  double *out) {
  Param p = make_param(*pv);
  out[0] = mixture_ve_energy(p, t, y, &out[1]);
  out[2] = mixture_ve_energy(p, tve, y, &out[3]);
  out[4] = invert_tve_from_eve(p, out[2], y, t);
  out[5] = vt_relaxation_source(p, rho, t, tve, y, &out[6], &out[7]);
}

// Species e_ve and cv_ve at t: e[n_spec], cv[n_spec]
void oracle_species_ve(const cb2_param_view *pv, double t, double *e, double *cv) {
  Param p = make_param(*pv);
  for (int s = 0; s < p.n_spec; ++s) {
    e[s] = ve_energy(p, s, t);
    cv[s] = ve_cv(p, s, t);
  }
}

int oracle_cv_from_bv(const cb2_param_view *pv, const cb2_zone_view *zv) {
  Param p = make_param(*pv);
  Zone z = make_zone(*zv, nullptr, 0, p);
  compute_cv_from_bv(z, p);
  return 0;
}

void oracle_set_step(long long step) { set_step(step); }

int oracle_rhs(const cb2_param_view *pv, const cb2_zone_view *zv, const cb2_face_bc *faces, int n_faces,
               unsigned mask) {
  Param p = make_param(*pv);
  Zone z = make_zone(*zv, faces, n_faces, p);
  std::memset(z.dq.p, 0, (size_t)z.dq.sz * p.n_var * sizeof(double));
  if (mask & CB2_RHS_VISCOUS) compute_viscous_flux(z, p);
  if ((mask & CB2_RHS_CHEMISTRY) && p.reaction) compute_chemistry(z, p);
  if (mask & CB2_RHS_INVISCID) {
    compute_inviscid_flux(z, p);
    outflow_nonreflecting(z, p);
  }
  return 0;
}

int oracle_boundary(const cb2_param_view *pv, const cb2_zone_view *zv, const cb2_face_bc *faces, int n_faces) {
  Param p = make_param(*pv);
  Zone z = make_zone(*zv, faces, n_faces, p);
  apply_boundary_conditions(z, p);
  return 0;
}

int oracle_shock_sensor(const cb2_param_view *pv, const cb2_zone_view *zv) {
  Param p = make_param(*pv);
  Zone z = make_zone(*zv, nullptr, 0, p);
  compute_shock_sensor(z, p);
  return 0;
}

int oracle_properties(const cb2_param_view *pv, const cb2_zone_view *zv) {
  Param p = make_param(*pv);
  Zone z = make_zone(*zv, nullptr, 0, p);
  update_physical_properties(z, p);
  return 0;
}

int oracle_cfl_dt(const cb2_param_view *pv, const cb2_zone_view *zv, double *dt) {
  Param p = make_param(*pv);
  Zone z = make_zone(*zv, nullptr, 0, p);
  *dt = local_time_step_min(z, p);
  return 0;
}

// One RK3 step over n_zones blocks; faces of zone b are faces[off_b .. off_b + n_faces[b]).
int oracle_rk3_step(const cb2_param_view *pv, const cb2_zone_view *zvs, const cb2_face_bc *faces,
                    const int *n_faces, int n_zones, double *dt, int fixed_dt) {
  Param p = make_param(*pv);
  std::vector<Zone> zones;
  int off = 0;
  for (int b = 0; b < n_zones; ++b) {
    zones.push_back(make_zone(zvs[b], faces + off, n_faces[b], p));
    off += n_faces[b];
  }
  rk3_step(zones, p, *dt, fixed_dt != 0);
  return 0;
}

// The same step for a multi-block grid: the inner faces of zone b are
// inner[ioff_b .. ioff_b + n_inner[b]) (registered form, cb2_inner_face).
int oracle_rk3_step_inner(const cb2_param_view *pv, const cb2_zone_view *zvs, const cb2_face_bc *faces,
                          const int *n_faces, const cb2_inner_face *inner, const int *n_inner, int n_zones,
                          double *dt, int fixed_dt) {
  Param p = make_param(*pv);
  std::vector<Zone> zones;
  int off = 0, ioff = 0;
  for (int b = 0; b < n_zones; ++b) {
    zones.push_back(make_zone(zvs[b], faces + off, n_faces[b], p));
    zones.back().inner.assign(inner + ioff, inner + ioff + n_inner[b]);
    off += n_faces[b];
    ioff += n_inner[b];
  }
  rk3_step(zones, p, *dt, fixed_dt != 0);
  return 0;
}

// The inner-face exchange alone over n_zones blocks (cb2_halo).
int oracle_halo(const cb2_param_view *pv, const cb2_zone_view *zvs, const cb2_inner_face *inner, const int *n_inner,
                int n_zones) {
  Param p = make_param(*pv);
  std::vector<Zone> zones;
  int ioff = 0;
  for (int b = 0; b < n_zones; ++b) {
    zones.push_back(make_zone(zvs[b], nullptr, 0, p));
    zones.back().inner.assign(inner + ioff, inner + ioff + n_inner[b]);
    ioff += n_inner[b];
  }
  inner_exchange(zones, p);
  return 0;
}

void oracle_nasa7_h_cp(const cb2_mechanism *m, double t, double *h, double *cp) {
  cb2_param_view pv{};
  pv.mech = m;
  pv.n_spec = m->n_spec;
  Param p = make_param(pv);
  nasa7_h_cp(t, p.mech, h, cp);
}

// omega_k and the destruction part omega_d,k [kg/(m^3 s)] of one state (rho, T, Y).
void oracle_chemistry_source(const cb2_mechanism *m, double rho, double t, const double *y, double *omega,
                             double *omega_d) {
  cb2_param_view pv{};
  pv.mech = m;
  pv.n_spec = m->n_spec;
  Param p = make_param(pv);
  chemistry_source(p.mech, rho, t, y, omega, omega_d);
}

void oracle_gibbs_rt(const cb2_mechanism *m, double t, double *g) {
  cb2_param_view pv{};
  pv.mech = m;
  pv.n_spec = m->n_spec;
  Param p = make_param(pv);
  species_gibbs_rt(t, p.mech, g);
}

// The same at (T, Tve): with the mechanism's control-temperature model each reaction runs at its
// own smoothed T^a Tve^b.
void oracle_chemistry_source_2t(const cb2_mechanism *m, double rho, double t, double tve, const double *y,
                                double *omega, double *omega_d) {
  cb2_param_view pv{};
  pv.mech = m;
  pv.n_spec = m->n_spec;
  Param p = make_param(pv);
  chemistry_source_2t(p.mech, rho, t, tve, y, omega, omega_d);
}

// A 0-D reactor from (T0, p0, Y) advanced by at most max_attempts ROK4E attempts (or to t_end),
// with the full Jacobian or (krylov != 0) on the Arnoldi basis;
// the state is returned in the cb2_reactor layout of include/cb200_serve.h.
void oracle_reactor_run(const cb2_mechanism *m, double T0, double p0, const double *Y, double t_end, double h0,
                        double rtol, double atol, int max_attempts, cb2_reactor *out, int krylov) {
  cb2_param_view pv{};
  pv.mech = m;
  pv.n_spec = m->n_spec;
  Param p = make_param(pv);
  ReactorState st;
  reactor_setup(p.mech, T0, p0, Y, t_end, h0, st);
  reactor_advance(p.mech, st, max_attempts, rtol, atol, krylov != 0);
  std::memset(out, 0, sizeof(*out));
  for (int l = 0; l < m->n_spec; ++l) out->rhoY[l] = st.rhoY[l];
  out->rho = st.rho; out->E = st.E; out->T = st.T; out->p = st.p;
  out->time = st.time; out->t_end = st.t_end; out->h = st.h; out->err_last = st.err_last;
  out->step = st.step; out->n_reject = st.n_reject; out->status = st.status;
}

// The same reactor advanced by at most max_steps fixed steps of dt (or to t_end) in the form
// scheme (CB2_REACTOR_EXPLICIT .. CB2_REACTOR_RK3, optionally | CB2_REACTOR_CONSERVE_MASS).
void oracle_reactor_run_fixed(const cb2_mechanism *m, double T0, double p0, const double *Y, double t_end,
                              double dt, int scheme, int max_steps, cb2_reactor *out) {
  cb2_param_view pv{};
  pv.mech = m;
  pv.n_spec = m->n_spec;
  Param p = make_param(pv);
  ReactorState st;
  reactor_setup(p.mech, T0, p0, Y, t_end, dt, st);
  reactor_advance_fixed(p.mech, st, max_steps, scheme & 0xf, (scheme & CB2_REACTOR_CONSERVE_MASS) != 0);
  std::memset(out, 0, sizeof(*out));
  for (int l = 0; l < m->n_spec; ++l) out->rhoY[l] = st.rhoY[l];
  out->rho = st.rho; out->E = st.E; out->T = st.T; out->p = st.p;
  out->time = st.time; out->t_end = st.t_end; out->h = st.h; out->err_last = st.err_last;
  out->step = st.step; out->n_reject = st.n_reject; out->status = st.status;
}

}  // extern "C"
