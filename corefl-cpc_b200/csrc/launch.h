// Host-side launch helpers and the declarations of every kernel launcher in the library.
#pragma once
#include <cuda_runtime.h>
#include "common.cuh"
#include "cb200_serve.h"

namespace cb2 {

void set_cuda_error(cudaError_t e);

#define CB2_TRY(expr)                 \
  do {                                \
    int _rc = (expr);                 \
    if (_rc != CB2_OK) return _rc;    \
  } while (0)

inline int check_launch() {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_cuda_error(e);
    return CB2_ERR_CUDA;
  }
  return CB2_OK;
}

inline int check_cuda(cudaError_t e) {
  if (e != cudaSuccess) {
    set_cuda_error(e);
    return CB2_ERR_CUDA;
  }
  return CB2_OK;
}

// Per-launch timing (enabled per context by cb2_profile_enable): the API entry points make
// the context's profiler current for the calling thread; every launcher brackets its
// kernels with a ProfScope, which records a CUDA event pair on the launch stream.
struct Profiler;
extern thread_local Profiler *g_prof;
void prof_begin(Profiler *p, const char *name, cudaStream_t s);
void prof_end(Profiler *p, cudaStream_t s);

struct ProfScope {
  cudaStream_t s;
  ProfScope(const char *name, cudaStream_t st) : s(st) {
    if (g_prof) prof_begin(g_prof, name, s);
  }
  ~ProfScope() {
    if (g_prof) prof_end(g_prof, s);
  }
};

template <typename K>
inline int prepare_smem(K kern, size_t bytes) {
  if (bytes > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) { set_cuda_error(e); return CB2_ERR_CUDA; }
  }
  return CB2_OK;
}

// Face boundary condition in device-usable form (after the reference's register_boundary).
struct FaceBC {
  int type, face, direction;
  int nonreflecting;  // outflow with the non-reflecting correction of dq (CB2_BC_NONREFLECTING)
  int start[3], end[3];
  double rho, u, v, w, p, T, wall_T, wall_Tve;
  const double *sv;  // inflow scalars (device copy of cb2_face_bc::sv)
  int blow, blow_start, blow_end;  // blowing wall (cb2_face_bc::blow_*)
  double blow_coef;
};

// ---- launchers (each returns CB2_OK or an error code; n_launch counts kernels) ----------
int launch_inviscid_char(const Zone &z, const Param &p, cudaStream_t s, int &n_launch);
int launch_inviscid_comp(const Zone &z, const Param &p, cudaStream_t s, int &n_launch);
int launch_inviscid_pv(const Zone &z, const Param &p, cudaStream_t s, int &n_launch);
int launch_inviscid_pv_f32(const Zone &z, const Param &p, cudaStream_t s, int &n_launch);
int launch_stage_update(const Zone &z, const Param &p, double dt, int rk, cudaStream_t s, int &n_launch);
int launch_cv_from_bv(const Zone &z, const Param &p, cudaStream_t s, int &n_launch);
// two-temperature VT relaxation over dt_stage of every interior node (a standalone
// apply_vt_relaxation_rk; launch_stage_update runs it itself for two-temperature contexts)
int launch_vt_relaxation(const Zone &z, const Param &p, double dt_stage, cudaStream_t s, int &n_launch);
int launch_properties(const Zone &z, const Param &p, cudaStream_t s, int &n_launch);
int launch_boundary(const Zone &z, const Param &p, const FaceBC *faces, int n_faces, cudaStream_t s,
                    int &n_launch);
// one inner face of a multi-block grid: z's face nodes and ghosts from / with zt
int launch_inner_exchange(const Zone &z, const Zone &zt, const Param &p, const cb2_inner_face &f, cudaStream_t s,
                          int &nl);
int launch_eliminate_k_gradient(const Zone &z, const Param &p, cudaStream_t s, int &n_launch);
// the non-reflecting correction of dq at the nodes of every outflow face that asks for it
int launch_nonreflecting(const Zone &z, const Param &p, const FaceBC *faces, int n_faces, cudaStream_t s,
                         int &n_launch);
int launch_periodic_flux_exchange(const Zone &z, const Param &p, const FaceBC *faces, int n_faces, cudaStream_t s,
                                  int &n_launch);
// The 8th-order air viscous term writes dq instead of adding to it (assign = true) when it runs
// first in a residual; viscous_assigns_dq tells whether the settings take that path.
bool viscous_assigns_dq(const Param &p);
// Whether the 8th-order node fluxes live in the block's FP32 copies (the mixed form of air); the
// node-flux, flux-exchange and divergence kernels all follow it.
inline bool visc8_f32(const Param &p) { return p.precision == CB2_PREC_MIXED && p.n_spec == 0; }
// With p.visc8_fused the 8th-order path stops after the node fluxes and their periodic
// exchange: the WENO7 primitive sweeps take the divergence.  phase (order 8 only): 0 the whole
// viscous term; 1 the node fluxes only; 2 the periodic node-flux exchange and the divergence
// (between the two, a multi-block step exchanges the node fluxes across inner faces).
int launch_viscous(const Zone &z, const Param &p, const FaceBC *faces, int n_faces, bool assign, cudaStream_t s,
                   int &n_launch, int phase = 0);
// the 8th-order node fluxes across one inner face of a multi-block grid (exchange_value task 1)
int launch_inner_flux_exchange(const Zone &z, const Zone &zt, const Param &p, const cb2_inner_face &f,
                               cudaStream_t s, int &n_launch);
int launch_chemistry(const Zone &z, const Param &p, cudaStream_t s, int &n_launch);
int launch_shock_sensor(const Zone &z, const Param &p, cudaStream_t s, int &n_launch);
int launch_local_dt(const Zone &z, const Param &p, cudaStream_t s, int &n_launch);
int launch_min_reduce(const double *src, long long n, double *partial, int n_partial, double *out,
                      cudaStream_t s, int &n_launch);
int min_reduce_partials(long long n);
int launch_set_value(double *dst, double v, cudaStream_t s, int &n_launch);
// dst[i] = float(src[i]) for i < n (the mixed form's FP32 copies)
int launch_to_f32(const double *src, float *dst, size_t n, cudaStream_t s, int &n_launch);

// State of the device-driven step loop (cb2_rk3_run, graph.cu): the loop repeats while
// step < max_steps, time < t_end, dt is positive and finite and the status word is clear.
struct RunState {
  double time, t_end;
  double dt;  // fixed mode: the step every iteration takes; CFL mode: the last step taken
  long long step, max_steps;
};
int launch_run_advance(RunState *r, const double *dt, const unsigned *status, cudaGraphConditionalHandle h,
                       cudaStream_t s, int &n_launch);

// batched 0-D reactors (reactor.cu); the state type is cb2_reactor of cb200_serve.h
int launch_reactor_setup(const Param &p, cb2_reactor *r, int n, const double *T0, const double *p0,
                         const double *Y, const double *t_end, double h0, cudaStream_t s);
int launch_reactor_fixed(const Param &p, cb2_reactor *r, int n, int max_steps, int scheme, cudaStream_t s);
int launch_reactor_advance(const Param &p, cb2_reactor *r, int n, int max_attempts, double rtol, double atol,
                           cudaStream_t s, bool krylov = false);

}  // namespace cb2
