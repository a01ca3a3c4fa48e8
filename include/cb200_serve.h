/* cb200_serve.h -- batched and served solves on top of libcb200.
 *
 * Two request kinds share one GPU:
 *   - 0-D constant-volume reactors, advanced by the adaptive ROK4E Rosenbrock scheme with the
 *     full chemistry Jacobian, as the reference's const_volume_reactor does with
 *     advance_scheme = 1, build_arnoldi = 0, adaptive_time_step = 1
 *     (src/ConstVolumeReactor.cpp:385-700);
 *   - 1-D blocks (e.g. reactive shock tubes), advanced by whole SSP-RK3 steps of the same
 *     per-node operations as cb2_rk3_step, one CTA per case.
 * Both run many independent cases of uneven size in one launch.  The server keeps every
 * admitted case resident in device memory, admits new requests as slots and HBM free up, and
 * reports per-request latency. */
#ifndef CB200_SERVE_H
#define CB200_SERVE_H

#include "cb200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- 0-D constant-volume reactors ------------------------------------------------------ */

#define CB2_REACTOR_MAX_SPEC 9

/* State of one reactor (device memory, one struct per reactor).  rho and E (internal energy per
 * unit mass) are constant; rhoY, T, p, time, h and err_last evolve. */
typedef struct {
  double rhoY[CB2_REACTOR_MAX_SPEC]; /* partial densities, kg/m^3 */
  double rho, E, T, p;
  double time, t_end, h, err_last;   /* h: next step size, err_last: last accepted error norm */
  int step, n_reject, status, pad;   /* accepted steps, rejected steps, CB2_REACTOR_* bits */
} cb2_reactor;

#define CB2_REACTOR_DONE 1u        /* time reached t_end */
#define CB2_REACTOR_NONPHYSICAL 2u /* T or a partial density left the physical range: stopped */

/* Sets n reactors from (T0 [K], p0 [Pa], Y[n * n_spec] mass fractions, t_end [s]) as
 * const_volume_reactor does (src/ConstVolumeReactor.cpp:61-66, 328-336): rho = p/(R_u imw T),
 * rhoY = rho Y, E = sum Y h(T) - p/rho; the first step size is h0.  All pointers are device
 * pointers; ctx supplies the mechanism (cb2_init with n_spec 5 or 9). */
int cb2_reactor_setup(cb2_ctx *ctx, cb2_reactor *reactors, int n, const double *T0, const double *p0,
                      const double *Y, const double *t_end, double h0, void *stream);

/* Advances each unfinished reactor by at most max_attempts ROK4E step attempts (accepted or
 * rejected) or until it reaches t_end, with the error norm of the reference
 * (RTol rhoY + ATol per species). */
int cb2_reactor_advance(cb2_ctx *ctx, cb2_reactor *reactors, int n, int max_attempts, double rtol, double atol,
                        void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CB200_SERVE_H */
