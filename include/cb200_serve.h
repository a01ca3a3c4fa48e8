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

/* cb2_reactor_advance with build_arnoldi = 1 (src/ConstVolumeReactor.cpp:446-594, buildArnoldi
 * :1858-1930): J replaced by its projection on an Arnoldi basis of finite-difference products
 * (Krylov limit n_spec, minimum 4; n_spec extra source evaluations per attempt).  Stages 3 and 4
 * take the projected correction with the opposite sign to stages 1 and 2, as the reference does;
 * its steps shrink until they stall short of t_end on the H2/air reactors. */
int cb2_reactor_advance_krylov(cb2_ctx *ctx, cb2_reactor *reactors, int n, int max_attempts, double rtol,
                               double atol, void *stream);

/* Fixed-step forms of const_volume_reactor (src/ConstVolumeReactor.cpp:403-441, 708-763). */
#define CB2_REACTOR_EXPLICIT 0          /* advance_scheme 0, implicit_method 0: rhoY += omega dt  */
#define CB2_REACTOR_EPI 1               /* implicit_method 1: omega <- (I - dt J)^-1 omega (EPI)   */
#define CB2_REACTOR_DA 2                /* implicit_method 2: omega_l <- omega_l / (1 - dt J_ll)   */
#define CB2_REACTOR_RK3 3               /* advance_scheme 3: explicit three-stage Runge-Kutta     */
#define CB2_REACTOR_CONSERVE_MASS 0x10  /* | with forms 0-2: conserve_mass_corefl = 1             */

/* Advances each unfinished reactor by at most max_steps fixed steps of dt = its h (the h0 of
 * cb2_reactor_setup, left unchanged) in the form `scheme`, or until it reaches t_end; partial
 * densities are clipped at 0 after each step as the reference does.  CB2_ERR_INVALID for an
 * unknown form or CONSERVE_MASS with RK3 (the reference applies it to forms 0-2 only). */
int cb2_reactor_advance_fixed(cb2_ctx *ctx, cb2_reactor *reactors, int n, int max_steps, int scheme, void *stream);

/* ---- serving: continuous batching of reactors and shock tubes --------------------------- */

#define CB2_REQ_REACTOR 0 /* 0-D constant-volume reactor from (T0, p0, Y) to t_end            */
#define CB2_REQ_TUBE 1    /* 1-D two-state shock tube of n_nodes nodes to t_end               */

typedef struct {
  int kind;             /* CB2_REQ_* */
  int n_nodes;          /* tube: nodes (8 .. 2^22) */
  double arrival;       /* seconds after the start of cb2_serve_run */
  double T0, p0;        /* reactor: initial temperature [K] and pressure [Pa] */
  double t_end;         /* physical end time [s] */
  double Y[CB2_REACTOR_MAX_SPEC]; /* reactor: mass fractions */
  void *out_state;      /* optional host buffer for the final state: a cb2_reactor, or for a tube
                         * the interior primitives bv[6][n_nodes] followed by sv[n_spec][n_nodes] */
} cb2_request;

typedef struct {
  double t_arrival, t_admit, t_done; /* seconds after the start, host clock */
  double latency;                    /* t_done - t_arrival */
  double T, p;                       /* reactor: final T and p; tube: peak T (p unused) */
  double time;                       /* physical time reached */
  int steps, status;                 /* accepted steps; CB2_REACTOR_* bits, or for a tube
                                      * 1 = done, 2 = failed (non-finite dt or state) */
} cb2_result;

typedef struct {
  long long iterations;      /* batched launches per kind */
  long long peak_pool_bytes; /* peak device memory held by admitted tubes */
  double wall_s;             /* duration of the run */
} cb2_serve_stats;

typedef struct {
  size_t hbm_budget_bytes;            /* device pool for the admitted tubes' state */
  int max_tubes, max_reactors;        /* concurrent slots of each kind */
  int tube_steps_per_launch;          /* RK3 steps per batched tube launch */
  int reactor_attempts_per_launch;    /* ROK4E attempts per batched reactor launch */
  double rtol, atol, h0;              /* reactor error control and first step */
  double tube_length;                 /* [m]; the two states meet at the middle */
  double tube_TL, tube_pL, tube_TR, tube_pR;
  const double *tube_Y;               /* host, n_spec mass fractions of the tube gas */
  double time_limit_s;                /* > 0: give up with CB2_ERR_TIMEOUT after this wall time */
  cb2_serve_stats *stats;             /* optional */
} cb2_serve_options;

/* Serves n requests that arrive on the timeline reqs[].arrival: admits each one as soon as it
 * has arrived, a slot of its kind is free and its state fits in the pool, keeps it resident
 * until it finishes, and advances all admitted cases with one batched launch per kind per
 * iteration (reactors on ctx_reactor's mechanism; tubes with ctx_tube's scheme: 1-D, inviscid,
 * 9-species mixture, WENO5 with HLLC or AUSM+).  Fills out[i] for reqs[i].  A case's result does
 * not depend on which other cases share its launches.  Blocks until every request is done.
 * No counterpart in the reference, which runs one case per process. */
int cb2_serve_run(cb2_ctx *ctx_reactor, cb2_ctx *ctx_tube, const cb2_request *reqs, int n,
                  const cb2_serve_options *opt, cb2_result *out);

/* ---- batched blocks ---------------------------------------------------------------------- */

/* One block of a batch: a closed (all faces periodic) 2-D (mz = 1) or 3-D block of any size,
 * its device arrays in the cb2_zone_view layout (cv, bv, qn, dq, metric, jac, mul; mach
 * optional), and its run state. */
typedef struct cb2_block_case {
  cb2_zone_view zone;
  double time, t_end;  /* in: current time and end time; out: time reached                  */
  double dt;           /* > 0: the fixed step; 0: each step's CFL step (the context's cfl)   */
  double last_dt;      /* out: the last step taken                                         */
  int steps;           /* out: steps taken by the call                                     */
  int status;          /* out: CB2_BLOCK_DONE (time >= t_end) | CB2_BLOCK_FAILED            */
} cb2_block_case;
#define CB2_BLOCK_DONE 1
#define CB2_BLOCK_FAILED 2 /* a non-finite or non-positive step, or a non-physical state */

/* Advances every block of cases[0..n) (host array) by up to max_steps SSP-RK3 steps, stopping
 * each at its own t_end, in ONE persistent launch: each thread-block cluster takes the next
 * block from a work queue ordered by decreasing size (largest first), runs its whole steps (qn
 * copy, dt, three stages of zeroed residual, x/y/z primitive sweeps, stage update, periodic
 * ghost fill, properties) with the phases' tiles and nodes spread over its CTAs and cluster
 * barriers between the phases, then takes the next block.  The arithmetic
 * per node is the block path's: a block's results equal cb2_rk3_step on the same block bit for
 * bit and do not depend on the other blocks of the batch.  Built for the air model, inviscid,
 * WENO5/WENO7 primitive reconstruction with AUSM+ or HLLC, FP64; every block needs
 * m >= ngg + 2 nodes along each periodic direction.  The y/z sweep tile width and the cluster
 * size are the ones cb2_block_batch_autotune picked for this context (8 and 8 until then).
 * Synchronises `stream`. */
int cb2_block_batch_advance(cb2_ctx *ctx, cb2_block_case *cases, int n, int max_steps, void *stream);

/* Times the batch's residual phase (zeroed dq and the three sweeps of every block, one
 * persistent launch per candidate) for every y/z tile width (4, 8, 16) and cluster size (1, 2,
 * 4, 8 CTAs per block) and keeps the fastest pair for this context's later batches; writes it
 * to schedule_out[2] = {tile width, cluster size} when not NULL.  Only the blocks' dq (a
 * per-stage scratch) changes.  Synchronises `stream`. */
int cb2_block_batch_autotune(cb2_ctx *ctx, cb2_block_case *cases, int n, int *schedule_out, void *stream);

/* Sets the batch's y/z tile width (4, 8 or 16) and cluster size (1, 2, 4 or 8) directly, e.g.
 * from an earlier tuning run.  Every choice gives the same results bit for bit. */
int cb2_block_batch_set_schedule(cb2_ctx *ctx, int tile_ni, int cluster_ctas);

#ifdef __cplusplus
}
#endif

#endif /* CB200_SERVE_H */
