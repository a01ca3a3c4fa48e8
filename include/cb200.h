/*
 * cb200.h -- C ABI of the B200-native explicit residual-and-update path of COREFL.
 *
 * The reference calls this path from `RK3<mix>()` (src/RK.cuh:107-272) as a sequence of
 * C++ launches on `DZone*` / `DParameter*`.  Every entry point below replaces one of those
 * calls (cited per function).  The library never allocates or frees the caller's field
 * arrays: it borrows the device pointers of the caller's padded per-block arrays, exactly
 * as `Field::setup_device_memory` (src/Field.cu:440-672) lays them out.
 *
 * Array layout (ggxl::VectorField3D<real>, ColMajor, src/gxl_lib/Array.cuh:307-328):
 *   a padded array with `g` ghost layers on (mx,my,mz) nodes holds element (i,j,k,l) at
 *     val[k*disp1 + j*disp2 + i + dispt + l*sz]
 *   with disp2 = mx+2g, disp1 = (my+2g)*disp2, dispt = (disp1+disp2+1)*g,
 *        sz = (mx+2g)*(my+2g)*(mz+2g);  -g <= i < mx+g etc.
 *   The ghost width of each array is the one the reference allocates: `ngg` for the flow
 *   fields, 0 for dq and dt_local, 1 for vis_flux.
 *
 * All pointers in cb2_zone_view are DEVICE pointers of the current CUDA device.  All
 * pointers in cb2_param_view / cb2_mechanism are HOST pointers; cb2_init copies them.
 * Streams are passed as `void*` (a cudaStream_t; NULL = legacy default stream).
 *
 * Every function returns 0 on success or a negative CB2_ERR_* code; none aborts.
 */
#ifndef CB200_H
#define CB200_H

#ifdef __cplusplus
extern "C" {
#endif

#define CB2_ABI_VERSION 6

/* ---- status codes ---------------------------------------------------------------- */
#define CB2_OK 0
#define CB2_ERR_CUDA (-1)        /* a CUDA runtime call failed (see cb2_last_cuda_error) */
#define CB2_ERR_INVALID (-2)     /* bad argument, view or parameter combination          */
#define CB2_ERR_NONPHYSICAL (-3) /* a kernel met rho<=0, T<=0 or a non-finite state      */
#define CB2_ERR_TIMEOUT (-4)     /* a bounded device-side wait gave up                    */
#define CB2_ERR_UNSUPPORTED (-5) /* scheme/model combination not built                    */
#define CB2_ERR_NOMEM (-6)       /* private scratch could not be allocated                */

/* ---- scheme codes (the reference's setup.txt keys, src/Parameter.cpp:234-312) -------- */
#define CB2_INV_ROE 2     /* inviscid_scheme = 2  : Roe + Harten fix, MUSCL/NND/1st       */
#define CB2_INV_AUSMP 3   /* inviscid_scheme = 3  : AUSM+ with primitive reconstruction   */
#define CB2_INV_HLLC 4    /* inviscid_scheme = 4  : HLLC with primitive reconstruction    */
#define CB2_INV_WENO5_CP 51
#define CB2_INV_WENO5_CH 52
#define CB2_INV_WENO7_CP 71
#define CB2_INV_WENO7_CH 72

#define CB2_REC_FIRST 1 /* reconstruction = 1 */
#define CB2_REC_MUSCL 2 /* reconstruction = 2 (kappa = 1/3, minmod) */
#define CB2_REC_NND2 3  /* reconstruction = 3 */
#define CB2_REC_WENO5 5 /* added: WENO5-JS weights on primitive variables (no reference kernel) */
#define CB2_REC_WENO7 7 /* added: WENO7-Z weights on primitive variables (no reference kernel)  */

/* boundary types: the reference's BC kinds (src/BoundCond.cu:3846-3998 comments) */
#define CB2_BC_WALL 2
#define CB2_BC_FARFIELD 4
#define CB2_BC_SYMMETRY 3
#define CB2_BC_INFLOW 5
#define CB2_BC_OUTFLOW 6
#define CB2_BC_PERIODIC 8
/* OR'd into CB2_BC_OUTFLOW: the face is also a non-reflecting outflow (an Outflow with
 * nonReflecting = 1): after the inviscid flux, cb2_rhs adds the characteristic correction of
 * DBoundCond::nonReflectingBoundary (apply_outflow_nr_conserv, src/BoundCond.cu:3580-3845; called
 * at src/RK.cuh:190-193) to dq at the face's nodes.  The ghost fill is the outflow's. */
#define CB2_BC_NONREFLECTING 0x100

/* precision forms */
#define CB2_PREC_FP64 0  /* plain form: FP64 throughout                                    */
#define CB2_PREC_MIXED 1 /* FP32 reconstruction/fluxes/viscous stencils, FP64 elsewhere      */

/* stage masks for cb2_rhs */
#define CB2_RHS_VISCOUS 1u
#define CB2_RHS_CHEMISTRY 2u
#define CB2_RHS_INVISCID 4u
#define CB2_RHS_ALL 7u
/* with the terms above: add them to the caller's dq instead of starting from zero (after
 * cb2_viscous, whose viscous residual the rest of the stage adds to) */
#define CB2_RHS_ACCUMULATE 8u

/* ---- views ------------------------------------------------------------------------- */

/* Device arrays of one block (the fields of `DZone`, src/Field.h:12-112).  Arrays the
 * configured path does not read may be NULL. */
typedef struct cb2_zone_view {
  int mx, my, mz, ngg;
  double *cv;       /* n_var comps, ghost ngg  (DZone::cv)                 */
  double *bv;       /* 6 comps (rho,u,v,w,p,T), ghost ngg  (DZone::bv)      */
  double *sv;       /* n_scalar comps, ghost ngg (DZone::sv)                */
  double *qn;       /* n_var comps, ghost ngg (DZone::qn)                   */
  double *dq;       /* n_var comps, ghost 0   (DZone::dq)                   */
  double *metric;   /* 9 comps (xi_xyz, eta_xyz, zeta_xyz), ghost ngg        */
  double *jac;      /* ghost ngg (DZone::jac)                               */
  double *mul;      /* ghost ngg (DZone::mul)                               */
  double *thermal_conductivity; /* ghost ngg, mixtures                       */
  double *rho_D;    /* n_spec comps, ghost ngg, mixtures                    */
  double *acoustic_speed; /* ghost ngg, mixtures                             */
  double *gamma;    /* ghost ngg, mixtures                                  */
  double *mach;     /* ghost ngg, optional                                  */
  double *fFlux, *gFlux, *hFlux; /* n_var comps, ghost ngg (8th-order viscous node fluxes) */
  double *vis_flux; /* n_var-1 comps, ghost 1 (2nd-order viscous face fluxes)  */
  double *shock_sensor;         /* ghost ngg, hybrid schemes only           */
  double *dt_local;             /* ghost 0                                  */
  double *reaction_timeScale;   /* ghost ngg, reacting cases                */
  double *entropy_fix_delta;    /* ghost 1, Roe                             */
  double *temperature_ve;       /* ghost ngg, two-temperature cases (DZone::temperature_ve) */
  double *thermal_conductivity_ve; /* ghost ngg, two-temperature mixtures with viscous terms
                                    * (DZone::thermal_conductivity_ve)                          */
} cb2_zone_view;

/* One face boundary condition of a block (cfd::Boundary, src/Mesh.h:8-30, after
 * register_boundary, src/Mesh.cpp:14-32): node ranges are inclusive, `face` is the normal
 * direction (0 i, 1 j, 2 k) and `direction` is -1 on the low face, +1 on the high face. */
typedef struct cb2_face_bc {
  int type;          /* CB2_BC_* */
  int face, direction;
  int range_start[3], range_end[3];
  /* inflow / farfield state and wall data; an outflow with p > 0 is the back-pressure outflow
   * (Outflow::if_backPressure, src/BoundCond.cu:2219-2320) with p its back pressure */
  double rho, u, v, w, p, T;
  double wall_temperature; /* <=0 : adiabatic wall */
  /* two temperatures: the T_ve of an isothermal wall (Wall::temperature_ve; <= 0: the wall
   * temperature) or of a farfield state (FarField::temperature_ve; <= 0: its boundary T) */
  double wall_temperature_ve;
  /* inflow and farfield: the n_scalar scalars of the state, Y_k and then (two temperatures) e_ve
   * (Inflow::sv / FarField::sv, src/BoundCond.h:23-169); required with species.  A wall of a
   * mixture: NULL for a non-catalytic wall (the ghosts copy the interior's Y_k), else the n_spec
   * mass fractions of a fully catalytic wall (Wall::yk with catalytic_type 1, src/BoundCond.h:105-107),
   * which its face node and ghosts take.  A HOST array copied at bind. */
  const double *sv;
  /* a wall that blows (Wall::if_blow_shock_wave, src/BoundCond.cu:3226-3245): while the context's
   * step (cb2_set_step) lies in [blow_start_step, blow_end_step], the wall moves along its inward
   * normal at blow_coefficient x max(normal velocity of the node inside towards the wall, seed),
   * the seed being the freestream's normal velocity (u, v, w of this face: ux_inf, uy_inf, uz_inf)
   * for steps <= 50.  blow_shock_wave = 0: a wall at rest.  (ABI version 6) */
  int blow_shock_wave, blow_start_step, blow_end_step;
  double blow_coefficient;
} cb2_face_bc;

/* One inner face of a multi-block grid, as cfd::InnerFace holds it after register_boundary
 * (src/Mesh.h:33-60, src/Mesh.cpp:39-172): the node range of this block covering the face layer
 * and its ngg ghost layers, the neighbour's block index and starting node, and the orientation
 * that maps a step n along this range to the neighbour's nodes:
 *   idx[a]     = range_start[a] + loop_dir[a] * n[a]
 *   idx_tar[a] = target_start[a] + target_loop_dir[a] * (loop_dir[src_tar[a]] * n[src_tar[a]]).
 * The fields have the reference's meaning and order, so a caller copies them from InnerFace. */
typedef struct cb2_inner_face {
  int range_start[3], range_end[3];
  int face, direction;
  int target_start[3], target_end[3];
  int target_block;
  int target_face, target_direction;
  int src_tar[3];
  int loop_dir[3], target_loop_dir[3];
  int n_point[3];
} cb2_inner_face;

/* Species / reaction data (the fields of `DParameter` that come from cfd::Species and
 * cfd::Reaction, src/DParameter.cuh:82-130).  All arrays are host arrays, row-major. */
typedef struct cb2_mechanism {
  int n_spec, n_reac;
  const double *mw;            /* [n_spec] kg/kmol                                         */
  /* NASA7 two-range polynomials (Combustion2Part): coefficients a0..a6 */
  const double *low_temp_coeff;  /* [n_spec*7] */
  const double *high_temp_coeff; /* [n_spec*7] */
  const double *t_low, *t_mid, *t_high; /* [n_spec] */
  /* transport (Species::geometry etc., src/ChemData.cpp) */
  const double *geometry;       /* [n_spec] 0 atom, 1 linear, 2 nonlinear                 */
  const double *LJ_potent_inv;  /* [n_spec] 1/(eps/kB)                                    */
  const double *vis_coeff;      /* [n_spec] viscosity prefactor                           */
  const double *WjDivWi_to_One4th;      /* [n_spec*n_spec] */
  const double *sqrt_WiDivWjPl1Mul8;    /* [n_spec*n_spec] */
  const double *binary_diffusivity_coeff; /* [n_spec*n_spec] */
  const double *kb_over_eps_jk;         /* [n_spec*n_spec] */
  const double *ZRotF298;               /* [n_spec] */
  /* reactions (Reaction, src/ChemData.h:60-115) */
  const int *reac_type;   /* [n_reac] */
  const int *rev_type;    /* [n_reac] */
  const int *stoi_f;      /* [n_reac*n_spec] */
  const int *stoi_b;      /* [n_reac*n_spec] */
  const int *reac_order;  /* [n_reac] */
  const double *A, *b, *Ea;          /* [n_reac], Ea already divided by R_c */
  const double *A2, *b2, *Ea2;       /* [n_reac] low-pressure / reverse Arrhenius        */
  const double *third_body_coeff;    /* [n_reac*n_spec] */
  const double *troe_alpha, *troe_t3, *troe_t1, *troe_t2; /* [n_reac] */
  /* NASA9 multi-range polynomials (the reference's high-temperature build, therm_nasa_7_9 = 9,
   * Species::read_therm_nasa9, src/ChemData.cpp:865-1034); replace the NASA7 tables above when
   * therm_nasa_7_9 == 9.  Below the first and above the last boundary h is extended linearly
   * with the edge cp and cp is held (src/Thermo.cu:76-112). */
  int therm_nasa_7_9;                 /* 0 or 7: the NASA7 two-range tables; 9: the tables below */
  int max_range;                      /* most temperature ranges of any species (1..4)           */
  const int *n_temperature_range;     /* [n_spec]                                                */
  const double *temperature_range;    /* [n_spec*(max_range+1)] range boundaries [K]             */
  const double *therm_poly_coeff;     /* [n_spec*max_range*9]: a0..a6, b1, b2 of each range      */
  /* Control temperatures of the two-temperature reaction rates (Reaction::tcf_a .. tcb_b, the
   * AIR5 model of src/ChemData.cpp:1247-1262): with the switch on, reaction i runs forward at
   * smooth(T^tcf_a Tve^tcf_b) and backward at smooth(T^tcb_a Tve^tcb_b)
   * (src/FiniteRateChem.cu:1490-1503). */
  int two_temperature_reaction_temperature;
  const double *tcf_a, *tcf_b, *tcb_a, *tcb_b; /* [n_reac] */
} cb2_mechanism;

/* Vibrational-electronic data of the species for the two-temperature model, as
 * cfd::Species::read_two_temperature parses two_temperature.dat (src/ChemData.cpp:130-233).
 * Host arrays, row-major, in the mechanism's species order. */
typedef struct cb2_two_temperature {
  int n_spec;                /* must equal the mechanism's n_spec                       */
  int max_level;             /* row length of elec_theta / elec_g (>= 1)                */
  const double *theta_v;     /* [n_spec] characteristic vibrational temperature, K; <= 0: none */
  const int *n_level;        /* [n_spec] electronic levels of each species              */
  const double *elec_theta;  /* [n_spec*max_level] electronic level temperatures, K     */
  const double *elec_g;      /* [n_spec*max_level] degeneracies                         */
  const double *lt_a, *lt_b; /* [n_spec*n_spec] Millikan-White A_ij, B_ij; <= 0: default */
  const double *park_sigma;  /* [n_spec] Park limiting cross-section, m^2               */
  int enable_vt_relaxation;  /* DParameter::enable_vt_relaxation                        */
} cb2_two_temperature;

/* Scalar settings (the scalar fields of `DParameter`, src/DParameter.cuh:13-160, with the
 * setup.txt meaning given in src/Parameter.cpp:358-546). */
typedef struct cb2_param_view {
  int abi_version;         /* must be CB2_ABI_VERSION */
  int dim;                 /* 1, 2 or 3 (only decides the 2D/3D branches the reference has) */
  int n_var, n_spec, n_scalar, n_scalar_transported;
  int inviscid_scheme;     /* CB2_INV_* */
  int reconstruction;      /* CB2_REC_* (primitive-reconstruction schemes only) */
  int limiter;             /* 0 minmod */
  int viscous_order;       /* 0, 2 or 8 */
  int positive_preserving; /* 0/1: species positivity limiter (characteristic WENO, mixtures) */
  int gradP_in_diffusion_flux;
  int reaction;            /* 0 or 1 (finite-rate chemistry) */
  int shock_sensor;        /* 0 Ducros, 1 Jameson, 2 jump */
  double sensor_eps, sensor_threshold; /* threshold <= 1e-10: WENO weights everywhere */
  double entropy_fix_factor;
  double Pr, cfl;
  double rho_ref, v_ref;   /* rho_inf, v_inf: WENO eps = 1e-40*(rho_ref*v_ref)^2 */
  /* air viscosity: <= 0 -> Sutherland (the reference's only air model,
   * src/FieldOperation.cuh:244); > 0 -> this constant value (added for constant-mu cases) */
  double mu_constant;
  int precision;           /* CB2_PREC_* */
  const cb2_mechanism *mech; /* NULL for the calorically perfect air model */
  /* limit_flow (src/TimeAdvanceFunc.cuh:129-232, bounds src/DParameter.cu:371-387): after each
   * stage update, nodes with NaN or rho, u, v, w, p outside [1e-6, 1e3] x rho_ref / p_ref and
   * +-1000 x velocity scale (v_ref, or c_ref when |v_ref| < 1) take the mean of their good
   * neighbours */
  int limit_flow;
  double p_ref, c_ref;     /* p_inf, speed_of_sound */
  /* time step the positivity limiter starts with (DParameter::dt, the setup's fixed step);
   * cb2_cfl_dt and cb2_rk3_step replace it with the step they take */
  double dt;
  /* two-temperature model (the reference's COREFL_ENABLE_TWO_TEMPERATURE build): NULL for one
   * temperature.  With it the last scalar is the vibrational-electronic energy e_ve
   * (i_eve = n_spec, src/Parameter.cpp:647-656): n_scalar = n_scalar_transported = n_spec + 1,
   * n_var = 6 + n_spec, cv holds rho*e_ve at 5 + n_spec, and zones carry temperature_ve. */
  const cb2_two_temperature *two_t;
} cb2_param_view;

typedef struct cb2_ctx cb2_ctx;

/* ---- life cycle ---------------------------------------------------------------------- */

/* Replaces the construction of `DParameter` (src/DParameter.cu:6-436) as the hot path
 * sees it: validates the scheme combination and copies the scalar settings and the
 * mechanism tables to the device.  Allocates only the library's private tables. */
int cb2_init(const cb2_param_view *param, cb2_ctx **ctx_out);

/* Borrows the device arrays of block `blk` (Field::d_ptr / h_ptr, src/Field.h:164-167)
 * and its face boundary conditions.  Calling it again for the same `blk` rebinds. */
int cb2_bind_block(cb2_ctx *ctx, int blk, const cb2_zone_view *zone, const cb2_face_bc *faces,
                   int n_faces);

/* The inner faces of block `blk` (the Block::inner_face list the reference's Mesh builds):
 * replaces the list that inner_communication reads through DZone::innerFace
 * (src/Field.cu:478-480).  Every target block must be bound when cb2_halo runs; the ranges are
 * checked against both blocks' padded extents then.  Calling it again replaces the list. */
int cb2_bind_inner_faces(cb2_ctx *ctx, int blk, const cb2_inner_face *faces, int n_faces);

void cb2_destroy(cb2_ctx *ctx);

/* ---- the stage pieces (each one replaces one call of RK3, src/RK.cuh) --------------- */

/* qn <- cv: replaces the per-step cudaMemcpy D2D at src/RK.cuh:126-129. */
int cb2_store_qn(cb2_ctx *ctx, int blk, void *stream);

/* dq <- 0, then the viscous (compute_viscous_flux, src/RK.cuh:173), chemistry
 * (finite_rate_chemistry, src/RK.cuh:180) and inviscid (compute_inviscid_flux,
 * src/RK.cuh:186) residual contributions selected by `mask` (CB2_RHS_*). */
int cb2_rhs(cb2_ctx *ctx, int blk, unsigned mask, void *stream);

/* Shock sensor (Ducros / Jameson / density-pressure jump by `shock_sensor`) on the interior
 * nodes: replaces compute_shock_sensor (src/FieldOperation.cu:207-228, src/RK.cuh:139-143).
 * With sensor_threshold > 1e-10 the WENO kernels use nonlinear weights only where the
 * sensor exceeds the threshold within the stencil window, and linear weights elsewhere. */
/* The viscous term of every bound block at once, as the reference's compute_viscous_flux runs over
 * the whole mesh (src/ViscousScheme.cu:14-100): each block's dq becomes its viscous residual (with
 * 8th-order terms: every block's node fluxes, then their exchange across the inner faces
 * (exchange_value task 1, src/DataCommunication.cu:437-527), then each block's periodic node-flux
 * exchange and divergence).  Then, per block, cb2_rhs with CB2_RHS_CHEMISTRY | CB2_RHS_INVISCID |
 * CB2_RHS_ACCUMULATE completes the residual.  Needed for 8th-order viscous terms on grids with
 * inner faces, where cb2_rhs of one block refuses them; cb2_rk3_step and cb2_rk3_run call it
 * themselves. */
int cb2_viscous(cb2_ctx *ctx, void *stream);

int cb2_shock_sensor(cb2_ctx *ctx, int blk, void *stream);

/* Shu-Osher stage `rk` (0,1,2) with time step dt, species clipping and primitive recovery:
 * replaces update_cv_and_bv_rk<mix> (src/RK.cuh:277-367), followed by limit_flow when set.
 * Two-temperature contexts recover T_ve and T with the two-temperature inversion
 * (src/FieldOperation.cu:24-63) and relax e_ve over {1, 1/4, 2/3}[rk] x dt before limit_flow,
 * as RK3 does (apply_vt_relaxation_rk, src/RK.cuh:199-203). */
int cb2_stage_update(cb2_ctx *ctx, int blk, double dt, int rk, void *stream);

/* Two-temperature VT relaxation of every interior node over dt_stage alone: replaces
 * apply_vt_relaxation_rk (src/RK.cuh:20-28, apply_vt_relaxation_1_point,
 * src/FieldOperation.cuh:60-88), for callers that run their own stage update.  e_v relaxes
 * towards equilibrium at T with the Millikan-White + Park time, then T_ve and T follow.
 * CB2_ERR_UNSUPPORTED for one-temperature contexts.
 *
 * Two-temperature contexts (cb2_param_view::two_t) run the characteristic WENO5/WENO7 fluxes,
 * the 2nd- and 8th-order viscous terms, the chemistry, every face condition and the inner-face
 * exchange, and so the whole step (cb2_rk3_step, cb2_rk3_run).  The primitive-variable fluxes
 * (AUSM+, HLLC, Roe), the shock sensor, the autotuner, the batched paths and the 0-D reactors
 * return CB2_ERR_UNSUPPORTED for them. */
int cb2_vt_relaxation(cb2_ctx *ctx, int blk, double dt_stage, void *stream);

/* Ghost fill of bv/sv/cv from the face conditions bound with the block (periodic,
 * outflow, ...): replaces DBoundCond::apply_boundary_conditions (src/BoundCond.cu:3846). */
int cb2_boundary(cb2_ctx *ctx, int blk, void *stream);

/* Device-side copies across the inner faces of every bound block, in block and face order, and
 * for 2-D blocks the k = 0 plane into the k ghost planes afterwards: replaces the inner-face part
 * of data_communication<mix> (src/DataCommunication.cu:6-27, inner_communication :36-124) and the
 * eliminate_k_gradient that follows it (src/RK.cuh:218-226).  cb2_rk3_step and cb2_rk3_run call
 * it after the boundary conditions of every stage.  Grids with inner faces take 2nd-order
 * viscous terms only (the 8th-order node-flux exchange across blocks is not built). */
int cb2_halo(cb2_ctx *ctx, void *stream);

/* gamma, c, Mach, mu, kappa, rho*D over interior and ghosts: replaces
 * update_physical_properties<mix> (src/FieldOperation.cuh:183-247). */
int cb2_properties(cb2_ctx *ctx, int blk, void *stream);

/* cv from bv/sv over interior and ghosts: replaces compute_cv_from_bv<mix>
 * (src/FieldOperation.cuh:136-161); two-temperature contexts first bring e_ve and T_ve into
 * agreement (sync_two_temperature_state_from_sv, :28-58). */
int cb2_cv_from_bv(cb2_ctx *ctx, int blk, void *stream);

/* Metrics and Jacobian of one block from its node coordinates: replaces
 * Block::compute_jac_metric (src/Mesh.cpp:244-528, its 2nd-order branch), which the reference
 * runs on the host.  x, y, z are device arrays on the padded lattice of ghost width g_coord
 * (>= ngg + 1: the ghost coordinates the reference's init_ghost_grid builds, src/Mesh.cpp:1013-1163,
 * filled by the caller); metric (9 comps) and jac receive the values on the ghost-ngg lattice of
 * cb2_zone_view.  Allocates a 4-byte flag, synchronizes the stream, and returns
 * CB2_ERR_NONPHYSICAL if any node's Jacobian is not positive (where the reference aborts). */
int cb2_metrics(const double *x, const double *y, const double *z, int mx, int my, int mz, int g_coord, int ngg,
                double *metric, double *jac, void *stream);

/* The step number the face conditions see (the reference's `step`, src/RK.cuh:69-108: a new run
 * starts from 0, a restart from its step file, and each step counts one before its stages).
 * cb2_rk3_step adds one at its start; cb2_boundary uses the value as it is.  Only the blowing wall
 * reads it; cb2_rk3_run refuses contexts with one.  (ABI version 6) */
int cb2_set_step(cb2_ctx *ctx, long long step);

/* Flowfield file of every bound block (blocks 0 .. n-1, all bound): the reference's
 * output/flowfield.plt (FieldIO::initialize / print_field, src/FieldIO.h:77-470), a Tecplot binary
 * file (version 112, one ordered zone "zone <b>" per block, double data at the nodes) holding x, y,
 * z, density, u, v, w, pressure, temperature, the n_spec species (`species_names`, the mechanism's
 * order), Eve (two temperatures), mach and Tve (two temperatures), over the block's nodes and
 * `ngg_out` ghost layers (the reference writes 0).  xyz[3 b + c] are HOST arrays of block b's
 * coordinates x, y, z, padded like its field arrays (ghost ngg).  The blocks' bv, sv, mach and
 * T_ve are copied to the host over `stream`, which is synchronised.  Error: CB2_ERR_INVALID
 * (bad arguments, no mach array, the file cannot be written). */
int cb2_write_flowfield(cb2_ctx *ctx, const char *path, const double *const *xyz, const char *const *species_names,
                        int ngg_out, double solution_time, void *stream);

/* Restart from a flowfield file (read_flowfield with the same blocks, src/Initialize.cu:167-411): the
 * file's zones must be the bound blocks in order, each with the same number g <= ngg of ghost layers
 * on every side.  Variables are matched by name, ignoring case, as the reference does: density (or
 * rho), u, v, w, pressure (or p), temperature (or t) into bv, the species names into sv, Eve into
 * e_ve's sv slot and Tve into T_ve (two temperatures; without Tve, T_ve is set to 0 so that the next
 * cv-from-bv pass finds it from e_ve); other variables are skipped.  The file's nodes (with its g
 * ghost layers) are overwritten; the rest keeps its values.  The caller then rebuilds cv and the
 * properties (cb2_cv_from_bv, cb2_properties) as after any change of bv.  *solution_time (if not
 * NULL) receives the zones' solution time.  Synchronises `stream`. */
int cb2_read_flowfield(cb2_ctx *ctx, const char *path, const char *const *species_names, double *solution_time,
                       void *stream);

/* Local CFL time step of every node and the min over all bound blocks, returned to the
 * host: replaces local_time_step<mix> + global_time_step (src/TimeAdvanceFunc.cuh:28-127,
 * src/TimeAdvanceFunc.cu:114-139).  Synchronises `stream`. */
int cb2_cfl_dt(cb2_ctx *ctx, double *dt_out, void *stream);

/* Allocation-free minimum of a per-node time-step array (no counterpart in the reference).
 * For callers that may not allocate device memory, e.g. codes that give all device memory
 * to their own pool before the solve, or that cannot afford the device-wide synchronisation
 * of cudaFree while other streams run.  `dt_local` (device, n doubles, e.g. the dt_local
 * array local_time_step fills) is reduced to its minimum, seeded with 1e6 as the reference
 * does, and the result is written to the device double *dt_min.  Nothing is allocated: the
 * partial minima use a fixed device array of CB2_NOALLOC_MAX_PARTIALS doubles (128 KiB) that
 * every GPU loading the library holds until the process exits, so n may not exceed
 * CB2_NOALLOC_MAX_NODES (CB2_ERR_INVALID beyond).  The first call on a device resolves that
 * array's device address, so make it before any stream capture; the address is kept for the
 * process, which assumes the runtime's primary context and no cudaDeviceReset afterwards.  All
 * calls share the array: calls that overlap on the GPU race. */
#define CB2_NOALLOC_MAX_PARTIALS 16384
#define CB2_NOALLOC_MAX_NODES (16384LL * 2048LL)
int cb2_min_dt_noalloc(const double *dt_local, long long n, double *dt_min, void *stream);

/* One whole SSP-RK3 step over all bound blocks (src/RK.cuh:107-237): qn<-cv, [CFL dt],
 * 3 x (rhs, stage update, boundary, properties).  With fixed_dt != 0 the step uses
 * *dt_inout and performs no host synchronisation; otherwise the CFL dt is computed first
 * and written to *dt_inout. */
int cb2_rk3_step(cb2_ctx *ctx, double *dt_inout, int fixed_dt, void *stream);

/* Device-driven time loop (the while loop of RK3<mix>, src/RK.cuh:107-261): up to max_steps
 * SSP-RK3 steps over all bound blocks, stopping once the accumulated time *time_inout
 * reaches t_end (physical_time >= total_simulation_time, src/RK.cuh:257), all in ONE launch of
 * a CUDA graph whose conditional WHILE node repeats a captured step; the loop test runs on
 * the device, so there is no host round trip per step.  With fixed_dt != 0 every step takes
 * dt; otherwise each step computes the CFL dt on the device first (cb2_cfl_dt's kernels) and
 * every bound block needs dt_local.  The loop also ends after a step that sets the status
 * word (clear it first with cb2_read_status) or takes a non-positive or non-finite dt; the
 * call then returns CB2_ERR_NONPHYSICAL and the status word stays set.  On return
 * *time_inout holds the time reached, *steps_out the steps taken and *dt_last_out (may be
 * NULL) the last dt.  Synchronises `stream` once, at the end.  The graph is captured on the
 * first call and again after cb2_bind_block or a change of fixed_dt; the steps give results
 * identical to as many cb2_rk3_step calls.  Per-launch profiling does not see the graph's
 * kernels. */
int cb2_rk3_run(cb2_ctx *ctx, double dt, int fixed_dt, long long max_steps, double t_end, double *time_inout,
                long long *steps_out, double *dt_last_out, void *stream);

/* ---- autotuning (no counterpart in the reference) ----------------------------------------- */

/* Picks, for block `blk`, the y and z sweep tile widths of the primitive-variable WENO5/WENO7
 * air sweeps (4, 8 or 16 i-columns by 64, 32 or 16 nodes along the sweep) by timing every
 * candidate three times with CUDA events on the block's own data.  The candidates write a
 * scratch residual that is allocated for the call and freed after it, so the caller's arrays
 * are untouched.  The widths stay with the block until it is rebound; every width gives the
 * same results bit for bit.  Writes the chosen widths to tile_ni_out[3] (x: 0, the x sweep
 * streams k-planes) when it is not NULL.  Other schemes keep their fixed tiles (CB2_OK).
 * Synchronises `stream`; call it outside stream capture. */
int cb2_autotune(cb2_ctx *ctx, int blk, int *tile_ni_out, void *stream);

/* Sets the widths cb2_autotune would pick (tile_ni[1], tile_ni[2] in {0 = default, 4, 8, 16};
 * tile_ni[0] is ignored), e.g. to reuse the result of an earlier tuning run. */
int cb2_set_tile_widths(cb2_ctx *ctx, int blk, const int *tile_ni);

/* ---- diagnostics --------------------------------------------------------------------- */

/* Reads and clears the device status word that kernels set on non-physical states
 * (bit 0: rho<=0 or non-finite after a stage update; bit 1: T<=0 or Newton failure). */
int cb2_read_status(cb2_ctx *ctx, unsigned *flags_out, void *stream);

const char *cb2_strerror(int code);
const char *cb2_last_cuda_error(void);

/* Number of kernels this context launched since creation (a counter the bench reports). */
unsigned long long cb2_launch_count(const cb2_ctx *ctx);

/* Per-kernel timing, the counterpart of the reference's `profile_rk_breakdown` switch
 * (src/RK.cuh:90-101, 248-255), without its device-wide synchronisations: while enabled,
 * every launch is bracketed by a CUDA event pair on its stream and the durations are
 * aggregated by kernel name.  cb2_profile_count/entry synchronise on the recorded events. */
int cb2_profile_enable(cb2_ctx *ctx, int on);
int cb2_profile_reset(cb2_ctx *ctx);
int cb2_profile_count(cb2_ctx *ctx);
int cb2_profile_entry(cb2_ctx *ctx, int idx, char *name, int name_len, unsigned long long *count,
                      double *total_ms);

#ifdef __cplusplus
}
#endif
#endif /* CB200_H */
