"""ctypes mirror of include/cb200.h (structs and constants)."""
import ctypes as C

ABI_VERSION = 6

OK = 0
ERR_CUDA, ERR_INVALID, ERR_NONPHYSICAL, ERR_TIMEOUT, ERR_UNSUPPORTED, ERR_NOMEM = -1, -2, -3, -4, -5, -6

INV_ROE, INV_AUSMP, INV_HLLC = 2, 3, 4
INV_WENO5_CP, INV_WENO5_CH, INV_WENO7_CP, INV_WENO7_CH = 51, 52, 71, 72
REC_FIRST, REC_MUSCL, REC_NND2, REC_WENO5, REC_WENO7 = 1, 2, 3, 5, 7
BC_WALL, BC_SYMMETRY, BC_INFLOW, BC_OUTFLOW, BC_PERIODIC = 2, 3, 5, 6, 8
BC_FARFIELD = 4
BC_NONREFLECTING = 0x100  # OR'd into BC_OUTFLOW: non-reflecting outflow
PREC_FP64, PREC_MIXED = 0, 1
RHS_VISCOUS, RHS_CHEMISTRY, RHS_INVISCID, RHS_ALL = 1, 2, 4, 7
RHS_ACCUMULATE = 8  # add to the caller's dq

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)

ZONE_ARRAYS = ("cv", "bv", "sv", "qn", "dq", "metric", "jac", "mul", "thermal_conductivity", "rho_D",
               "acoustic_speed", "gamma", "mach", "fFlux", "gFlux", "hFlux", "vis_flux", "shock_sensor",
               "dt_local", "reaction_timeScale", "entropy_fix_delta", "temperature_ve",
               "thermal_conductivity_ve")


class ZoneView(C.Structure):
    _fields_ = [("mx", C.c_int), ("my", C.c_int), ("mz", C.c_int), ("ngg", C.c_int)] + \
               [(n, C.c_void_p) for n in ZONE_ARRAYS]


class FaceBC(C.Structure):
    _fields_ = [("type", C.c_int), ("face", C.c_int), ("direction", C.c_int),
                ("range_start", C.c_int * 3), ("range_end", C.c_int * 3),
                ("rho", C.c_double), ("u", C.c_double), ("v", C.c_double), ("w", C.c_double),
                ("p", C.c_double), ("T", C.c_double), ("wall_temperature", C.c_double),
                ("wall_temperature_ve", C.c_double), ("sv", C.c_void_p),
                ("blow_shock_wave", C.c_int), ("blow_start_step", C.c_int), ("blow_end_step", C.c_int),
                ("blow_coefficient", C.c_double)]


class InnerFace(C.Structure):
    """cb2_inner_face: an inner face after the reference's register_boundary."""
    _fields_ = [("range_start", C.c_int * 3), ("range_end", C.c_int * 3), ("face", C.c_int), ("direction", C.c_int),
                ("target_start", C.c_int * 3), ("target_end", C.c_int * 3), ("target_block", C.c_int),
                ("target_face", C.c_int), ("target_direction", C.c_int), ("src_tar", C.c_int * 3),
                ("loop_dir", C.c_int * 3), ("target_loop_dir", C.c_int * 3), ("n_point", C.c_int * 3)]


MECH_DOUBLE = ("mw", "low_temp_coeff", "high_temp_coeff", "t_low", "t_mid", "t_high", "geometry",
               "LJ_potent_inv", "vis_coeff", "WjDivWi_to_One4th", "sqrt_WiDivWjPl1Mul8",
               "binary_diffusivity_coeff", "kb_over_eps_jk", "ZRotF298")
MECH_INT = ("reac_type", "rev_type", "stoi_f", "stoi_b", "reac_order")
MECH_REAC = ("A", "b", "Ea", "A2", "b2", "Ea2", "third_body_coeff", "troe_alpha", "troe_t3", "troe_t1", "troe_t2")


MECH_NASA9 = ("temperature_range", "therm_poly_coeff")
MECH_RT = ("tcf_a", "tcf_b", "tcb_a", "tcb_b")


class Mechanism(C.Structure):
    _fields_ = [("n_spec", C.c_int), ("n_reac", C.c_int)] + \
               [(n, _dp) for n in MECH_DOUBLE] + [(n, _ip) for n in MECH_INT] + [(n, _dp) for n in MECH_REAC] + \
               [("therm_nasa_7_9", C.c_int), ("max_range", C.c_int), ("n_temperature_range", _ip)] + \
               [(n, _dp) for n in MECH_NASA9] + [("two_temperature_reaction_temperature", C.c_int)] + \
               [(n, _dp) for n in MECH_RT]


class TwoTemperature(C.Structure):
    _fields_ = [("n_spec", C.c_int), ("max_level", C.c_int), ("theta_v", _dp), ("n_level", _ip),
                ("elec_theta", _dp), ("elec_g", _dp), ("lt_a", _dp), ("lt_b", _dp), ("park_sigma", _dp),
                ("enable_vt_relaxation", C.c_int)]


class ParamView(C.Structure):
    _fields_ = [("abi_version", C.c_int), ("dim", C.c_int), ("n_var", C.c_int), ("n_spec", C.c_int),
                ("n_scalar", C.c_int), ("n_scalar_transported", C.c_int), ("inviscid_scheme", C.c_int),
                ("reconstruction", C.c_int), ("limiter", C.c_int), ("viscous_order", C.c_int),
                ("positive_preserving", C.c_int), ("gradP_in_diffusion_flux", C.c_int), ("reaction", C.c_int),
                ("shock_sensor", C.c_int), ("sensor_eps", C.c_double), ("sensor_threshold", C.c_double),
                ("entropy_fix_factor", C.c_double), ("Pr", C.c_double), ("cfl", C.c_double),
                ("rho_ref", C.c_double), ("v_ref", C.c_double), ("mu_constant", C.c_double),
                ("precision", C.c_int), ("mech", C.POINTER(Mechanism)), ("limit_flow", C.c_int), ("p_ref", C.c_double),
                ("c_ref", C.c_double), ("dt", C.c_double), ("two_t", C.POINTER(TwoTemperature))]


# ---- batched solves (include/cb200_serve.h) ---------------------------------------------------
REACTOR_MAX_SPEC = 9
REACTOR_DONE, REACTOR_NONPHYSICAL = 1, 2
REACTOR_EXPLICIT, REACTOR_EPI, REACTOR_DA, REACTOR_RK3, REACTOR_CONSERVE_MASS = 0, 1, 2, 3, 0x10


class Reactor(C.Structure):
    _fields_ = [("rhoY", C.c_double * REACTOR_MAX_SPEC), ("rho", C.c_double), ("E", C.c_double),
                ("T", C.c_double), ("p", C.c_double), ("time", C.c_double), ("t_end", C.c_double),
                ("h", C.c_double), ("err_last", C.c_double), ("step", C.c_int), ("n_reject", C.c_int),
                ("status", C.c_int), ("pad", C.c_int)]

REQ_REACTOR, REQ_TUBE = 0, 1
TUBE_DONE, TUBE_FAILED = 1, 2


class Request(C.Structure):
    _fields_ = [("kind", C.c_int), ("n_nodes", C.c_int), ("arrival", C.c_double), ("T0", C.c_double),
                ("p0", C.c_double), ("t_end", C.c_double), ("Y", C.c_double * REACTOR_MAX_SPEC),
                ("out_state", C.c_void_p)]


class Result(C.Structure):
    _fields_ = [("t_arrival", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double),
                ("latency", C.c_double), ("T", C.c_double), ("p", C.c_double), ("time", C.c_double),
                ("steps", C.c_int), ("status", C.c_int)]


class ServeStats(C.Structure):
    _fields_ = [("iterations", C.c_longlong), ("peak_pool_bytes", C.c_longlong), ("wall_s", C.c_double)]


class ServeOptions(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_size_t), ("max_tubes", C.c_int), ("max_reactors", C.c_int),
                ("tube_steps_per_launch", C.c_int), ("reactor_attempts_per_launch", C.c_int),
                ("rtol", C.c_double), ("atol", C.c_double), ("h0", C.c_double), ("tube_length", C.c_double),
                ("tube_TL", C.c_double), ("tube_pL", C.c_double), ("tube_TR", C.c_double),
                ("tube_pR", C.c_double), ("tube_Y", C.POINTER(C.c_double)), ("time_limit_s", C.c_double),
                ("stats", C.POINTER(ServeStats))]


BLOCK_DONE, BLOCK_FAILED = 1, 2


class BlockCase(C.Structure):
    _fields_ = [("zone", ZoneView), ("time", C.c_double), ("t_end", C.c_double), ("dt", C.c_double),
                ("last_dt", C.c_double), ("steps", C.c_int), ("status", C.c_int)]
