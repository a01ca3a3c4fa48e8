"""ctypes binding of the FP64 host oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg to check or time the CUDA library; never by the library itself.
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "corefl-cpc_b200"))
from cb200 import abi  # noqa: E402

LIB_PATH = os.path.join(HERE, "liboracle.so")
_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            import importlib.util
            spec = importlib.util.spec_from_file_location("oracle_build", os.path.join(HERE, "build.py"))
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            mod.build()
        lib = C.CDLL(LIB_PATH)
        P = C.POINTER
        sig = {
            "oracle_set_threads": (None, [C.c_int]),
            "oracle_set_step": (None, [C.c_longlong]),
            "oracle_max_threads": (C.c_int, []),
            "oracle_stage_update": (C.c_int, [P(abi.ParamView), P(abi.ZoneView), C.c_double, C.c_int]),
            "oracle_cv_from_bv": (C.c_int, [P(abi.ParamView), P(abi.ZoneView)]),
            "oracle_rhs": (C.c_int, [P(abi.ParamView), P(abi.ZoneView), P(abi.FaceBC), C.c_int, C.c_uint]),
            "oracle_boundary": (C.c_int, [P(abi.ParamView), P(abi.ZoneView), P(abi.FaceBC), C.c_int]),
            "oracle_properties": (C.c_int, [P(abi.ParamView), P(abi.ZoneView)]),
            "oracle_shock_sensor": (C.c_int, [P(abi.ParamView), P(abi.ZoneView)]),
            "oracle_cfl_dt": (C.c_int, [P(abi.ParamView), P(abi.ZoneView), P(C.c_double)]),
            "oracle_rk3_step": (C.c_int, [P(abi.ParamView), P(abi.ZoneView), P(abi.FaceBC), P(C.c_int), C.c_int,
                                          P(C.c_double), C.c_int]),
            "oracle_rk3_step_inner": (C.c_int, [P(abi.ParamView), P(abi.ZoneView), P(abi.FaceBC), P(C.c_int),
                                                P(abi.InnerFace), P(C.c_int), C.c_int, P(C.c_double), C.c_int]),
            "oracle_halo": (C.c_int, [P(abi.ParamView), P(abi.ZoneView), P(abi.InnerFace), P(C.c_int), C.c_int]),
            "oracle_nasa7_h_cp": (None, [P(abi.Mechanism), C.c_double, P(C.c_double), P(C.c_double)]),
            "oracle_vt_relaxation": (C.c_int, [P(abi.ParamView), P(abi.ZoneView), C.c_double]),
            "oracle_two_temperature_state": (None, [P(abi.ParamView), C.c_double, C.c_double, C.c_double,
                                                    P(C.c_double), P(C.c_double)]),
            "oracle_species_ve": (None, [P(abi.ParamView), C.c_double, P(C.c_double), P(C.c_double)]),
            "oracle_gibbs_rt": (None, [P(abi.Mechanism), C.c_double, P(C.c_double)]),
        }
        for n, (r, a) in sig.items():
            f = getattr(lib, n)
            f.restype = r
            f.argtypes = a
        _lib = lib
    return _lib


def _faces(faces):
    arr = (abi.FaceBC * max(1, len(faces)))()
    for a, f in enumerate(faces):
        arr[a] = f
    return arr


def set_step(step):
    """The step number the face conditions see (the library's cb2_set_step)."""
    load().oracle_set_step(step)


def set_threads(n):
    load().oracle_set_threads(n)


def max_threads():
    return load().oracle_max_threads()


def rhs(param, block, faces, mask=abi.RHS_ALL):
    v = block.view()
    load().oracle_rhs(C.byref(param), C.byref(v), _faces(faces), len(faces), mask)


def stage_update(param, block, dt, rk):
    v = block.view()
    load().oracle_stage_update(C.byref(param), C.byref(v), dt, rk)


def boundary(param, block, faces):
    v = block.view()
    load().oracle_boundary(C.byref(param), C.byref(v), _faces(faces), len(faces))


def shock_sensor(param, block):
    v = block.view()
    load().oracle_shock_sensor(C.byref(param), C.byref(v))


def properties(param, block):
    v = block.view()
    load().oracle_properties(C.byref(param), C.byref(v))


def vt_relaxation(param, block, dt_stage):
    v = block.view()
    load().oracle_vt_relaxation(C.byref(param), C.byref(v), dt_stage)


def two_temperature_state(param, rho, t, tve, y):
    """(e_ve(T), cv_ve(T), e_ve(Tve), cv_ve(Tve), Tve inverted from e_ve(Tve) starting at T,
    VT source, e_ve equilibrium, effective relaxation time)"""
    yy = np.ascontiguousarray(np.asarray(y, dtype=np.float64))
    out = np.zeros(8)
    P = C.POINTER(C.c_double)
    load().oracle_two_temperature_state(C.byref(param), rho, t, tve, yy.ctypes.data_as(P), out.ctypes.data_as(P))
    return out


def species_ve(param, t):
    ns = param.n_spec
    e, cv = np.zeros(ns), np.zeros(ns)
    P = C.POINTER(C.c_double)
    load().oracle_species_ve(C.byref(param), t, e.ctypes.data_as(P), cv.ctypes.data_as(P))
    return e, cv


def cv_from_bv(param, block):
    v = block.view()
    load().oracle_cv_from_bv(C.byref(param), C.byref(v))


def cfl_dt(param, block):
    v = block.view()
    d = C.c_double()
    load().oracle_cfl_dt(C.byref(param), C.byref(v), C.byref(d))
    return d.value


def rk3_step(param, blocks, faces_per_block, dt, fixed_dt=True):
    views = (abi.ZoneView * len(blocks))(*[b.view() for b in blocks])
    flat = [f for fl in faces_per_block for f in fl]
    nf = (C.c_int * len(blocks))(*[len(fl) for fl in faces_per_block])
    d = C.c_double(dt)
    load().oracle_rk3_step(C.byref(param), views, _faces(flat), nf, len(blocks), C.byref(d), 1 if fixed_dt else 0)
    return d.value


def rk3_step_inner(param, blocks, faces_per_block, inner_per_block, dt, fixed_dt=True):
    """One RK3 step of a multi-block grid with its inner faces (abi.InnerFace lists per block)."""
    views = (abi.ZoneView * len(blocks))(*[b.view() for b in blocks])
    flat = [f for fl in faces_per_block for f in fl]
    nf = (C.c_int * len(blocks))(*[len(fl) for fl in faces_per_block])
    iflat = [f for fl in inner_per_block for f in fl]
    inner = (abi.InnerFace * max(1, len(iflat)))(*iflat)
    ni = (C.c_int * len(blocks))(*[len(fl) for fl in inner_per_block])
    d = C.c_double(dt)
    load().oracle_rk3_step_inner(C.byref(param), views, _faces(flat), nf, inner, ni, len(blocks), C.byref(d),
                                 1 if fixed_dt else 0)
    return d.value


def halo(param, blocks, inner_per_block):
    """The inner-face exchange alone (cb2_halo) over the host blocks."""
    views = (abi.ZoneView * len(blocks))(*[b.view() for b in blocks])
    iflat = [f for fl in inner_per_block for f in fl]
    inner = (abi.InnerFace * max(1, len(iflat)))(*iflat)
    ni = (C.c_int * len(blocks))(*[len(fl) for fl in inner_per_block])
    load().oracle_halo(C.byref(param), views, inner, ni, len(blocks))


def chemistry_source(mech, rho, t, y):
    """(omega, omega_d) [kg/(m^3 s)] of one state from the oracle's finite-rate chemistry."""
    import numpy as np
    lib = load()
    lib.oracle_chemistry_source.restype = None
    P = C.POINTER(C.c_double)
    lib.oracle_chemistry_source.argtypes = [C.POINTER(abi.Mechanism), C.c_double, C.c_double, P, P, P]
    y = np.ascontiguousarray(y, dtype=np.float64)
    om = np.zeros(mech.ns)
    od = np.zeros(mech.ns)
    lib.oracle_chemistry_source(mech.ptr(), rho, t, y.ctypes.data_as(P), om.ctypes.data_as(P), od.ctypes.data_as(P))
    return om, od


def chemistry_source_2t(mech, rho, t, tve, y):
    """(omega, omega_d) of one state at (T, Tve) (the control-temperature rates when the mechanism
    has them)."""
    lib = load()
    lib.oracle_chemistry_source_2t.restype = None
    P = C.POINTER(C.c_double)
    lib.oracle_chemistry_source_2t.argtypes = [C.POINTER(abi.Mechanism), C.c_double, C.c_double, C.c_double, P, P, P]
    y = np.ascontiguousarray(y, dtype=np.float64)
    om = np.zeros(mech.ns)
    od = np.zeros(mech.ns)
    lib.oracle_chemistry_source_2t(mech.ptr(), rho, t, tve, y.ctypes.data_as(P), om.ctypes.data_as(P),
                                   od.ctypes.data_as(P))
    return om, od


def gibbs_rt(mech, t):
    g = np.zeros(mech.ns)
    P = C.POINTER(C.c_double)
    load().oracle_gibbs_rt(mech.ptr(), C.c_double(t), g.ctypes.data_as(P))
    return g


def nasa7_h_cp(mech, t):
    import numpy as np
    h = np.zeros(mech.ns)
    cp = np.zeros(mech.ns)
    P = C.POINTER(C.c_double)
    load().oracle_nasa7_h_cp(mech.ptr(), t, h.ctypes.data_as(P), cp.ctypes.data_as(P))
    return h, cp


def reactor_run(mech, T0, p0, Y, t_end, h0=1e-8, rtol=1e-6, atol=1e-12, max_attempts=10**9, krylov=False):
    """A 0-D constant-volume reactor from (T0, p0, Y) advanced by the oracle's ROK4E integrator;
    returns the state as an abi.Reactor."""
    import numpy as np
    lib = load()
    f = lib.oracle_reactor_run
    f.restype = None
    f.argtypes = [C.POINTER(abi.Mechanism), C.c_double, C.c_double, C.POINTER(C.c_double), C.c_double, C.c_double,
                  C.c_double, C.c_double, C.c_int, C.POINTER(abi.Reactor), C.c_int]
    y = np.ascontiguousarray(Y, dtype=np.float64)
    out = abi.Reactor()
    f(mech.ptr(), T0, p0, y.ctypes.data_as(C.POINTER(C.c_double)), t_end, h0, rtol, atol,
      min(int(max_attempts), 2**31 - 1), C.byref(out), int(bool(krylov)))
    return out


def reactor_run_fixed(mech, T0, p0, Y, t_end, dt, scheme, max_steps=10**9):
    """A 0-D constant-volume reactor from (T0, p0, Y) advanced by the oracle's fixed-step form
    `scheme` (abi.REACTOR_EXPLICIT .. abi.REACTOR_RK3, optionally | abi.REACTOR_CONSERVE_MASS)
    with the step dt; returns the state as an abi.Reactor."""
    import numpy as np
    lib = load()
    f = lib.oracle_reactor_run_fixed
    f.restype = None
    f.argtypes = [C.POINTER(abi.Mechanism), C.c_double, C.c_double, C.POINTER(C.c_double), C.c_double, C.c_double,
                  C.c_int, C.c_int, C.POINTER(abi.Reactor)]
    y = np.ascontiguousarray(Y, dtype=np.float64)
    out = abi.Reactor()
    f(mech.ptr(), T0, p0, y.ctypes.data_as(C.POINTER(C.c_double)), t_end, dt, int(scheme),
      min(int(max_steps), 2**31 - 1), C.byref(out))
    return out
