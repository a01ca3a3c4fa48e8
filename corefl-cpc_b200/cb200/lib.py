"""ctypes binding of libcb200.so.

The shared library is the product: if it is missing this module raises instead of falling
back to anything else.
"""
import ctypes as C
import os

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "libcb200.so")
_lib = None


class CB2Error(RuntimeError):
    def __init__(self, code, what):
        self.code = code
        lib = load()
        msg = lib.cb2_strerror(code).decode()
        if code == abi.ERR_CUDA:
            msg += ": " + lib.cb2_last_cuda_error().decode()
        super().__init__(f"{what} failed ({code}): {msg}")


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} is not built; run corefl-cpc_b200/build.py")
    lib = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    P = C.POINTER
    sig = {
        "cb2_init": (C.c_int, [P(abi.ParamView), P(vp)]),
        "cb2_bind_block": (C.c_int, [vp, C.c_int, P(abi.ZoneView), P(abi.FaceBC), C.c_int]),
        "cb2_destroy": (None, [vp]),
        "cb2_store_qn": (C.c_int, [vp, C.c_int, vp]),
        "cb2_rhs": (C.c_int, [vp, C.c_int, C.c_uint, vp]),
        "cb2_viscous": (C.c_int, [vp, vp]),
        "cb2_set_step": (C.c_int, [vp, C.c_longlong]),
        "cb2_shock_sensor": (C.c_int, [vp, C.c_int, vp]),
        "cb2_stage_update": (C.c_int, [vp, C.c_int, C.c_double, C.c_int, vp]),
        "cb2_boundary": (C.c_int, [vp, C.c_int, vp]),
        "cb2_vt_relaxation": (C.c_int, [vp, C.c_int, C.c_double, vp]),
        "cb2_autotune": (C.c_int, [vp, C.c_int, P(C.c_int), vp]),
        "cb2_block_batch_advance": (C.c_int, [vp, vp, C.c_int, C.c_int, vp]),
        "cb2_block_batch_autotune": (C.c_int, [vp, vp, C.c_int, P(C.c_int), vp]),
        "cb2_block_batch_set_schedule": (C.c_int, [vp, C.c_int, C.c_int]),
        "cb2_set_tile_widths": (C.c_int, [vp, C.c_int, P(C.c_int)]),
        "cb2_properties": (C.c_int, [vp, C.c_int, vp]),
        "cb2_cv_from_bv": (C.c_int, [vp, C.c_int, vp]),
        "cb2_cfl_dt": (C.c_int, [vp, P(C.c_double), vp]),
        "cb2_rk3_step": (C.c_int, [vp, P(C.c_double), C.c_int, vp]),
        "cb2_rk3_run": (C.c_int, [vp, C.c_double, C.c_int, C.c_longlong, C.c_double, P(C.c_double),
                                  P(C.c_longlong), P(C.c_double), vp]),
        "cb2_read_status": (C.c_int, [vp, P(C.c_uint), vp]),
        "cb2_strerror": (C.c_char_p, [C.c_int]),
        "cb2_last_cuda_error": (C.c_char_p, []),
        "cb2_launch_count": (C.c_ulonglong, [vp]),
        "cb2_profile_enable": (C.c_int, [vp, C.c_int]),
        "cb2_profile_reset": (C.c_int, [vp]),
        "cb2_profile_count": (C.c_int, [vp]),
        "cb2_profile_entry": (C.c_int, [vp, C.c_int, C.c_char_p, C.c_int, P(C.c_ulonglong), P(C.c_double)]),
        "cb2_reactor_setup": (C.c_int, [vp, vp, C.c_int, vp, vp, vp, vp, C.c_double, vp]),
        "cb2_reactor_advance": (C.c_int, [vp, vp, C.c_int, C.c_int, C.c_double, C.c_double, vp]),
        "cb2_reactor_advance_fixed": (C.c_int, [vp, vp, C.c_int, C.c_int, C.c_int, vp]),
        "cb2_reactor_advance_krylov": (C.c_int, [vp, vp, C.c_int, C.c_int, C.c_double, C.c_double, vp]),
        "cb2_metrics": (C.c_int, [vp, vp, vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp, vp]),
        "cb2_write_flowfield": (C.c_int, [vp, C.c_char_p, P(vp), P(C.c_char_p), C.c_int, C.c_double, vp]),
        "cb2_read_flowfield": (C.c_int, [vp, C.c_char_p, P(C.c_char_p), P(C.c_double), vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def metrics(x, y, z, mx, my, mz, g_coord, ngg, metric, jac, stream=None):
    """cb2_metrics on device tensors: x, y, z on the ghost-g_coord lattice, metric [9, ...] and jac
    on the ghost-ngg lattice (written)."""
    lib = load()
    check(lib.cb2_metrics(x.data_ptr(), y.data_ptr(), z.data_ptr(), mx, my, mz, g_coord, ngg, metric.data_ptr(),
                          jac.data_ptr(), stream), "cb2_metrics")


def check(rc, what):
    if rc != abi.OK:
        raise CB2Error(rc, what)


class Context:
    """Owns one cb2_ctx; blocks are bound by index."""

    def __init__(self, param: abi.ParamView):
        self.lib = load()
        self._param = param  # keep the mechanism arrays alive
        h = C.c_void_p()
        check(self.lib.cb2_init(C.byref(param), C.byref(h)), "cb2_init")
        self.h = h
        self._keep = {}

    def bind(self, blk, zone_view, faces):
        from .field import faces_array
        arr = faces_array(faces)
        # the faces' scalar arrays (inflow states) must stay alive until the library copies them
        self._keep[blk] = (zone_view, arr, [getattr(f, "_sv_keep", None) for f in faces])
        check(self.lib.cb2_bind_block(self.h, blk, C.byref(zone_view), arr, len(faces)), "cb2_bind_block")

    def bind_inner_faces(self, blk, faces):
        """Inner faces (abi.InnerFace, registered form) of block blk (cb2_bind_inner_faces)."""
        arr = (abi.InnerFace * max(1, len(faces)))(*faces)
        self._keep[("inner", blk)] = arr
        check(self.lib.cb2_bind_inner_faces(self.h, blk, arr, len(faces)), "cb2_bind_inner_faces")

    def halo(self, stream=None):
        check(self.lib.cb2_halo(self.h, stream), "cb2_halo")

    def rhs(self, blk, mask=abi.RHS_ALL, stream=None):
        check(self.lib.cb2_rhs(self.h, blk, mask, stream), "cb2_rhs")

    def set_step(self, step):
        """cb2_set_step: the step number the face conditions see."""
        check(self.lib.cb2_set_step(self.h, step), "cb2_set_step")

    def viscous(self, stream=None):
        """cb2_viscous: the viscous term of every bound block (node fluxes exchanged across inner faces)."""
        check(self.lib.cb2_viscous(self.h, stream), "cb2_viscous")

    def shock_sensor(self, blk, stream=None):
        check(self.lib.cb2_shock_sensor(self.h, blk, stream), "cb2_shock_sensor")

    def stage_update(self, blk, dt, rk, stream=None):
        check(self.lib.cb2_stage_update(self.h, blk, dt, rk, stream), "cb2_stage_update")

    def autotune(self, blk=0, stream=None):
        """Tile widths of the block's y/z sweeps picked by timing (cb2_autotune)."""
        out = (C.c_int * 3)()
        check(self.lib.cb2_autotune(self.h, blk, out, stream), "cb2_autotune")
        return list(out)

    def block_batch_advance(self, cases, max_steps, stream=None):
        """Advance a ctypes array of abi.BlockCase in one persistent launch (cb2_block_batch_advance)."""
        check(self.lib.cb2_block_batch_advance(self.h, C.cast(cases, C.c_void_p), len(cases), max_steps, stream),
              "cb2_block_batch_advance")

    def block_batch_autotune(self, cases, stream=None):
        """(tile width, cluster size) picked by timing the batch's residual phase."""
        out = (C.c_int * 2)()
        check(self.lib.cb2_block_batch_autotune(self.h, C.cast(cases, C.c_void_p), len(cases), out, stream),
              "cb2_block_batch_autotune")
        return out[0], out[1]

    def block_batch_set_schedule(self, ni, cluster):
        check(self.lib.cb2_block_batch_set_schedule(self.h, ni, cluster), "cb2_block_batch_set_schedule")

    def set_tile_widths(self, blk, widths):
        arr = (C.c_int * 3)(*widths)
        check(self.lib.cb2_set_tile_widths(self.h, blk, arr), "cb2_set_tile_widths")

    def vt_relaxation(self, blk, dt_stage, stream=None):
        check(self.lib.cb2_vt_relaxation(self.h, blk, dt_stage, stream), "cb2_vt_relaxation")

    def boundary(self, blk, stream=None):
        check(self.lib.cb2_boundary(self.h, blk, stream), "cb2_boundary")

    def properties(self, blk, stream=None):
        check(self.lib.cb2_properties(self.h, blk, stream), "cb2_properties")

    def cv_from_bv(self, blk, stream=None):
        check(self.lib.cb2_cv_from_bv(self.h, blk, stream), "cb2_cv_from_bv")

    def write_flowfield(self, path, xyz, species_names=(), ngg_out=0, solution_time=0.0, stream=None):
        """cb2_write_flowfield: xyz = per block (x, y, z) float64 host arrays padded like the fields."""
        import numpy as np
        keep = [np.ascontiguousarray(a, dtype=np.float64) for blk in xyz for a in blk]
        ptrs = (C.c_void_p * len(keep))(*[a.ctypes.data for a in keep])
        names = (C.c_char_p * max(1, len(species_names)))(*[n.encode() for n in species_names])
        check(self.lib.cb2_write_flowfield(self.h, str(path).encode(), ptrs, names, ngg_out, solution_time, stream),
              "cb2_write_flowfield")

    def read_flowfield(self, path, species_names=(), stream=None):
        """cb2_read_flowfield; returns the file's solution time."""
        names = (C.c_char_p * max(1, len(species_names)))(*[n.encode() for n in species_names])
        t = C.c_double(0.0)
        check(self.lib.cb2_read_flowfield(self.h, str(path).encode(), names, C.byref(t), stream),
              "cb2_read_flowfield")
        return t.value

    def store_qn(self, blk, stream=None):
        check(self.lib.cb2_store_qn(self.h, blk, stream), "cb2_store_qn")

    def cfl_dt(self, stream=None):
        dt = C.c_double()
        check(self.lib.cb2_cfl_dt(self.h, C.byref(dt), stream), "cb2_cfl_dt")
        return dt.value

    def rk3_step(self, dt, fixed_dt=True, stream=None):
        d = C.c_double(dt)
        check(self.lib.cb2_rk3_step(self.h, C.byref(d), 1 if fixed_dt else 0, stream), "cb2_rk3_step")
        return d.value

    def rk3_run(self, max_steps, t_end=float("inf"), time=0.0, dt=0.0, fixed_dt=False, stream=None):
        """Device-driven loop of up to max_steps steps until time >= t_end (one graph launch).
        Returns (time reached, steps taken, last dt)."""
        t = C.c_double(time)
        n = C.c_longlong(0)
        d = C.c_double(0.0)
        check(self.lib.cb2_rk3_run(self.h, dt, 1 if fixed_dt else 0, max_steps, t_end, C.byref(t), C.byref(n),
                                   C.byref(d), stream), "cb2_rk3_run")
        return t.value, n.value, d.value

    def reactor_setup(self, reactors, n, T0, p0, Y, t_end, h0=1e-8, stream=None):
        """Set n reactors (device pointer to abi.Reactor[n]) from device pointers T0, p0, Y
        (n x n_spec mass fractions) and t_end."""
        check(self.lib.cb2_reactor_setup(self.h, reactors, n, T0, p0, Y, t_end, h0, stream), "cb2_reactor_setup")

    def reactor_advance(self, reactors, n, max_attempts, rtol=1e-6, atol=1e-12, stream=None):
        check(self.lib.cb2_reactor_advance(self.h, reactors, n, max_attempts, rtol, atol, stream),
              "cb2_reactor_advance")

    def reactor_advance_krylov(self, reactors, n, max_attempts, rtol=1e-6, atol=1e-12, stream=None):
        """reactor_advance with the Jacobian projected on an Arnoldi basis (build_arnoldi = 1)."""
        check(self.lib.cb2_reactor_advance_krylov(self.h, reactors, n, max_attempts, rtol, atol, stream),
              "cb2_reactor_advance_krylov")

    def reactor_advance_fixed(self, reactors, n, max_steps, scheme, stream=None):
        """At most max_steps fixed steps (dt = each reactor's h) of the form `scheme`
        (abi.REACTOR_EXPLICIT .. abi.REACTOR_RK3, optionally | abi.REACTOR_CONSERVE_MASS)."""
        check(self.lib.cb2_reactor_advance_fixed(self.h, reactors, n, max_steps, scheme, stream),
              "cb2_reactor_advance_fixed")

    def read_status(self, stream=None):
        f = C.c_uint()
        check(self.lib.cb2_read_status(self.h, C.byref(f), stream), "cb2_read_status")
        return f.value

    def launch_count(self):
        return int(self.lib.cb2_launch_count(self.h))

    def profile(self, on=True):
        check(self.lib.cb2_profile_enable(self.h, 1 if on else 0), "cb2_profile_enable")

    def profile_reset(self):
        check(self.lib.cb2_profile_reset(self.h), "cb2_profile_reset")

    def profile_read(self):
        """{kernel name: (launches, total ms)} of the launches recorded while profiling."""
        out = {}
        n = self.lib.cb2_profile_count(self.h)
        buf = C.create_string_buffer(128)
        cnt, ms = C.c_ulonglong(), C.c_double()
        for i in range(n):
            check(self.lib.cb2_profile_entry(self.h, i, buf, 128, C.byref(cnt), C.byref(ms)), "cb2_profile_entry")
            out[buf.value.decode()] = (int(cnt.value), float(ms.value))
        return out

    def close(self):
        if self.h:
            self.lib.cb2_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
