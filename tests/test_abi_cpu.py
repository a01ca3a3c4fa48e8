"""The C-ABI library loads and exports every symbol include/*.h declares, and argument
validation fails cleanly without touching a GPU."""
import ctypes as C
import os
import re

import pytest

import cb200
from cb200 import abi, cases, mech as mechmod

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(REPO, "include")
    for f in sorted(os.listdir(inc)):
        if f.endswith(".h"):
            hdr = re.sub(r"/\*.*?\*/", "", open(os.path.join(inc, f)).read(), flags=re.S)
            names.update(re.findall(r"\b(cb2_\w+)\s*\(", hdr))
    return sorted(names)


def test_library_exports_every_declared_symbol(cb200_lib):
    names = declared_symbols()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(cb200_lib, n)]
    assert not missing, missing


def test_struct_sizes_match_header():
    # 4 ints + 22 pointers; 3 ints + 6 ints + 7 doubles; versioned param view
    assert C.sizeof(abi.ZoneView) == 4 * 4 + 23 * 8
    # n_spec, n_reac; the NASA7, transport and reaction tables; the NASA9 header (two ints), its
    # three tables; the control-temperature switch (padded) and its four tables
    n_tab = len(abi.MECH_DOUBLE) + len(abi.MECH_INT) + len(abi.MECH_REAC)
    assert C.sizeof(abi.Mechanism) == 2 * 4 + n_tab * 8 + 2 * 4 + 3 * 8 + 8 + 4 * 8
    # 2 ints, 7 pointers, 1 int (padded to 8)
    assert C.sizeof(abi.TwoTemperature) == 2 * 4 + 7 * 8 + 8
    # 36 bytes of ints padded to 8, 8 doubles, a pointer, then the blowing wall's 3 ints padded to 8 and a double
    assert C.sizeof(abi.FaceBC) == 4 * 9 + 4 + 8 * 8 + 8 + 3 * 4 + 4 + 8
    assert C.sizeof(abi.InnerFace) == 4 * 29
    assert abi.ParamView.abi_version.offset == 0


def test_serve_struct_sizes_match_header():
    # sizes of include/cb200_serve.h's structs as a C compiler lays them out (x86-64)
    assert C.sizeof(abi.Reactor) == 152
    assert C.sizeof(abi.Request) == 120
    assert C.sizeof(abi.Result) == 64
    assert C.sizeof(abi.ServeOptions) == 112


def test_serve_rejects_bad_arguments(cb200_lib):
    f = cb200_lib.cb2_serve_run
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(abi.Request), C.c_int, C.POINTER(abi.ServeOptions),
                  C.POINTER(abi.Result)]
    reqs = (abi.Request * 1)()
    out = (abi.Result * 1)()
    opt = abi.ServeOptions()
    assert f(None, None, reqs, 1, C.byref(opt), out) == abi.ERR_INVALID  # a reactor without a context
    reqs[0].kind = 7
    assert f(None, None, reqs, 1, C.byref(opt), out) == abi.ERR_INVALID
    reqs[0].kind, reqs[0].n_nodes = abi.REQ_TUBE, 3  # too few nodes
    assert f(None, None, reqs, 1, C.byref(opt), out) == abi.ERR_INVALID
    assert f(None, None, reqs, 0, C.byref(opt), out) == abi.OK


def test_init_rejects_bad_arguments(cb200_lib):
    h = C.c_void_p()
    assert cb200_lib.cb2_init(None, C.byref(h)) == abi.ERR_INVALID
    p = cases.make_param()
    p.abi_version = 999
    assert cb200_lib.cb2_init(C.byref(p), C.byref(h)) == abi.ERR_INVALID
    p = cases.make_param(n_var=7)  # n_var must be 5 + n_spec
    assert cb200_lib.cb2_init(C.byref(p), C.byref(h)) == abi.ERR_UNSUPPORTED
    p = cases.make_param(inviscid_scheme=abi.INV_AUSMP, reconstruction=4)
    assert cb200_lib.cb2_init(C.byref(p), C.byref(h)) == abi.ERR_INVALID
    p = cases.make_param(viscous_order=3)
    assert cb200_lib.cb2_init(C.byref(p), C.byref(h)) == abi.ERR_INVALID
    p = cases.make_param(precision=7)
    assert cb200_lib.cb2_init(C.byref(p), C.byref(h)) == abi.ERR_INVALID
    # the mixed form covers the WENO5/7 primitive sweeps; the characteristic path stays FP64 only
    p = cases.make_param(inviscid_scheme=abi.INV_WENO5_CH, precision=abi.PREC_MIXED)
    assert cb200_lib.cb2_init(C.byref(p), C.byref(h)) == abi.ERR_UNSUPPORTED
    p = cases.make_param(inviscid_scheme=abi.INV_AUSMP, reconstruction=abi.REC_MUSCL, precision=abi.PREC_MIXED)
    assert cb200_lib.cb2_init(C.byref(p), C.byref(h)) == abi.ERR_UNSUPPORTED
    # two-temperature: e_ve is one more scalar and conservative variable, FP64 only
    gold = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    h2 = mechmod.load_json(os.path.join(gold, "h2_li2004.json"))
    tt = mechmod.load_two_temperature_json(os.path.join(gold, "h2_two_temperature.json"))
    p = cases.make_param(n_var=5 + h2.ns, n_spec=h2.ns, mech=h2.ptr(), two_t=tt.ptr(), inviscid_scheme=abi.INV_HLLC,
                         reconstruction=abi.REC_WENO5)
    assert cb200_lib.cb2_init(C.byref(p), C.byref(h)) == abi.ERR_INVALID
    p = cases.make_param(n_var=6 + h2.ns, n_spec=h2.ns, mech=h2.ptr(), two_t=tt.ptr(), inviscid_scheme=abi.INV_HLLC,
                         reconstruction=abi.REC_WENO5, precision=abi.PREC_MIXED)
    assert cb200_lib.cb2_init(C.byref(p), C.byref(h)) == abi.ERR_UNSUPPORTED
    p = cases.make_param(n_var=6, n_spec=0, two_t=tt.ptr())  # needs a mechanism
    assert cb200_lib.cb2_init(C.byref(p), C.byref(h)) == abi.ERR_INVALID
    assert not h.value


def test_strerror_covers_codes(cb200_lib):
    for code in (abi.OK, abi.ERR_CUDA, abi.ERR_INVALID, abi.ERR_NONPHYSICAL, abi.ERR_TIMEOUT,
                 abi.ERR_UNSUPPORTED, abi.ERR_NOMEM):
        assert cb200_lib.cb2_strerror(code).decode() != "unknown error"


def test_null_context_calls_are_invalid(cb200_lib):
    assert cb200_lib.cb2_rhs(None, 0, abi.RHS_ALL, None) == abi.ERR_INVALID
    assert cb200_lib.cb2_stage_update(None, 0, 1e-3, 0, None) == abi.ERR_INVALID
    assert cb200_lib.cb2_boundary(None, 0, None) == abi.ERR_INVALID
    d = C.c_double(0.0)
    assert cb200_lib.cb2_rk3_step(None, C.byref(d), 1, None) == abi.ERR_INVALID
    t, n = C.c_double(0.0), C.c_longlong(0)
    assert cb200_lib.cb2_rk3_run(None, 1e-3, 1, 10, 1.0, C.byref(t), C.byref(n), None, None) == abi.ERR_INVALID
    assert cb200_lib.cb2_launch_count(None) == 0
