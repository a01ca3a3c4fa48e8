"""cb2_min_dt_noalloc: the allocation-free minimum of the per-node time steps.

Callers that may not allocate device memory (their own pool owns it all, or a cudaFree
would synchronise the device under other streams) use this entry point instead of the
context's reduction.  It must give the same global time step as cb2_cfl_dt, call after call,
although every call reuses one fixed device scratch array.  This file is collected last so
that a run stopping at its first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import cb200
from cb200 import abi, cases
from cb200.field import DeviceBlock

pytestmark = pytest.mark.gpu


def _bind_noalloc(lib):
    fn = lib.cb2_min_dt_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_longlong, C.c_void_p, C.c_void_p]
    return fn


def test_noalloc_min_dt_matches_context_reduction(oracle_lib):
    import torch
    lib = cb200.load()
    noalloc = _bind_noalloc(lib)
    case = cases.sine_wave(n=40)
    p, hb, faces = case.param, case.blocks[0], case.faces[0]
    oracle_lib.boundary(p, hb, faces)
    dev = DeviceBlock(hb)
    ctx = cb200.Context(p)
    ctx.bind(0, dev.view(), faces)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    n = hb.mx * hb.my * hb.mz
    stream = torch.cuda.current_stream().cuda_stream
    results = []
    for call in range(2):
        if call == 1:
            # a different state between the two calls: the scratch must not carry anything over
            dev.t["bv"][1:4] *= 3.0
            dev.t["cv"][1:4] *= 3.0
        dt_ctx = ctx.cfl_dt(stream)  # existing entry point; also refreshes dt_local
        rc = noalloc(dev.t["dt_local"].data_ptr(), n, out.data_ptr(), stream)
        assert rc == abi.OK, lib.cb2_strerror(rc)
        torch.cuda.synchronize()
        dt_na = float(out.item())
        # a minimum is exact: both reductions must return the same double
        assert dt_na == dt_ctx, (call, dt_na, dt_ctx)
        assert dt_na == float(dev.t["dt_local"].min().item())
        results.append(dt_na)
    assert results[1] < results[0]  # faster flow, smaller CFL step
    ctx.close()


def test_noalloc_rejects_oversized_input():
    import torch
    lib = cb200.load()
    noalloc = _bind_noalloc(lib)
    buf = torch.ones(16, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    too_big = 16384 * 2048 + 1
    assert noalloc(buf.data_ptr(), too_big, out.data_ptr(), None) == abi.ERR_INVALID
    assert noalloc(buf.data_ptr(), 0, out.data_ptr(), None) == abi.ERR_INVALID
    assert noalloc(None, 16, out.data_ptr(), None) == abi.ERR_INVALID
