"""Batched 0-D reactors on the GPU in the fixed-step forms (cb2_reactor_advance_fixed: explicit,
EPI, DA, conserve_mass_corefl, explicit RK3) against the reference's own host functions run
through the same steps (tests/golden/h2_reactor_fixed_runs.json) and against the FP64 oracle."""
import ctypes as C
import json
import os

import numpy as np
import pytest

import cb200
from cb200 import abi, cases
from cb200 import mech as mechmod

from test_reactor_fixed_cpu import FORMS, check_state, final_tolerance, scheme_code

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def runs():
    with open(os.path.join(HERE, "golden", "h2_reactor_fixed_runs.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def h2():
    return mechmod.load_json(os.path.join(HERE, "golden", "h2_li2004.json"))


def _setup(h2, runs, form):
    import torch
    rr = runs["runs"]
    n = len(rr)
    p = cases.make_param(n_var=5 + h2.ns, n_spec=h2.ns, dim=1, inviscid_scheme=abi.INV_HLLC,
                         reconstruction=abi.REC_WENO5, mech=h2.ptr())
    ctx = cb200.Context(p)

    def dev(a):
        return torch.tensor(a, dtype=torch.float64, device="cuda")

    T0, p0 = dev([r["T0"] for r in rr]), dev([r["p0"] for r in rr])
    Y, t_end = dev([r["Y"] for r in rr]), dev([r[form]["t_end"] for r in rr])
    st = torch.zeros(n * C.sizeof(abi.Reactor), dtype=torch.uint8, device="cuda")
    ctx.reactor_setup(st.data_ptr(), n, T0.data_ptr(), p0.data_ptr(), Y.data_ptr(), t_end.data_ptr(),
                      rr[0][form]["dt"])
    return ctx, st, n, (T0, p0, Y, t_end)


def _read(st, n):
    raw = st.cpu().numpy().tobytes()
    return [abi.Reactor.from_buffer_copy(raw, i * C.sizeof(abi.Reactor)) for i in range(n)]


@pytest.mark.parametrize("form", FORMS)
def test_fixed_step_reactors_match_reference_and_oracle(oracle_lib, runs, h2, form):
    import torch
    code = scheme_code(runs["runs"][0][form])
    ctx, st, n, keep = _setup(h2, runs, form)
    ctx.reactor_advance_fixed(st.data_ptr(), n, 100, code)
    torch.cuda.synchronize()
    for s, r in zip(_read(st, n), runs["runs"]):
        check_state(s, r[form]["after_100_steps"], h2.ns, 1e-12)
    # the rest of the run in launches of 7,000 steps
    for _ in range(8):
        ctx.reactor_advance_fixed(st.data_ptr(), n, 7000, code)
    torch.cuda.synchronize()
    for s, r in zip(_read(st, n), runs["runs"]):
        f = r[form]
        assert s.status == abi.REACTOR_DONE
        check_state(s, f["final"], h2.ns, final_tolerance(f["final"]))
        o = oracle_lib.reactor_run_fixed(h2, r["T0"], r["p0"], r["Y"], f["t_end"], f["dt"], code)
        check_state(s, {"step": o.step, "time": o.time, "T": o.T, "p": o.p, "rhoY": list(o.rhoY)[:h2.ns]}, h2.ns,
                    final_tolerance(f["final"]))
    ctx.close()


def test_fixed_step_reactor_refuses_unknown_forms(runs, h2):
    ctx, st, n, keep = _setup(h2, runs, "rk3")
    for bad in (4, abi.REACTOR_RK3 | abi.REACTOR_CONSERVE_MASS, 0x20):
        with pytest.raises(cb200.CB2Error):
            ctx.reactor_advance_fixed(st.data_ptr(), n, 1, bad)
    with pytest.raises(cb200.CB2Error):
        ctx.reactor_advance_fixed(st.data_ptr(), n, 0, abi.REACTOR_EPI)
    ctx.close()
