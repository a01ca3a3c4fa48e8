"""Batched 0-D reactors on the GPU (cb2_reactor_setup / cb2_reactor_advance) against the
reference's own host functions run through the same ROK4E sequence
(tests/golden/h2_reactor_runs.json) and against the FP64 oracle."""
import ctypes as C
import json
import os

import numpy as np
import pytest

import cb200
from cb200 import abi, cases
from cb200 import mech as mechmod

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def runs():
    with open(os.path.join(HERE, "golden", "h2_reactor_runs.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def h2():
    return mechmod.load_json(os.path.join(HERE, "golden", "h2_li2004.json"))


def _batch(h2, runs, order=None):
    import torch
    rr = runs["runs"] if order is None else [runs["runs"][i] for i in order]
    n = len(rr)
    p = cases.make_param(n_var=5 + h2.ns, n_spec=h2.ns, dim=1, inviscid_scheme=abi.INV_HLLC,
                         reconstruction=abi.REC_WENO5, mech=h2.ptr())
    ctx = cb200.Context(p)

    def dev(a):
        return torch.tensor(a, dtype=torch.float64, device="cuda")

    T0, p0 = dev([r["T0"] for r in rr]), dev([r["p0"] for r in rr])
    Y, t_end = dev([r["Y"] for r in rr]), dev([r["t_end"] for r in rr])
    st = torch.zeros(n * C.sizeof(abi.Reactor), dtype=torch.uint8, device="cuda")
    ctx.reactor_setup(st.data_ptr(), n, T0.data_ptr(), p0.data_ptr(), Y.data_ptr(), t_end.data_ptr(), runs["h0"])
    return ctx, st, n, (T0, p0, Y, t_end)


def _read(st, n):
    raw = st.cpu().numpy().tobytes()
    return [abi.Reactor.from_buffer_copy(raw, i * C.sizeof(abi.Reactor)) for i in range(n)]


def test_reactor_struct_size():
    assert C.sizeof(abi.Reactor) == 9 * 8 + 8 * 8 + 4 * 4


def test_gpu_reactors_first_attempts_match_reference_and_oracle(oracle_lib, runs, h2):
    ctx, st, n, keep = _batch(h2, runs)
    ctx.reactor_advance(st.data_ptr(), n, 8, runs["rtol"], runs["atol"])
    out = _read(st, n)
    # the step controller takes err^0.1 and err^-0.175 of the error norm, so ulp differences
    # between the device and host arithmetic move the step sizes at the 1e-10 level
    for r, s in zip(runs["runs"], out):
        g = r["after_8_attempts"]
        assert s.step == g["step"] and s.n_reject == g["n_reject"]
        assert abs(s.time - g["time"]) <= 1e-9 * g["time"]
        assert abs(s.T - g["T"]) <= 1e-9 * g["T"]
        o = oracle_lib.reactor_run(h2, r["T0"], r["p0"], r["Y"], r["t_end"], runs["h0"], runs["rtol"], runs["atol"],
                                   max_attempts=8)
        rel = np.abs(np.array(list(s.rhoY)[:h2.ns]) - np.array(list(o.rhoY)[:h2.ns])).max() / max(o.rhoY)
        assert rel < 1e-9, rel
        assert abs(s.T - o.T) <= 1e-9 * o.T
    ctx.close()


def test_gpu_reactors_run_to_end_like_reference(runs, h2):
    import torch
    ctx, st, n, keep = _batch(h2, runs)
    for _ in range(20):
        ctx.reactor_advance(st.data_ptr(), n, 20000, runs["rtol"], runs["atol"])
        torch.cuda.synchronize()
        if all(s.status & abi.REACTOR_DONE for s in _read(st, n)):
            break
    out = _read(st, n)
    for r, s in zip(runs["runs"], out):
        g = r["final"]
        assert s.status == abi.REACTOR_DONE
        assert abs(s.T - g["T"]) <= 1e-5 * g["T"], (s.T, g["T"])
        assert abs(s.p - g["p"]) <= 1e-5 * g["p"]
    ctx.close()


def test_gpu_reactor_result_same_alone_and_in_a_batch(runs, h2):
    """Each reactor is advanced by its own thread: the batch composition cannot change it."""
    import torch
    ctx1, st1, n1, k1 = _batch(h2, runs, order=[3])
    ctxn, stn, nn, kn = _batch(h2, runs, order=[5, 3, 1, 8, 0])
    for ctx, st, n in ((ctx1, st1, n1), (ctxn, stn, nn)):
        ctx.reactor_advance(st.data_ptr(), n, 500, runs["rtol"], runs["atol"])
    torch.cuda.synchronize()
    alone, mixed = _read(st1, 1)[0], _read(stn, nn)[1]
    assert bytes(alone) == bytes(mixed)
    ctx1.close()
    ctxn.close()


def test_krylov_reactors_match_reference_and_oracle(oracle_lib, h2):
    """cb2_reactor_advance_krylov (build_arnoldi = 1) against the reference's cfd::buildArnoldi
    sequence (tests/golden/h2_reactor_krylov_runs.json) and the oracle: the same accepted and
    rejected attempts; the accepted time to 25% only: this form's error norm is dominated by
    last-bit differences of the finite-difference products (eps = 1e-6), which the step
    controller turns into step sizes (11% apart after 8 attempts on the device).  The states are
    taken at those slightly different times: T to 1e-8 after 8 attempts and 1e-4 after 2000, the
    major partial densities to 10x that of the largest."""
    import torch
    with open(os.path.join(HERE, "golden", "h2_reactor_krylov_runs.json")) as f:
        kr = json.load(f)
    ctx, st, n, keep = _batch(h2, kr)
    ctx.reactor_advance_krylov(st.data_ptr(), n, 8, kr["rtol"], kr["atol"])
    torch.cuda.synchronize()
    got8 = _read(st, n)
    ctx.reactor_advance_krylov(st.data_ptr(), n, 1992, kr["rtol"], kr["atol"])
    torch.cuda.synchronize()
    got2000 = _read(st, n)
    for i, r in enumerate(kr["runs"]):
        for s, key, n_att, tol in ((got8[i], "after_8_attempts", 8, 1e-8),
                                   (got2000[i], "after_2000_attempts", 2000, 1e-4)):
            g = r[key]
            o = oracle_lib.reactor_run(h2, r["T0"], r["p0"], r["Y"], r["t_end"], kr["h0"], kr["rtol"], kr["atol"],
                                       max_attempts=n_att, krylov=True)
            for ref in (g, {"T": o.T, "time": o.time, "step": o.step, "n_reject": o.n_reject,
                            "rhoY": list(o.rhoY)[:h2.ns]}):
                assert s.step == ref["step"] and s.n_reject == ref["n_reject"], key
                assert abs(s.T - ref["T"]) <= tol * ref["T"], (key, s.T, ref["T"])
                rho_y, ref_y = np.array(list(s.rhoY)[:h2.ns]), np.array(ref["rhoY"])
                major = ref_y > 1e-3 * ref_y.max()
                assert np.abs(rho_y - ref_y)[major].max() <= 10 * tol * ref_y.max(), key
                assert abs(s.time - ref["time"]) <= 0.25 * ref["time"], key
    ctx.close()
