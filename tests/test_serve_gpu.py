"""Served solves (cb2_serve_run): the batched 1-D tube kernel against the block path on the
same case, results that do not depend on the batch they were served in, and the served reactors
against the reference-driven golden runs."""
import ctypes as C
import json
import os

import numpy as np
import pytest

import cb200
from cb200 import abi, cases, serve
from cb200 import mech as mechmod
from cb200.field import DeviceBlock

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def h2():
    return mechmod.load_json(os.path.join(HERE, "golden", "h2_li2004.json"))


def _ctx_tube(h2):
    p = cases.make_param(n_var=5 + h2.ns, n_spec=h2.ns, dim=2, inviscid_scheme=abi.INV_HLLC,
                         reconstruction=abi.REC_WENO5, cfl=0.5, mech=h2.ptr())
    p.reaction = 1
    return cb200.Context(p)


def _tube_req(n, t_end, arrival=0.0, out=None):
    r = abi.Request()
    r.kind, r.n_nodes, r.t_end, r.arrival = abi.REQ_TUBE, n, t_end, arrival
    if out is not None:
        r.out_state = out.ctypes.data
    return r


def _reactor_req(h2, T0, p0, phi, t_end, arrival=0.0, out=None):
    r = abi.Request()
    r.kind, r.T0, r.p0, r.t_end, r.arrival = abi.REQ_REACTOR, T0, p0, t_end, arrival
    y = serve.h2_air_y(h2, phi)
    for s in range(h2.ns):
        r.Y[s] = y[s]
    if out is not None:
        r.out_state = C.addressof(out)
    return r


def test_served_tube_matches_block_path(h2):
    """The one-CTA tube kernel against cb2_rk3_step on the same one-row reactive shock tube."""
    import torch
    n, steps = 300, 20
    case = cases.reactive_shock_tube(h2, n_nodes=n)
    p, hb, faces = case.param, case.blocks[0], case.faces[0]
    dev = DeviceBlock(hb)
    ctx = cb200.Context(p)
    ctx.bind(0, dev.view(), faces)
    ctx.properties(0)
    t = 0.0
    for _ in range(steps):
        t += ctx.rk3_step(0.0, fixed_dt=False)
    torch.cuda.synchronize()
    g = hb.ngg
    ref_bv = dev.t["bv"][:, g, g, g:g + n].cpu().numpy()
    out = np.zeros((6 + h2.ns) * n)
    ctx_t = _ctx_tube(h2)
    opt = serve.options(h2, hbm_budget=1 << 28, tube_steps=7)
    # t_end just short of the block path's time after `steps` steps: the served tube stops at
    # the first step that reaches it, which is step `steps`
    res, st = serve.serve(None, ctx_t, [_tube_req(n, t * (1 - 1e-9), out=out)], opt)
    assert res[0].status == abi.TUBE_DONE
    assert res[0].steps == steps, (res[0].steps, steps)
    assert abs(res[0].time - t) <= 1e-12 * t
    bv = out[:6 * n].reshape(6, n)
    # the initial states are built on the host and on the device (ulp differences)
    for lv in range(6):
        assert np.abs(bv[lv] - ref_bv[lv]).max() <= 1e-10 * np.abs(ref_bv[lv]).max(), lv
    ctx.close()
    ctx_t.close()


def test_served_results_same_alone_and_in_the_mix(h2):
    n_t = 257
    ctx_t, ctx_r = _ctx_tube(h2), _ctx_tube(h2)
    opt = serve.options(h2, hbm_budget=1 << 28, tube_steps=5, reactor_attempts=40)
    out_t1 = np.zeros((6 + h2.ns) * n_t)
    out_r1 = abi.Reactor()
    # short end times: behind the hot side the reaction time scale limits the tube steps to ~1e-10 s
    res1, _ = serve.serve(ctx_r, ctx_t, [_tube_req(n_t, 2e-7, out=out_t1)], opt)
    res2, _ = serve.serve(ctx_r, ctx_t, [_reactor_req(h2, 1200.0, 3e5, 1.0, 5e-6, out=out_r1)], opt)
    out_t2 = np.zeros_like(out_t1)
    out_r2 = abi.Reactor()
    mix = [_tube_req(400, 3e-7, 0.0), _tube_req(n_t, 2e-7, 0.001, out=out_t2), _tube_req(1000, 1e-7, 0.0),
           _reactor_req(h2, 1400.0, 8e5, 0.7, 5e-6, 0.0), _reactor_req(h2, 1200.0, 3e5, 1.0, 5e-6, 0.002, out=out_r2),
           _tube_req(50, 5e-7, 0.0)]
    resm, stats = serve.serve(ctx_r, ctx_t, mix, opt)
    assert all(r.status == 1 for r in resm)
    assert res1[0].status == 1 and res2[0].status == 1
    assert np.array_equal(out_t1, out_t2)
    assert bytes(out_r1) == bytes(out_r2)
    assert resm[1].steps == res1[0].steps and resm[4].steps == res2[0].steps
    assert stats.iterations > 1
    ctx_t.close()
    ctx_r.close()


def test_served_reactors_reach_reference_end_state(h2):
    with open(os.path.join(HERE, "golden", "h2_reactor_runs.json")) as f:
        runs = json.load(f)
    ctx = _ctx_tube(h2)
    opt = serve.options(h2, hbm_budget=1 << 26, reactor_attempts=5000, rtol=runs["rtol"], atol=runs["atol"],
                        h0=runs["h0"])
    reqs = []
    for r in runs["runs"][1:]:
        q = abi.Request()
        q.kind, q.T0, q.p0, q.t_end = abi.REQ_REACTOR, r["T0"], r["p0"], r["t_end"]
        for s in range(h2.ns):
            q.Y[s] = r["Y"][s]
        reqs.append(q)
    res, _ = serve.serve(ctx, None, reqs, opt)
    for r, o in zip(runs["runs"][1:], res):
        assert o.status == abi.REACTOR_DONE
        assert abs(o.T - r["final"]["T"]) <= 1e-5 * r["final"]["T"]
        assert o.latency > 0 and o.t_done >= o.t_admit >= o.t_arrival
    ctx.close()


def test_tube_larger_than_the_pool_is_refused(h2):
    """A tube whose state can never fit the device pool makes the run fail at once with
    CB2_ERR_NOMEM, also without a time limit (it used to wait for memory forever)."""
    ctx_t = _ctx_tube(h2)
    opt = serve.options(h2, hbm_budget=1 << 20, tube_steps=5)
    opt.time_limit_s = 0.0
    with pytest.raises(cb200.CB2Error) as e:
        serve.serve(None, ctx_t, [_tube_req(50, 1e-7), _tube_req(4000, 1e-7, 0.001)], opt)
    assert e.value.code == abi.ERR_NOMEM
    ctx_t.close()
