"""Batched closed blocks (cb2_block_batch_advance): uneven 2-D and 3-D periodic air blocks in one
persistent launch must give, block by block, the same bits as cb2_rk3_step on that block, with
fixed and CFL steps, whatever other blocks share the batch and whatever tile width and cluster
size the autotuner picks."""
import numpy as np
import pytest

import cb200
from cb200 import abi
from cb200.field import DeviceBlock

import helpers

pytestmark = pytest.mark.gpu

DIMS = [(20, 18, 16), (30, 12, 10), (16, 14, 1), (12, 12, 12)]


def _sync():
    import torch
    torch.cuda.synchronize()


def _blocks(oracle, scheme, rec, dims=DIMS, seed=21):
    out = []
    for a, d in enumerate(dims):
        p, hb, faces = helpers.curvilinear_air_case(*d, scheme=scheme, reconstruction=rec, viscous_order=0,
                                                    bc="periodic", seed=seed + a)
        if d[2] == 1:
            # a closed 2-D block: periodic i and j faces, the k direction collapsed
            p.dim = 2
            faces = [f for f in faces if f.face < 2]
        oracle.boundary(p, hb, faces)
        out.append((p, hb, faces))
    return out


def _reference(p, hb, faces, steps, dt):
    dev = DeviceBlock(hb)
    ctx = cb200.Context(p)
    ctx.bind(0, dev.view(), faces)
    t = 0.0
    for _ in range(steps):
        t += ctx.rk3_step(dt, fixed_dt=dt > 0)
    _sync()
    return dev.to_host(["cv", "bv"]), t


def _batch(ctx, blocks, steps, dt, t_end=1e30):
    devs = [DeviceBlock(hb) for _, hb, _ in blocks]
    cases = (abi.BlockCase * len(blocks))()
    for c, d in zip(cases, devs):
        c.zone = d.view()
        c.time, c.t_end, c.dt = 0.0, t_end, dt
    ctx.block_batch_advance(cases, steps)
    _sync()
    return devs, cases


@pytest.mark.parametrize("scheme,rec", [(abi.INV_AUSMP, abi.REC_WENO7), (abi.INV_HLLC, abi.REC_WENO5)],
                         ids=["ausm_weno7", "hllc_weno5"])
@pytest.mark.parametrize("cfl", [False, True], ids=["fixed_dt", "cfl_dt"])
def test_batch_matches_block_path(oracle_lib, scheme, rec, cfl):
    blocks = _blocks(oracle_lib, scheme, rec)
    p0 = blocks[0][0]
    dts = [0.0 if cfl else 0.2 * oracle_lib.cfl_dt(p, hb) for p, hb, _ in blocks]
    ctx = cb200.Context(p0)
    devs = [DeviceBlock(hb) for _, hb, _ in blocks]
    cases = (abi.BlockCase * len(blocks))()
    for c, d, dt in zip(cases, devs, dts):
        c.zone = d.view()
        c.time, c.t_end, c.dt = 0.0, 1e30, dt
    ctx.block_batch_advance(cases, 4)
    _sync()
    for (p, hb, faces), d, c, dt in zip(blocks, devs, cases, dts):
        ref, t_ref = _reference(p, hb, faces, 4, dt)
        out = d.to_host(["cv", "bv"])
        assert c.steps == 4 and c.status == 0
        assert c.time == t_ref
        for n in ("cv", "bv"):
            assert np.array_equal(out[n], ref[n]), (hb.mx, hb.my, hb.mz, n)


def _cases_for(blocks, dt):
    devs = [DeviceBlock(hb) for _, hb, _ in blocks]
    cases = (abi.BlockCase * len(blocks))()
    for c, d in zip(cases, devs):
        c.zone = d.view()
        c.time, c.t_end, c.dt = 0.0, 1e30, dt
    return cases, devs


def test_batch_result_independent_of_company_and_tiles(oracle_lib):
    blocks = _blocks(oracle_lib, abi.INV_AUSMP, abi.REC_WENO7)
    dt = 0.2 * min(oracle_lib.cfl_dt(p, hb) for p, hb, _ in blocks)
    ctx = cb200.Context(blocks[0][0])
    alone, _ = _batch(ctx, blocks[1:2], 3, dt)
    ref = alone[0].to_host(["cv"])["cv"]
    for w in (4, 8, 16):
        for cs in (1, 2, 4, 8):
            ctx.block_batch_set_schedule(w, cs)
            together, cases = _batch(ctx, blocks, 3, dt)
            assert np.array_equal(together[1].to_host(["cv"])["cv"], ref), (w, cs)
    tune_cases, keep = _cases_for(blocks, dt)
    ni, cs = ctx.block_batch_autotune(tune_cases)
    assert ni in (4, 8, 16) and cs in (1, 2, 4, 8)
    # tuning touched only the residual scratch dq
    for (_, hb, _), d in zip(blocks, keep):
        assert np.array_equal(d.to_host(["cv"])["cv"], hb.a["cv"])


def test_batch_stops_each_block_at_its_end_time(oracle_lib):
    blocks = _blocks(oracle_lib, abi.INV_HLLC, abi.REC_WENO5)[:3]
    ctx = cb200.Context(blocks[0][0])
    devs = [DeviceBlock(hb) for _, hb, _ in blocks]
    cases = (abi.BlockCase * 3)()
    dt = 0.2 * min(oracle_lib.cfl_dt(p, hb) for p, hb, _ in blocks)
    for c, d, n in zip(cases, devs, (2.5, 4.5, 7.5)):
        c.zone = d.view()
        c.time, c.t_end, c.dt = 0.0, n * dt, dt
    ctx.block_batch_advance(cases, 100)
    assert [c.steps for c in cases] == [3, 5, 8]
    assert all(c.status == abi.BLOCK_DONE for c in cases)


def test_batch_rejects_unsupported_settings(oracle_lib):
    p, hb, faces = helpers.curvilinear_air_case(12, 12, 12, scheme=abi.INV_WENO5_CH, reconstruction=abi.REC_MUSCL,
                                                viscous_order=0, bc="periodic", seed=3)
    ctx = cb200.Context(p)
    d = DeviceBlock(hb)
    cases = (abi.BlockCase * 1)()
    cases[0].zone = d.view()
    cases[0].t_end = 1.0
    with pytest.raises(cb200.CB2Error) as e:
        ctx.block_batch_advance(cases, 1)
    assert e.value.code == abi.ERR_UNSUPPORTED
