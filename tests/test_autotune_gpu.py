"""Tile-width autotuning of the y/z primitive sweeps (cb2_autotune / cb2_set_tile_widths):
every width must give the same residual bit for bit, the tuner must leave the caller's arrays
untouched, and the chosen widths must be candidates."""
import numpy as np
import pytest

import cb200
from cb200 import abi
from cb200.field import DeviceBlock

import helpers

pytestmark = pytest.mark.gpu


def _sync():
    import torch
    torch.cuda.synchronize()


def _setup(oracle, scheme, rec, visc, precision=abi.PREC_FP64, dims=(20, 18, 16)):
    p, hb, faces = helpers.curvilinear_air_case(*dims, scheme=scheme, reconstruction=rec, viscous_order=visc,
                                                bc="periodic", seed=5)
    p.precision = precision
    oracle.boundary(p, hb, faces)
    dev = DeviceBlock(hb)
    ctx = cb200.Context(p)
    ctx.bind(0, dev.view(), faces)
    return p, hb, faces, dev, ctx


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("scheme,rec", [(abi.INV_AUSMP, abi.REC_WENO7), (abi.INV_HLLC, abi.REC_WENO5),
                                        (abi.INV_ROE, abi.REC_WENO7)], ids=["ausm_weno7", "hllc_weno5", "roe_weno7"])
def test_every_tile_width_gives_the_same_residual(oracle_lib, scheme, rec, precision):
    p, hb, faces, dev, ctx = _setup(oracle_lib, scheme, rec, 0, precision)
    results = []
    for w in (4, 8, 16):
        ctx.set_tile_widths(0, [0, w, w])
        ctx.rhs(0)
        _sync()
        results.append(dev.to_host(["dq"])["dq"])
    assert np.array_equal(results[0], results[1]) and np.array_equal(results[1], results[2])
    if precision == abi.PREC_FP64:
        oracle_lib.rhs(p, hb, faces)
        assert helpers.rel_err(results[0], hb.a["dq"]) < 1e-12


def test_autotune_picks_a_candidate_and_leaves_state_alone(oracle_lib):
    p, hb, faces, dev, ctx = _setup(oracle_lib, abi.INV_AUSMP, abi.REC_WENO7, 8, dims=(40, 36, 32))
    ctx.rhs(0)
    _sync()
    before = dev.to_host()
    widths = ctx.autotune(0)
    _sync()
    after = dev.to_host()
    assert widths[0] == 0 and widths[1] in (4, 8, 16) and widths[2] in (4, 8, 16)
    for n in before:
        assert np.array_equal(before[n], after[n]), n
    # a step after tuning equals a step with the default widths
    dev2 = DeviceBlock(hb)
    ctx2 = cb200.Context(p)
    ctx2.bind(0, dev2.view(), faces)
    dev.load(hb)
    dt = 0.2 * oracle_lib.cfl_dt(p, hb)
    ctx.rk3_step(dt, True)
    ctx2.rk3_step(dt, True)
    _sync()
    assert np.array_equal(dev.to_host(["cv"])["cv"], dev2.to_host(["cv"])["cv"])


def test_set_tile_widths_rejects_other_widths(oracle_lib):
    p, hb, faces, dev, ctx = _setup(oracle_lib, abi.INV_HLLC, abi.REC_WENO5, 0)
    with pytest.raises(cb200.CB2Error) as e:
        ctx.set_tile_widths(0, [0, 12, 8])
    assert e.value.code == abi.ERR_INVALID
