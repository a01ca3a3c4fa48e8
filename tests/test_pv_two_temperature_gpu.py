"""Two-temperature primitive-variable fluxes (AUSM+ and HLLC with e_ve, src/InviscidScheme.cu:171-219,
397-590 in the reference's two-temperature build: the reconstructed states' energy
rho (e_k + e_tr(T) + e_ve) and translational-rotational gamma, e_ve carried as a scalar) against
the FP64 oracle through the C ABI: the residual on the AIR5 box for each solver and reconstruction,
and three RK3 steps with Park chemistry and 2nd-order viscous terms.  The same solvers are pinned
to the reference's own kernels in tests/test_ref_kernels_gpu.py (air5_hllc_muscl_visc2_chem,
air5_ausm_muscl_chem)."""
import os

import numpy as np
import pytest

import cb200
from cb200 import abi, cases, mech as mechmod
from cb200.field import DeviceBlock

import helpers

pytestmark = pytest.mark.gpu
TOL = 1e-12
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "air5_park.json")


def _box(scheme, rec, visc=0, reaction=False):
    air5 = mechmod.load_json(GOLDEN)
    tt = mechmod.load_two_temperature_json(GOLDEN)
    c = cases.air5_box_2t(air5, tt, n_nodes=10, ngg=4 if rec == abi.REC_WENO7 else 3, viscous_order=visc,
                          reaction=reaction, scheme=scheme, reconstruction=rec)
    return c, (air5, tt)


@pytest.mark.parametrize("scheme,rec", [(abi.INV_HLLC, abi.REC_MUSCL), (abi.INV_AUSMP, abi.REC_MUSCL),
                                        (abi.INV_HLLC, abi.REC_WENO5), (abi.INV_AUSMP, abi.REC_WENO7)],
                         ids=["hllc_muscl", "ausm_muscl", "hllc_weno5", "ausm_weno7"])
def test_pv_two_temperature_rhs(oracle_lib, scheme, rec):
    c, keep = _box(scheme, rec)
    p, hb, faces = c.param, c.blocks[0], c.faces[0]
    oracle_lib.cv_from_bv(p, hb)
    oracle_lib.properties(p, hb)
    dev = DeviceBlock(hb)
    ctx = cb200.Context(p)
    ctx.bind(0, dev.view(), faces)
    ctx.rhs(0, abi.RHS_INVISCID)
    import torch
    torch.cuda.synchronize()
    dq = dev.to_host(["dq"])["dq"]
    oracle_lib.rhs(p, hb, faces, abi.RHS_INVISCID)
    assert np.isfinite(dq).all()
    assert helpers.rel_err(dq, hb.a["dq"]) < TOL
    ctx.close()


@pytest.mark.parametrize("scheme", [abi.INV_HLLC, abi.INV_AUSMP], ids=["hllc", "ausm"])
def test_pv_two_temperature_rk3(oracle_lib, scheme):
    c, keep = _box(scheme, abi.REC_MUSCL, visc=2, reaction=True)
    p, hb, faces = c.param, c.blocks[0], c.faces[0]
    oracle_lib.cv_from_bv(p, hb)
    oracle_lib.properties(p, hb)
    dev = DeviceBlock(hb)
    ctx = cb200.Context(p)
    ctx.bind(0, dev.view(), faces)
    for _ in range(3):
        ctx.rk3_step(2e-9, fixed_dt=True)
        oracle_lib.rk3_step(p, [hb], [faces], 2e-9, fixed_dt=True)
    import torch
    torch.cuda.synchronize()
    assert ctx.read_status() == 0
    out = dev.to_host(["cv", "temperature_ve"])
    g = hb.ngg
    sl = (slice(None), slice(g, -g), slice(g, -g), slice(g, -g))
    assert helpers.rel_err(out["cv"][sl], hb.a["cv"][sl]) < 3 * TOL
    assert helpers.rel_err(out["temperature_ve"][sl], hb.a["temperature_ve"][sl]) < 3 * TOL
    ctx.close()
