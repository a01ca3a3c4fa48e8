"""The non-reflecting outflow (DBoundCond::nonReflectingBoundary -> apply_outflow_nr_conserv,
src/BoundCond.cu:3580-3845, called after the inviscid flux at src/RK.cuh:190-193) against the FP64
oracle, through the C ABI: the residual with the correction and three RK3 steps, on the subsonic
2-D air channel (farfield inflow and far side, isothermal wall, non-reflecting exit: the upstream
acoustic wave is clipped) and its supersonic variant (every wave leaves), and on the 9-species
H2/air box with non-reflecting x faces (the mixture gamma and the species waves).  The same
channel and box are pinned to the reference's own kernels in tests/test_ref_kernels_gpu.py."""
import numpy as np
import pytest

import cb200
from cb200 import abi, cases
from cb200.field import DeviceBlock

import refcases

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _sync():
    import torch
    torch.cuda.synchronize()


def _channel(name, speed):
    p, hb, faces, extra = refcases.build(refcases.case_by_name(name))
    if speed != 1.0:
        for c in (1, 2):
            hb.a["bv"][c] *= speed
        cases.fill_cv_air(hb)
    return p, hb, faces, extra


def _err(a, b):
    """Largest error over the variables relative to each one's largest |value|; the momentum
    components share the largest of their scales (in 2-D the z momentum residual is rounding noise
    around zero)."""
    scale = [max(np.abs(b[c]).max(), 1e-300) for c in range(len(b))]
    scale[1:4] = [max(scale[1:4])] * 3
    return max(np.abs(a[c] - b[c]).max() / scale[c] for c in range(len(b)))


def _plain(faces):
    """The same faces with the non-reflecting flag taken off."""
    out = []
    for f in faces:
        g = abi.FaceBC.from_buffer_copy(f)
        g.type = f.type & ~abi.BC_NONREFLECTING
        if hasattr(f, "_sv_keep"):
            g._sv_keep = f._sv_keep
        out.append(g)
    return out


@pytest.mark.parametrize("name,speed", [("chan_nr_weno5ch", 1.0), ("chan_nr_ausm_muscl", 1.0),
                                        ("chan_nr_weno5ch", 4.0), ("mix_nr_weno5ch", 1.0)],
                         ids=["weno5ch", "ausm_muscl", "supersonic", "mixture"])
def test_nonreflecting_rhs(oracle_lib, name, speed):
    p, hb, faces, extra = _channel(name, speed)
    oracle_lib.properties(p, hb)
    oracle_lib.boundary(p, hb, faces)
    dev = DeviceBlock(hb)
    ctx = cb200.Context(p)
    ctx.bind(0, dev.view(), faces)
    ctx.rhs(0)
    _sync()
    dq = dev.to_host(["dq"])["dq"]
    oracle_lib.rhs(p, hb, faces)
    assert _err(dq, hb.a["dq"]) < TOL
    # the correction is there: the plain outflow's residual differs at the exit nodes only
    dq_nr = hb.a["dq"].copy()
    oracle_lib.rhs(p, hb, _plain(faces))
    diff = np.abs(hb.a["dq"] - dq_nr).max(axis=0)
    assert diff[:, :, -1].max() > 0 and diff[:, :, 1:-1].max() == 0
    ctx.close()


@pytest.mark.parametrize("name", ["chan_nr_weno5ch", "mix_nr_weno5ch"], ids=["channel", "mixture"])
def test_nonreflecting_rk3(oracle_lib, name):
    p, hb, faces, extra = _channel(name, 1.0)
    oracle_lib.properties(p, hb)
    oracle_lib.boundary(p, hb, faces)
    dev = DeviceBlock(hb)
    ctx = cb200.Context(p)
    ctx.bind(0, dev.view(), faces)
    dt = p.dt if p.n_spec else 0.2 * oracle_lib.cfl_dt(p, hb)
    for _ in range(3):
        ctx.rk3_step(dt, fixed_dt=True)
        oracle_lib.rk3_step(p, [hb], [faces], dt, fixed_dt=True)
    _sync()
    assert ctx.read_status() == 0
    out = dev.to_host(["cv"])
    g = hb.ngg
    if hb.mz == 1:
        sl = (slice(None), slice(None), slice(g, -g), slice(g, -g))
    else:
        sl = (slice(None), slice(g, -g), slice(g, -g), slice(g, -g))
    assert _err(out["cv"][sl], hb.a["cv"][sl]) < 3 * TOL
    ctx.close()


def test_nonreflecting_flag_only_on_outflow():
    p, hb, faces, extra = _channel("chan_nr_weno5ch", 1.0)
    bad = _plain(faces)
    bad[0].type |= abi.BC_NONREFLECTING  # a farfield face cannot be non-reflecting
    dev = DeviceBlock(hb)
    ctx = cb200.Context(p)
    with pytest.raises(cb200.lib.CB2Error):
        ctx.bind(0, dev.view(), bad)
    ctx.close()
