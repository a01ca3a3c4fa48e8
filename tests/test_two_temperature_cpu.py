"""Two-temperature model: the oracle's restatement of the reference's device functions against
the reference's own host twins (tests/golden/h2_two_temperature.json, written through
oracle/_ref/dump_2t by tests/golden/make_mech.py), and the physics of the VT relaxation step."""
import json
import os

import numpy as np
import pytest

from cb200 import abi, cases, mech as mechmod

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")


@pytest.fixture(scope="module")
def gold():
    with open(os.path.join(GOLD, "h2_two_temperature.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def h2():
    return mechmod.load_json(os.path.join(GOLD, "h2_li2004.json"))


@pytest.fixture(scope="module")
def tt():
    return mechmod.load_two_temperature_json(os.path.join(GOLD, "h2_two_temperature.json"))


def _param(h2, tt):
    return cases.make_param(n_var=6 + h2.ns, n_spec=h2.ns, mech=h2.ptr(), two_t=tt.ptr(),
                            inviscid_scheme=abi.INV_HLLC, reconstruction=abi.REC_WENO5)


def _close(a, b, rtol, atol=0.0):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return np.all(np.abs(a - b) <= rtol * np.abs(b) + atol)


def test_species_ve_ladder_matches_reference(oracle_lib, gold, h2, tt):
    p = _param(h2, tt)
    ns = h2.ns
    e_ref = np.asarray(gold["ladder_e_ve"]).reshape(-1, ns)
    c_ref = np.asarray(gold["ladder_cv_ve"]).reshape(-1, ns)
    for a, t in enumerate(gold["ladder_T"]):
        e, c = oracle_lib.species_ve(p, t)
        assert _close(e, e_ref[a], 1e-14, 1e-300), (t, e, e_ref[a])
        assert _close(c, c_ref[a], 1e-13, 1e-300), (t, c, c_ref[a])
    # atoms with electronic levels (H, O) and vibrators (H2, O2, ...) both contribute
    e_hot = e_ref[-2]
    assert (e_hot > 0).sum() >= 7


def test_mixture_states_match_reference(oracle_lib, gold, h2, tt):
    p = _param(h2, tt)
    active = 0
    for s in gold["states"]:
        out = oracle_lib.two_temperature_state(p, s["rho"], s["T"], s["Tve"], s["Y"])
        assert _close(out[0:4], [s["eve_T"], s["cv_ve_T"], s["eve_Tve"], s["cv_ve_Tve"]], 1e-14, 1e-300)
        # both sides run the same Newton iteration from T to a 1e-8 relative residual
        assert abs(out[4] - s["tve_inverted"]) <= 1e-12 * s["tve_inverted"]
        # VT source: the host twin takes molar masses as mw where the device takes 1/(1/mw)
        assert abs(out[5] - s["vt_source"]) <= 1e-12 * abs(s["vt_source"]) + 1e-300
        assert abs(out[6] - s["eve_eq"]) <= 1e-14 * abs(s["eve_eq"]) + 1e-300
        assert abs(out[7] - s["tau_eff"]) <= 1e-12 * abs(s["tau_eff"]), (out[7], s["tau_eff"])
        active += s["tau_eff"] < 1e29
    assert active >= len(gold["states"]) // 2


def test_vt_relaxation_conserves_energy_and_relaxes(oracle_lib, h2, tt):
    """One VT step moves e_v towards equilibrium at T, leaves rho E untouched, and drives T_ve
    towards T: the gap shrinks at every node.  A long step reaches e_v(T) of the temperature it
    started from, and the energy it moves shifts T, so the gap closes over repeated steps."""
    case = cases.h2_air_box_2t(h2, tt, n_nodes=6)
    p, b = case.param, case.blocks[0]
    oracle_lib.cv_from_bv(p, b)
    g = b.ngg
    sl = (slice(g, -g),) * 3
    E0 = b.a["cv"][4][sl].copy()
    gap0 = np.abs(b.a["temperature_ve"][0][sl] - b.a["bv"][5][sl])
    b1 = b.copy()
    oracle_lib.vt_relaxation(p, b1, 1e-7)
    gap1 = np.abs(b1.a["temperature_ve"][0][sl] - b1.a["bv"][5][sl])
    assert np.array_equal(b1.a["cv"][4][sl], E0)
    assert np.all(gap1 < gap0)
    b2 = b.copy()
    oracle_lib.vt_relaxation(p, b2, 1.0)
    gap2 = np.abs(b2.a["temperature_ve"][0][sl] - b2.a["bv"][5][sl])
    assert gap2.max() < 0.3 * gap0.min()
    for _ in range(12):
        oracle_lib.vt_relaxation(p, b2, 1.0)
    gap3 = np.abs(b2.a["temperature_ve"][0][sl] - b2.a["bv"][5][sl])
    assert gap3.max() < 1e-3 * gap0.min()
    assert np.array_equal(b2.a["cv"][4][sl], E0)


def two_temperature_residual(b, dt, rng, scale=1e-3):
    """dq that moves every conservative variable by about `scale` of itself in one stage."""
    g = b.ngg
    inner = b.a["cv"][:, g:-g, g:-g, g:-g]
    jac = b.a["jac"][0, g:-g, g:-g, g:-g]
    return scale * rng.standard_normal(inner.shape) * np.abs(inner) * jac / dt


def test_two_temperature_stage_update_runs(oracle_lib, h2, tt):
    """Three stages with the VT step: finite state and a positive e_ve everywhere."""
    case = cases.h2_air_box_2t(h2, tt, n_nodes=6)
    p, b = case.param, case.blocks[0]
    oracle_lib.cv_from_bv(p, b)
    b.a["qn"][...] = b.a["cv"]
    b.a["dq"][...] = two_temperature_residual(b, 1e-8, np.random.default_rng(3))
    for rk in range(3):
        oracle_lib.stage_update(p, b, 1e-8, rk)
    g = b.ngg
    sl = (slice(g, -g),) * 3
    assert np.isfinite(b.a["bv"][:, g:-g, g:-g, g:-g]).all()
    assert np.isfinite(b.a["temperature_ve"][0][sl]).all()
    assert (b.a["sv"][h2.ns][sl] > 0).all()
