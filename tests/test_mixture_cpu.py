"""CPU checks of the oracle's mixture thermodynamics, chemistry and temperature Newton
against the reference's own host code (fixtures written by tests/golden/make_mech.py from
the reference's Species::compute_enthalpy_and_cp, cfd::compute_src and cfd::update_t)."""
import json
import os

import numpy as np
import pytest

from cb200 import abi, cases, mech as mechmod
from cb200.field import HostBlock, array_specs

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def h2():
    return mechmod.load_json(os.path.join(GOLDEN, "h2_li2004.json"))


@pytest.fixture(scope="module")
def states():
    with open(os.path.join(GOLDEN, "h2_chem_states.json")) as f:
        return json.load(f)["states"]


def test_mechanism_fixture_shape(h2):
    assert h2.ns == 9 and h2.nr == 19
    assert h2.species[-1] == "N2"
    # third-body (4) and Troe (6) reactions are present
    assert 4 in h2.d["reac_type"] and 6 in h2.d["reac_type"]


def test_nasa7_matches_reference_host(oracle_lib, h2, states):
    for s in states:
        h, cp = oracle_lib.nasa7_h_cp(h2, s["t"])
        np.testing.assert_allclose(h, s["h"], rtol=1e-15, atol=1e-9)
        np.testing.assert_allclose(cp, s["cp"], rtol=1e-15, atol=0)


def test_chemistry_source_matches_reference_host(oracle_lib, h2, states):
    worst = 0.0
    for s in states:
        om, od = oracle_lib.chemistry_source(h2, s["rho"], s["t"], s["y"])
        ref_om, ref_od = np.array(s["omega"]), np.array(s["omega_d"])
        scale = max(np.abs(ref_od).max(), np.abs(ref_om).max(), 1e-300)
        worst = max(worst, np.abs(om - ref_om).max() / scale, np.abs(od - ref_od).max() / scale)
    assert worst < 1e-12, worst


def _one_node_block(h2, rho, t_guess, e, y):
    ns = h2.ns
    specs = array_specs(1, 1, 1, 1, 5 + ns, ns)
    b = HostBlock(1, 1, 1, 1, specs)
    b.a["jac"][...] = 1.0
    b.a["bv"][5] = t_guess
    q = b.a["qn"]
    q[0] = rho
    q[4] = rho * e
    for k in range(ns):
        q[5 + k] = rho * y[k]
    return b


def test_newton_temperature_matches_reference(oracle_lib, h2, states):
    """Stage update with dq = 0 recovers T from e by the reference's Newton iteration
    (tolerance 1e-5 per step); the reference's host solver iterates to 1e-8."""
    p = cases.make_param(n_var=5 + h2.ns, n_spec=h2.ns, mech=h2.ptr())
    for s in states:
        b = _one_node_block(h2, s["rho"], s["t_guess"], s["e"], s["y"])
        oracle_lib.stage_update(p, b, 1e-9, 0)
        t = b.interior("bv", 5).item()
        assert abs(t - s["t_newton"]) <= 1e-8 * s["t_newton"], (t, s["t_newton"])
