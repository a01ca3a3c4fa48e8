"""Mechanism tables for cb2_mechanism.

A mechanism is a dict with the fields of cb2_mechanism (the JSON the reference's own parser
writes; see tests/golden/make_mech.py).  `to_struct` keeps the numpy arrays alive on the
returned object so the pointers stay valid while the struct is in use.
"""
import ctypes as C
import json

import numpy as np

from . import abi


class MechStruct:
    def __init__(self, d):
        self.d = d
        self.ns = int(d["n_spec"])
        self.nr = int(d.get("n_reac", 0))
        self.arrays = {}
        s = abi.Mechanism()
        s.n_spec = self.ns
        s.n_reac = self.nr
        for name in abi.MECH_DOUBLE + abi.MECH_REAC:
            if name in d:
                a = np.ascontiguousarray(np.asarray(d[name], dtype=np.float64))
                self.arrays[name] = a
                setattr(s, name, a.ctypes.data_as(C.POINTER(C.c_double)))
        for name in abi.MECH_INT + ("n_temperature_range",):
            if name in d:
                a = np.ascontiguousarray(np.asarray(d[name], dtype=np.int32))
                self.arrays[name] = a
                setattr(s, name, a.ctypes.data_as(C.POINTER(C.c_int)))
        for name in abi.MECH_NASA9 + abi.MECH_RT:
            if name in d:
                a = np.ascontiguousarray(np.asarray(d[name], dtype=np.float64))
                self.arrays[name] = a
                setattr(s, name, a.ctypes.data_as(C.POINTER(C.c_double)))
        # NASA9 multi-range thermo and the two-temperature control temperatures, when present
        s.therm_nasa_7_9 = int(d.get("nasa_7_or_9", 7))
        s.max_range = int(d.get("max_range", 0))
        s.two_temperature_reaction_temperature = int(d.get("two_temperature_reaction_temperature", 0))
        self.struct = s

    @property
    def species(self):
        return list(self.d.get("species", []))

    @property
    def mw(self):
        return np.asarray(self.d["mw"], dtype=np.float64)

    def index(self, name):
        return self.species.index(name)

    def ptr(self):
        return C.pointer(self.struct)


def load_json(path):
    with open(path) as f:
        return MechStruct(json.load(f))


def stoich_h2_air(mech):
    """Mass fractions of stoichiometric H2/air (X_H2 : X_O2 : X_N2 = 2 : 1 : 3.76)."""
    y = np.zeros(mech.ns)
    x = {"H2": 2.0, "O2": 1.0, "N2": 3.76}
    w = mech.mw
    tot = sum(x[n] * w[mech.index(n)] for n in x)
    for n, v in x.items():
        y[mech.index(n)] = v * w[mech.index(n)] / tot
    return y


class TwoTemperatureStruct:
    """cb2_two_temperature from the JSON the reference's two-temperature parser writes
    (tests/golden/h2_two_temperature.json); keeps the arrays alive like MechStruct."""

    def __init__(self, d, enable_vt_relaxation=True):
        self.d = d
        ns = int(d["n_spec"])
        s = abi.TwoTemperature()
        s.n_spec = ns
        s.max_level = int(d["max_level"])
        s.enable_vt_relaxation = 1 if enable_vt_relaxation else 0
        self.arrays = {}
        for name in ("theta_v", "elec_theta", "elec_g", "lt_a", "lt_b", "park_sigma"):
            a = np.ascontiguousarray(np.asarray(d[name], dtype=np.float64))
            self.arrays[name] = a
            setattr(s, name, a.ctypes.data_as(C.POINTER(C.c_double)))
        a = np.ascontiguousarray(np.asarray(d["n_level"], dtype=np.int32))
        self.arrays["n_level"] = a
        s.n_level = a.ctypes.data_as(C.POINTER(C.c_int))
        self.struct = s

    def ptr(self):
        return C.pointer(self.struct)


def load_two_temperature_json(path, enable_vt_relaxation=True):
    with open(path) as f:
        return TwoTemperatureStruct(json.load(f), enable_vt_relaxation)


R_U = 8314.462618


def species_ve_energy(tt, mw, t):
    """e_ve [J/kg] of every species at temperature t: the harmonic-oscillator vibration
    R theta_v / (exp(theta_v / T) - 1) plus the Boltzmann average of the electronic levels
    (compute_ve_energy, src/Thermo.cu:635-668), with T held at >= 1 K.  Host-side, for building
    inflow states; the kernels evaluate the same model on the device."""
    d = tt.d
    ns = int(d["n_spec"])
    ml = int(d["max_level"])
    temp = max(float(t), 1.0)
    theta = np.asarray(d["theta_v"], dtype=np.float64)
    nlev = np.asarray(d["n_level"], dtype=np.int64)
    eth = np.asarray(d["elec_theta"], dtype=np.float64).reshape(ns, ml)
    eg = np.asarray(d["elec_g"], dtype=np.float64).reshape(ns, ml)
    e = np.zeros(ns)
    for i in range(ns):
        r = R_U / float(mw[i])
        if theta[i] > 0:
            x = theta[i] / temp
            if x < 200:
                e[i] += r * theta[i] / np.expm1(x)
        if nlev[i] > 0:
            bz = eg[i, :nlev[i]] * np.exp(-eth[i, :nlev[i]] / temp)
            zs = bz.sum()
            if zs > 0:
                e[i] += r * (bz * eth[i, :nlev[i]]).sum() / zs
    return e


def mixture_ve_energy(tt, mw, t, y):
    """Mixture e_ve = sum Y_k e_ve,k (compute_mixture_ve_energy, src/Thermo.cu:711-723)."""
    e = species_ve_energy(tt, mw, t)
    total = 0.0
    for i in range(len(e)):
        total += float(y[i]) * e[i]
    return total
