"""Served solves: 0-D constant-volume reactors and 1-D reactive shock tubes under continuous
batching (cb2_serve_run of include/cb200_serve.h).

`request_stream` draws the seeded request mix of the served workload: Poisson arrivals; reactors
with T0 ~ U[1000, 1500] K, p0 ~ U[1, 10] atm, phi ~ U[0.5, 2] to 1 ms; shock tubes with
N ~ U{200..4000} nodes, (1500 K, 5 atm) | (300 K, 1 atm) stoichiometric H2/air to 50 us.
`serve` runs a list of requests and returns per-request results.
"""
import ctypes as C

import numpy as np

from . import abi
from .lib import check, load
from .mech import stoich_h2_air


def h2_air_y(mech, phi):
    """Mass fractions of H2/air at equivalence ratio phi (X_H2 : X_O2 : X_N2 = 2 phi : 1 : 3.76)."""
    x = {"H2": 2.0 * phi, "O2": 1.0, "N2": 3.76}
    w = mech.mw
    y = np.zeros(mech.ns)
    tot = sum(v * w[mech.index(k)] for k, v in x.items())
    for k, v in x.items():
        y[mech.index(k)] = v * w[mech.index(k)] / tot
    return y


def request_stream(mech, rate=2000.0, duration=1.0, frac_reactor=0.5, seed=0, t_reactor=1e-3, t_tube=50e-6,
                   n_range=(200, 4000)):
    """Seeded Poisson arrivals over `duration` seconds at `rate` requests per second."""
    rng = np.random.default_rng(seed)
    t = 0.0
    reqs = []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            break
        r = abi.Request()
        r.arrival = t
        if rng.uniform() < frac_reactor:
            r.kind = abi.REQ_REACTOR
            r.T0 = rng.uniform(1000.0, 1500.0)
            r.p0 = 101325.0 * rng.uniform(1.0, 10.0)
            y = h2_air_y(mech, rng.uniform(0.5, 2.0))
            for s in range(mech.ns):
                r.Y[s] = y[s]
            r.t_end = t_reactor
        else:
            r.kind = abi.REQ_TUBE
            r.n_nodes = int(rng.integers(n_range[0], n_range[1] + 1))
            r.t_end = t_tube
        reqs.append(r)
    return reqs


def options(mech, hbm_budget=8 << 30, max_tubes=296, max_reactors=4096, tube_steps=50, reactor_attempts=200,
            rtol=1e-6, atol=1e-12, h0=1e-8, tube_length=0.1, time_limit=600.0):
    o = abi.ServeOptions()
    o.hbm_budget_bytes = hbm_budget
    o.max_tubes, o.max_reactors = max_tubes, max_reactors
    o.tube_steps_per_launch, o.reactor_attempts_per_launch = tube_steps, reactor_attempts
    o.rtol, o.atol, o.h0 = rtol, atol, h0
    o.tube_length = tube_length
    o.tube_TL, o.tube_pL, o.tube_TR, o.tube_pR = 1500.0, 5 * 101325.0, 300.0, 101325.0
    y = np.ascontiguousarray(stoich_h2_air(mech), dtype=np.float64)
    o._y = y  # keep alive
    o.tube_Y = y.ctypes.data_as(C.POINTER(C.c_double))
    o.time_limit_s = time_limit
    o._stats = abi.ServeStats()
    o.stats = C.pointer(o._stats)
    return o


def serve(ctx_reactor, ctx_tube, reqs, opt):
    """Run the requests; returns (list of abi.Result, abi.ServeStats)."""
    fn = load().cb2_serve_run
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(abi.Request), C.c_int, C.POINTER(abi.ServeOptions),
                   C.POINTER(abi.Result)]
    n = len(reqs)
    arr = (abi.Request * n)(*reqs)
    out = (abi.Result * n)()
    check(fn(ctx_reactor.h if ctx_reactor else None, ctx_tube.h if ctx_tube else None, arr, n, C.byref(opt), out),
          "cb2_serve_run")
    return list(out), opt._stats


def latency_summary(results):
    lat = np.array([r.latency for r in results])
    return {"n": int(lat.size), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "max_s": float(lat.max())}
