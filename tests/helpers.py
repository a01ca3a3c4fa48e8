"""Small seeded cases and comparison helpers shared by the tests."""
import math

import numpy as np

from cb200 import abi, cases
from cb200.field import HostBlock, array_specs, box_faces


def rel_err(a, b, axis_comp=True):
    """max |a-b| / max|b| per component (first axis), returned as the max over components."""
    a = np.asarray(a)
    b = np.asarray(b)
    if axis_comp and a.ndim > 1:
        errs = []
        for c in range(a.shape[0]):
            scale = max(np.abs(b[c]).max(), 1e-300)
            errs.append(np.abs(a[c] - b[c]).max() / scale)
        return max(errs)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def curvilinear_air_case(mx=20, my=18, mz=16, ngg=4, scheme=abi.INV_WENO5_CH, reconstruction=abi.REC_MUSCL,
                         viscous_order=0, bc="periodic", seed=0, jump=True, mu=None, sensor=None):
    """A small 3-D air block on the perturbed sine-wave map (non-uniform metrics), with a
    smooth random state, an optional density/pressure jump and periodic or outflow faces.
    sensor = (kind, threshold, eps) switches on the hybrid linear/WENO weights."""
    rng = np.random.default_rng(seed)
    n = max(mx, my, mz) - 1
    specs = array_specs(mx, my, mz, ngg, 5, 0, viscous_order=viscous_order, roe=(scheme == abi.INV_ROE),
                        hybrid=sensor is not None)
    b = HostBlock(mx, my, mz, ngg, specs)
    (x, y, z), metric, det = cases.sine_wave_metrics(n, ngg, 0.05)
    sl = (slice(0, mz + 2 * ngg), slice(0, my + 2 * ngg), slice(0, mx + 2 * ngg))
    x, y, z, det = x[sl], y[sl], z[sl], det[sl]
    b.a["metric"][...] = metric[(slice(None),) + sl]
    b.a["jac"][0] = det
    ph = rng.uniform(0, 2 * math.pi, 8)
    tp = 2 * math.pi
    rho = 1.0 + 0.2 * np.sin(tp * (x + y + z) + ph[0])
    u = 0.6 + 0.3 * np.sin(tp * y + ph[1])
    v = -0.4 + 0.3 * np.cos(tp * z + ph[2])
    w = 0.5 + 0.2 * np.sin(tp * x + ph[3])
    p = 1.0 + 0.1 * np.cos(tp * (x - y) + ph[4])
    if jump:
        mask = (x > 0.45) & (x < 0.7)
        rho = np.where(mask, rho * 0.3, rho)
        p = np.where(mask, p * 0.25, p)
    bv = b.a["bv"]
    bv[0], bv[1], bv[2], bv[3], bv[4] = rho, u, v, w, p
    bv[5] = p / (rho * cases.R_AIR)
    if "mul" in b.a:
        b.a["mul"][0] = mu if mu is not None else 1e-3
    cases.fill_cv_air(b)
    t = abi.BC_PERIODIC if bc == "periodic" else abi.BC_OUTFLOW
    faces = box_faces(mx, my, mz, {(d, s): t for d in range(3) for s in (-1, 1)})
    param = cases.make_param(dim=3, inviscid_scheme=scheme, reconstruction=reconstruction,
                             viscous_order=viscous_order, cfl=0.5, rho_ref=1.0, v_ref=1.0,
                             mu_constant=(mu if mu is not None else 1e-3) if viscous_order else 0.0)
    if sensor is not None:
        param.shock_sensor, param.sensor_threshold, param.sensor_eps = sensor
    return param, b, faces
