"""Per-block field arrays in the reference's padded layout.

An array with `g` ghost layers and `nc` components is stored as a C-ordered array of shape
(nc, mz+2g, my+2g, mx+2g); element (i,j,k,l) sits at
l*sz + (k+g)*disp1 + (j+g)*disp2 + (i+g), which is exactly
val[k*disp1 + j*disp2 + i + dispt + l*sz] of ggxl::VectorField3D (src/gxl_lib/Array.cuh:315-324).
"""
import ctypes as C

import numpy as np

from . import abi


def array_specs(mx, my, mz, ngg, n_var, n_spec, viscous_order=0, roe=False, hybrid=False, reaction=False):
    """(ncomp, ghost) of every DZone array the path reads or writes (src/Field.cu:440-672)."""
    s = {
        "cv": (n_var, ngg), "bv": (6, ngg), "qn": (n_var, ngg), "dq": (n_var, 0),
        "metric": (9, ngg), "jac": (1, ngg), "mul": (1, ngg), "dt_local": (1, 0), "mach": (1, ngg),
    }
    if n_spec > 0:
        s.update({"sv": (n_spec, ngg), "rho_D": (n_spec, ngg), "thermal_conductivity": (1, ngg),
                  "acoustic_speed": (1, ngg), "gamma": (1, ngg)})
    if viscous_order == 8:
        s.update({"fFlux": (n_var, ngg), "gFlux": (n_var, ngg), "hFlux": (n_var, ngg)})
    if viscous_order == 2:
        s["vis_flux"] = (n_var - 1, 1)
    if roe:
        s["entropy_fix_delta"] = (1, 1)
    if hybrid:
        s["shock_sensor"] = (1, ngg)
    if reaction:
        s["reaction_timeScale"] = (1, ngg)
    return s


def shape_of(mx, my, mz, nc, g):
    return (nc, mz + 2 * g, my + 2 * g, mx + 2 * g)


class HostBlock:
    """numpy-backed block; `a[name][l, k+g, j+g, i+g]` is element (i,j,k,l)."""

    def __init__(self, mx, my, mz, ngg, specs):
        self.mx, self.my, self.mz, self.ngg = mx, my, mz, ngg
        self.specs = dict(specs)
        self.a = {n: np.zeros(shape_of(mx, my, mz, nc, g), dtype=np.float64) for n, (nc, g) in specs.items()}

    def interior(self, name, comp=None):
        nc, g = self.specs[name]
        arr = self.a[name]
        sl = (slice(g, g + self.mz), slice(g, g + self.my), slice(g, g + self.mx))
        return arr[(slice(None),) + sl] if comp is None else arr[(comp,) + sl]

    def view(self):
        v = abi.ZoneView(self.mx, self.my, self.mz, self.ngg)
        for n in abi.ZONE_ARRAYS:
            if n in self.a:
                setattr(v, n, self.a[n].ctypes.data)
        return v

    def copy(self):
        b = HostBlock(self.mx, self.my, self.mz, self.ngg, self.specs)
        for n in self.a:
            b.a[n][...] = self.a[n]
        return b


class DeviceBlock:
    """torch.cuda-backed mirror of a HostBlock (torch is only the device allocator here)."""

    def __init__(self, host: HostBlock, device="cuda"):
        import torch
        self.mx, self.my, self.mz, self.ngg = host.mx, host.my, host.mz, host.ngg
        self.specs = dict(host.specs)
        self.t = {n: torch.from_numpy(a).to(device) for n, a in host.a.items()}

    def view(self):
        v = abi.ZoneView(self.mx, self.my, self.mz, self.ngg)
        for n in abi.ZONE_ARRAYS:
            if n in self.t:
                setattr(v, n, self.t[n].data_ptr())
        return v

    def to_host(self, names=None):
        out = {}
        for n in (names or self.t.keys()):
            out[n] = self.t[n].cpu().numpy()
        return out

    def load(self, host: HostBlock, names=None):
        import torch
        for n in (names or host.a.keys()):
            self.t[n].copy_(torch.from_numpy(host.a[n]))


def faces_array(faces):
    arr = (abi.FaceBC * max(1, len(faces)))()
    for a, f in enumerate(faces):
        arr[a] = f
    return arr


def face(type_, face_dim, direction, start, end, sv=None, **state):
    """A cb2_face_bc; sv (sequence of the n_scalar inflow scalars) is kept with the struct."""
    f = abi.FaceBC()
    f.type, f.face, f.direction = type_, face_dim, direction
    for a in range(3):
        f.range_start[a], f.range_end[a] = start[a], end[a]
    for k, v in state.items():
        setattr(f, k, v)
    if sv is not None:
        keep = np.ascontiguousarray(sv, dtype=np.float64)
        f.sv = keep.ctypes.data
        f._sv_keep = keep
    return f


def box_faces(mx, my, mz, types):
    """Faces of a whole block: types = {(dim, dir): bc_type} for the faces that exist."""
    out = []
    ext = (mx, my, mz)
    for (d, s), t in types.items():
        start = [0, 0, 0]
        end = [mx - 1, my - 1, mz - 1]
        start[d] = end[d] = 0 if s < 0 else ext[d] - 1
        out.append(face(t, d, s, start, end))
    return out
