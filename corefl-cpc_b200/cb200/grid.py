"""Multi-block grids as the reference's Mesh prepares them: the registered inner faces, the ghost
coordinates and the metrics / Jacobian of every padded node.

The hot path consumes metric and jac as given (they are DZone inputs), so this host module plays
the part of the reference's grid stage for the cases built here:
  register_inner_face  InnerFace::register_boundary (src/Mesh.cpp:39-172) -> abi.InnerFace
  extend_coordinates   Mesh::init_ghost_grid + init_inner_ghost_grid (src/Mesh.cpp:1013-1217)
  metrics              Block::compute_jac_metric (src/Mesh.cpp:244-528): central differences of
                       the coordinates on every padded node (a grid with a non-positive Jacobian
                       is refused rather than patched from a neighbour)
  square_cylinder      the four body-fitted blocks around a square cylinder of the AIR5 Mach-10
                       configuration, with their faces and inner faces
Arrays are indexed [k, j, i] like HostBlock arrays; "raw" faces use the reference's grid-file
conventions (1-based inner-face ranges as in inner%4d.txt, 0-based boundary ranges).
"""
import math

import numpy as np

from . import abi


def _sgn(v):
    return (v > 0) - (v < 0)


def register_inner_face(raw, raw_target, dim, ngg):
    """abi.InnerFace from one face pair of the reference's inner-face file: raw = (i1, i2, j1, j2,
    k1, k2) of this block, raw_target = (i1, i2, j1, j2, k1, k2, target block id, 1-based)."""
    rs = [raw[0], raw[2], raw[4]]
    re = [raw[1], raw[3], raw[5]]
    ts = [raw_target[0], raw_target[2], raw_target[4]]
    te = [raw_target[1], raw_target[3], raw_target[5]]
    face, direction = 0, 1
    for a in range(dim):
        if rs[a] == re[a]:
            face = a
            if rs[a] == 1:
                direction = -1
            rs[a] -= 1
            re[a] -= 1
            break
    tface, tdir = 0, 1
    for a in range(dim):
        if ts[a] == te[a]:
            tface = a
            if ts[a] == 1:
                tdir = -1
            ts[a] -= 1
            te[a] -= 1
            break
    src = [0, 0, 0]
    src[tface] = -(direction * tdir) * (face + 1)
    if dim == 2:
        nf, tnf = 1 - face, 1 - tface
        rs[nf], re[nf] = abs(rs[nf]) - 1, abs(re[nf]) - 1
        ts[tnf], te[tnf] = abs(ts[tnf]) - 1, abs(te[tnf]) - 1
        src[tnf] = _sgn((te[tnf] - ts[tnf]) * (re[nf] - rs[nf])) * (nf + 1)
        src[2] = 3
        rs[2] = re[2] = ts[2] = te[2] = 0
    else:
        nf = tnf = 0
        for a in range(dim):
            if rs[a] < 0:
                nf = a
                rs[a], re[a] = -rs[a] - 1, -re[a] - 1
                break
        for a in range(dim):
            if ts[a] < 0:
                tnf = a
                ts[a], te[a] = -ts[a] - 1, -te[a] - 1
                break
        src[tnf] = _sgn((te[tnf] - ts[tnf]) * (re[nf] - rs[nf])) * (nf + 1)
        nf, tnf = 3 - face - nf, 3 - tface - tnf
        rs[nf] -= 1
        re[nf] -= 1
        ts[tnf] -= 1
        te[tnf] -= 1
        src[tnf] = _sgn((te[tnf] - ts[tnf]) * (re[nf] - rs[nf])) * (nf + 1)
    # the exchanged range: the face layer and its ngg ghost layers
    rs_face = -ngg if direction < 0 else re[face]
    re_face = 0 if direction < 0 else re[face] + ngg
    rs[face], re[face] = rs_face, re_face
    sgn_tar = _sgn(src[tface])
    if tdir > 0:
        ts[tface] = te[tface] - ngg if sgn_tar > 0 else te[tface]
    else:
        ts[tface] = 0 if sgn_tar > 0 else ngg
    f = abi.InnerFace()
    for a in range(3):
        f.range_start[a], f.range_end[a] = rs[a], re[a]
        f.target_start[a], f.target_end[a] = ts[a], te[a]
        f.loop_dir[a] = 1 if rs[a] <= re[a] else -1
        f.target_loop_dir[a] = _sgn(src[a])
        f.src_tar[a] = abs(src[a]) - 1
        f.n_point[a] = abs(rs[a] - re[a]) + 1
    f.face, f.direction = face, direction
    f.target_face, f.target_direction = tface, tdir
    f.target_block = raw_target[6] - 1
    return f


def extend_coordinates(xyz, inner, ngg):
    """Ghost coordinates of every block, ngg + 1 layers (init_ghost_grid, src/Mesh.cpp:1013-1167):
    mirror extrapolation across each face, planes z0 - 1, z0 + 1, ... for 2-D blocks, ghosts
    across inner faces copied from the neighbour (init_inner_ghost_grid, :1169-1217), then edges
    and corners by the parallelogram rule.  xyz[b] = (x, y, z) arrays [k, j, i] of the block's
    nodes; inner[b] = its abi.InnerFace list.  Returns padded (x, y, z) per block, offset g1."""
    g1 = ngg + 1
    out = []
    dim = 2 if all(c[0].shape[0] == 1 for c in xyz) else 3
    for x, y, z in xyz:
        mz, my, mx = x.shape
        P = []
        for c in (x, y, z):
            a = np.zeros((mz + 2 * g1, my + 2 * g1, mx + 2 * g1))
            a[g1:g1 + mz, g1:g1 + my, g1:g1 + mx] = c
            P.append(a)
        out.append(P)

    def at(a, i, j, k):
        return a[k + g1, j + g1, i + g1]

    for b, (x, y, z) in enumerate(xyz):
        mz, my, mx = x.shape
        for a in out[b]:
            for i in range(1, g1 + 1):  # i direction, j in [0,my), k in [0,mz)
                a[g1:g1 + mz, g1:g1 + my, g1 - i] = 2 * a[g1:g1 + mz, g1:g1 + my, g1] - a[g1:g1 + mz, g1:g1 + my, g1 + i]
                a[g1:g1 + mz, g1:g1 + my, g1 + mx - 1 + i] = (2 * a[g1:g1 + mz, g1:g1 + my, g1 + mx - 1] -
                                                              a[g1:g1 + mz, g1:g1 + my, g1 + mx - 1 - i])
            for j in range(1, g1 + 1):
                a[g1:g1 + mz, g1 - j, g1:g1 + mx] = 2 * a[g1:g1 + mz, g1, g1:g1 + mx] - a[g1:g1 + mz, g1 + j, g1:g1 + mx]
                a[g1:g1 + mz, g1 + my - 1 + j, g1:g1 + mx] = (2 * a[g1:g1 + mz, g1 + my - 1, g1:g1 + mx] -
                                                              a[g1:g1 + mz, g1 + my - 1 - j, g1:g1 + mx])
        X, Y, Z = out[b]
        if dim == 3:
            for a in out[b]:
                for k in range(1, g1 + 1):
                    a[g1 - k, g1:g1 + my, g1:g1 + mx] = 2 * a[g1, g1:g1 + my, g1:g1 + mx] - a[g1 + k, g1:g1 + my, g1:g1 + mx]
                    a[g1 + mz - 1 + k, g1:g1 + my, g1:g1 + mx] = (2 * a[g1 + mz - 1, g1:g1 + my, g1:g1 + mx] -
                                                                  a[g1 + mz - 1 - k, g1:g1 + my, g1:g1 + mx])
        else:
            for k in range(1, g1 + 1):
                for a in (X, Y):
                    a[g1 - k, g1:g1 + my, g1:g1 + mx] = a[g1, g1:g1 + my, g1:g1 + mx]
                    a[g1 + k, g1:g1 + my, g1:g1 + mx] = a[g1, g1:g1 + my, g1:g1 + mx]
                Z[g1 - k, g1:g1 + my, g1:g1 + mx] = Z[g1, g1:g1 + my, g1:g1 + mx] - k
                Z[g1 + k, g1:g1 + my, g1:g1 + mx] = Z[g1, g1:g1 + my, g1:g1 + mx] + k
    # ghosts across inner faces from the neighbour's nodes
    for b in range(len(xyz)):
        for f in inner[b]:
            t = f.target_block
            mn = list(f.range_start)
            mxr = list(f.range_end)
            mt = list(f.target_start)
            shift = -1 if f.direction < 0 else 1
            mn[f.face] += shift
            mxr[f.face] += shift
            mt[f.target_face] += -1 if f.target_direction > 0 else 1
            ld, tl, st = list(f.loop_dir), list(f.target_loop_dir), list(f.src_tar)
            i1 = mn[0]
            while ld[0] * (i1 - mxr[0]) != 1:
                j1 = mn[1]
                while ld[1] * (j1 - mxr[1]) != 1:
                    k1 = mn[2]
                    while ld[2] * (k1 - mxr[2]) != 1:
                        di = (i1 - mn[0], j1 - mn[1], k1 - mn[2])
                        i2 = mt[0] + tl[0] * di[st[0]]
                        j2 = mt[1] + tl[1] * di[st[1]]
                        k2 = mt[2] + tl[2] * di[st[2]]
                        for c in range(3):
                            out[b][c][k1 + g1, j1 + g1, i1 + g1] = out[t][c][k2 + g1, j2 + g1, i2 + g1]
                        k1 += ld[2]
                    j1 += ld[1]
                i1 += ld[0]
    # edges and corners (parallelogram)
    for b, (x, y, z) in enumerate(xyz):
        mz, my, mx = x.shape
        for a in out[b]:
            A = lambda i, j, k: a[k + g1, j + g1, i + g1]  # noqa: E731

            def setv(i, j, k, v):
                a[k + g1, j + g1, i + g1] = v
            for i in range(1, g1 + 1):
                for j in range(1, g1 + 1):
                    for k in range(0, mz):
                        i1, j1, i2, j2 = -i, -j, mx - 1 + i, my - 1 + j
                        setv(i1, j1, k, A(i1, 0, k) + A(0, j1, k) - A(0, 0, k))
                        setv(i2, j2, k, A(i2, my - 1, k) + A(mx - 1, j2, k) - A(mx - 1, my - 1, k))
                        setv(i1, j2, k, A(i1, my - 1, k) + A(0, j2, k) - A(0, my - 1, k))
                        setv(i2, j1, k, A(i2, 0, k) + A(mx - 1, j1, k) - A(mx - 1, 0, k))
            for i in range(1, g1 + 1):
                for j in range(0, my):
                    for k in range(1, g1 + 1):
                        i1, k1, i2, k2 = -i, -k, mx - 1 + i, mz - 1 + k
                        setv(i1, j, k1, A(i1, j, 0) + A(0, j, k1) - A(0, j, 0))
                        setv(i2, j, k2, A(i2, j, mz - 1) + A(mx - 1, j, k2) - A(mx - 1, j, mz - 1))
                        setv(i1, j, k2, A(i1, j, mz - 1) + A(0, j, k2) - A(0, j, mz - 1))
                        setv(i2, j, k1, A(i2, j, 0) + A(mx - 1, j, k1) - A(mx - 1, j, 0))
            for i in range(-g1, mx + g1):
                for j in range(1, g1 + 1):
                    for k in range(1, g1 + 1):
                        j1, k1, j2, k2 = -j, -k, my - 1 + j, mz - 1 + k
                        setv(i, j1, k1, A(i, j1, 0) + A(i, 0, k1) - A(i, 0, 0))
                        setv(i, j2, k2, A(i, j2, mz - 1) + A(i, my - 1, k2) - A(i, my - 1, mz - 1))
                        setv(i, j1, k2, A(i, j1, mz - 1) + A(i, 0, k2) - A(i, 0, mz - 1))
                        setv(i, j2, k1, A(i, j2, 0) + A(i, my - 1, k1) - A(i, my - 1, 0))
    return out, g1


def metrics(padded, g1, ngg):
    """(metric[9], jac) on the nodes of ghost width ngg from coordinates padded by g1 >= ngg + 1
    (compute_jac_metric, src/Mesh.cpp:244-528): dx/dxi etc. are half the central differences."""
    X, Y, Z = padded
    nz, ny, nx = X.shape
    s = (slice(g1 - ngg, nz - g1 + ngg), slice(g1 - ngg, ny - g1 + ngg), slice(g1 - ngg, nx - g1 + ngg))

    def d(a, axis):
        sl_p = [s[0], s[1], s[2]]
        sl_m = [s[0], s[1], s[2]]
        sl_p[axis] = slice(s[axis].start + 1, s[axis].stop + 1)
        sl_m[axis] = slice(s[axis].start - 1, s[axis].stop - 1)
        return (a[tuple(sl_p)] - a[tuple(sl_m)]) * 0.5

    dxd1, dyd1, dzd1 = d(X, 2), d(Y, 2), d(Z, 2)
    dxd2, dyd2, dzd2 = d(X, 1), d(Y, 1), d(Z, 1)
    dxd3, dyd3, dzd3 = d(X, 0), d(Y, 0), d(Z, 0)
    jac = (dxd1 * dyd2 * dzd3 + dxd2 * dyd3 * dzd1 + dxd3 * dyd1 * dzd2 - dxd1 * dyd3 * dzd2 -
           dxd2 * dyd1 * dzd3 - dxd3 * dyd2 * dzd1)
    if not np.all(jac > 0):
        raise ValueError("non-positive Jacobian in the grid")
    m = np.empty((9,) + jac.shape)
    m[0] = (dyd2 * dzd3 - dyd3 * dzd2) / jac
    m[1] = (dxd3 * dzd2 - dxd2 * dzd3) / jac
    m[2] = (dxd2 * dyd3 - dxd3 * dyd2) / jac
    m[3] = (dyd3 * dzd1 - dyd1 * dzd3) / jac
    m[4] = (dxd1 * dzd3 - dxd3 * dzd1) / jac
    m[5] = (dxd3 * dyd1 - dxd1 * dyd3) / jac
    m[6] = (dyd1 * dzd2 - dyd2 * dzd1) / jac
    m[7] = (dxd2 * dzd1 - dxd1 * dzd2) / jac
    m[8] = (dxd1 * dyd2 - dxd2 * dyd1) / jac
    return m, jac


def wall_stretching(n, first, length):
    """Node distances from the wall along a line of `length` with n nodes, one-sided tanh
    clustering whose first spacing is `first`: s(eta) = L (1 + tanh(beta (eta - 1)) / tanh(beta))."""
    eta = np.linspace(0.0, 1.0, n)
    target = first / length

    def first_of(beta):
        return 1.0 + math.tanh(beta * (eta[1] - 1.0)) / math.tanh(beta)

    lo, hi = 1e-6, 50.0
    if first_of(lo) <= target:  # uniform spacing is already fine enough
        return length * eta
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if first_of(mid) > target:
            lo = mid
        else:
            hi = mid
    beta = 0.5 * (lo + hi)
    return length * (1.0 + np.tanh(beta * (eta - 1.0)) / math.tanh(beta))


def square_cylinder(n_side, n_normal, side=0.01, half_box=0.04, first=1e-6):
    """Four body-fitted blocks around a square cylinder of side `side` centred at the origin, in
    a square box of half-width `half_box`: block b follows one side of the body clockwise
    (0 bottom, 1 left = upstream, 2 top, 3 right = downstream), i along the side, j from the wall
    (j = 0) to the box along straight lines, clustered to a first spacing `first` at the middle of
    the side.  Returns dict(xyz = [(x, y, z)] per block ([k, j, i], k = 1), faces = raw boundary
    lines per block (0-based "i1 i2 j1 j2 k1 k2 label": wall 2 on j = 0, inflow 5 on the box except
    the downstream side, outflow 6 there), inner = raw inner-face pairs per block (1-based, as
    inner%4d.txt), and the pieces used."""
    h, H = 0.5 * side, half_box
    body = [(h, -h), (-h, -h), (-h, h), (h, h)]   # clockwise corners
    box = [(H, -H), (-H, -H), (-H, H), (H, H)]
    s = wall_stretching(n_normal, first, H - h) / (H - h)  # fraction of each normal line
    xyz, faces, inner = [], [], []
    for b in range(4):
        c0, c1 = np.array(body[b]), np.array(body[(b + 1) % 4])
        o0, o1 = np.array(box[b]), np.array(box[(b + 1) % 4])
        t = np.linspace(0.0, 1.0, n_side)
        w = c0[None, :] * (1 - t)[:, None] + c1[None, :] * t[:, None]     # wall points [i, 2]
        o = o0[None, :] * (1 - t)[:, None] + o1[None, :] * t[:, None]     # box points
        pts = w[None, :, :] + s[:, None, None] * (o - w)[None, :, :]      # [j, i, 2]
        x = pts[..., 0][None].copy()
        y = pts[..., 1][None].copy()
        xyz.append((x, y, np.zeros_like(x)))
        outer = 6 if b == 3 else 5
        faces.append([(0, n_side - 1, 0, 0, 0, 0, 2), (0, n_side - 1, n_normal - 1, n_normal - 1, 0, 0, outer)])
        nxt, prv = (b + 1) % 4, (b + 3) % 4
        inner.append([((n_side, n_side, 1, n_normal, 1, 1, b + 1), (1, 1, 1, n_normal, 1, 1, nxt + 1)),
                      ((1, 1, 1, n_normal, 1, 1, b + 1), (n_side, n_side, 1, n_normal, 1, 1, prv + 1))])
    return dict(xyz=xyz, faces=faces, inner=inner, side=side, half_box=half_box, first=first)
