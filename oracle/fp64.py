"""FP64 restatement of the particle-to-grid path (test infrastructure only).

The definitions are those of orc_interp.c (src/particles.f90: TSC 16-271, PPART_DENS
742-801, VVEL_INTERP_SPH_VW 806-929 with KERNEL_FUNC 935-963, FILL_H_ZEROS
398-430, DDENS_INTERP_SPH 434-617), but every quantity is double precision and
the neighbour searches rank double-precision distances (scipy's cKDTree).  It
states the error of the REAL*4 path -- the oracle, which the GPU's SPH fields
equal bit for bit and its TSC fields within 1e-5 -- against the same method in
FP64, field by field.

Only the arithmetic differs from the REAL*4 path: grid coordinates are the
REAL*4 RADX values, the ball fallback is taken where the K-th distance is at
most DX, DDENS does not wrap (cells outside 1..NX are skipped), and a particle
whose kernel sum is zero puts its mass in its own cell.
"""
from __future__ import annotations

import numpy as np
from scipy.spatial import cKDTree


def _m4(d, h, gauss=False):
    """KERNEL_FUNC: W(d; h) with q = d / (h / 2): the M4 branch, or with
    KERNEL_MODE = 2 the Gaussian exp(-q^2) (src/particles.f90:935-963)."""
    q = d / (h / 2.0)
    if gauss:
        return np.exp(-q * q)
    return np.where(q <= 1.0, 1.0 - 1.5 * q * q * (1.0 - 0.5 * q),
                    np.where(q <= 2.0, 0.25 * (2.0 - q) ** 3, 0.0))


def particles_to_grid_fp64(p, x, y, z, vx, vy, vz, m):
    """(u_mass, u2, u3, u4, hpart, part_dens) of the SPH/SPH path in FP64 (inner
    grid, column-major, x fastest), for flag_vel_interp = flag_dens_interp = 1."""
    from .oracle import grid_setup
    g, radx = grid_setup(p)
    nx, K, box, per = int(p.nx), int(p.kneighbours), float(p.lado0), bool(p.periodic)
    gauss = int(getattr(p, "kernel_mode", 1)) == 2
    dx = float(g.dx)
    rad = np.asarray(radx, np.float64)
    off = int(g.rad_lo)
    x, y, z, vx, vy, vz, mm = (np.asarray(a, np.float64) for a in (x, y, z, vx, vy, vz, m))
    n = len(x)
    pts = np.stack([x, y, z], 1)
    if per:
        tree = cKDTree(np.mod(pts + box / 2.0, box), boxsize=box)
        wrap = lambda q: np.mod(q + box / 2.0, box)
    else:
        tree = cKDTree(pts)
        wrap = lambda q: q
    # PPART_DENS
    d, idx = tree.query(wrap(pts), k=K)
    part_dens = mm[idx].sum(1) / ((4.0 / 3.0) * np.pi * d[:, K - 1] ** 3)
    own_rk = d[:, K - 1]
    # VVEL_INTERP_SPH_VW: cells in column-major order
    c = np.arange(nx ** 3)
    ci, cj, ck = c % nx + 1, (c // nx) % nx + 1, c // (nx * nx) + 1
    q = np.stack([rad[ci - off], rad[cj - off], rad[ck - off]], 1)
    dc, ic = tree.query(wrap(q), k=K)
    hpart = np.zeros(n)
    u2, u3, u4 = np.zeros(nx ** 3), np.zeros(nx ** 3), np.zeros(nx ** 3)
    knn = dc[:, K - 1] > dx
    ds, js = dc[knn], ic[knn]
    np.maximum.at(hpart, js.ravel(), ds.ravel())
    w = _m4(ds, ds[:, K - 1:K], gauss) * (mm[js] / part_dens[js])
    b = w.sum(1)
    u2[knn], u3[knn], u4[knn] = (w * vx[js]).sum(1) / b, (w * vy[js]).sum(1) / b, (w * vz[js]).sum(1) / b
    for cc in np.nonzero(~knn)[0]:                      # ball of radius DX
        lst = np.asarray(tree.query_ball_point(wrap(q[cc]), r=dx), np.int64)
        dd = np.sqrt(((_min_image(pts[lst] - q[cc], box) if per else pts[lst] - q[cc]) ** 2).sum(1))
        np.maximum.at(hpart, lst, dd)
        w = _m4(dd, dd.max(), gauss) * (mm[lst] / part_dens[lst])
        u2[cc], u3[cc], u4[cc] = (w * vx[lst]).sum() / w.sum(), (w * vy[lst]).sum() / w.sum(), \
            (w * vz[lst]).sum() / w.sum()
    # FILL_H_ZEROS
    hpart = np.where(hpart > 0.0, hpart, own_rk)
    u_mass = _ddens(x, y, z, hpart, mm, rad, off, nx, dx, gauss=gauss)
    return dict(u_mass=u_mass, u2=u2, u3=u3, u4=u4, hpart=hpart, part_dens=part_dens)


def _min_image(dv, box):
    return dv - box * np.round(dv / box)


def _ddens(x, y, z, h, mm, rad, off, nx, dx, chunk_cells=2 ** 24, gauss=False):
    """DDENS_INTERP_SPH: per particle, the in-grid cells of its (2 INC + 1)^3 box
    with d^2 <= 4 h^2, M4 (or Gaussian exp(-4 d^2 / h^2)) weights normalised to
    the particle's mass."""
    r1 = rad[1 - off]
    cell = lambda v: np.floor((v - r1) / dx).astype(np.int64) + 1
    ix, jy, kz = cell(x), cell(y), cell(z)
    inc = np.floor(2.0 * h / dx + 0.5).astype(np.int64)
    u = np.zeros(nx ** 3)
    radin = rad[np.arange(1, nx + 1) - off]              # RAD(1..NX)
    for v in np.unique(inc):
        ps = np.nonzero(inc == v)[0]
        o = np.arange(-v, v + 1)
        oz, oy, ox = (a.ravel() for a in np.meshgrid(o, o, o, indexing="ij"))
        step = max(1, chunk_cells // len(ox))
        for s in range(0, len(ps), step):
            pp = ps[s:s + step]
            i2, j2, k2 = ix[pp, None] + ox, jy[pp, None] + oy, kz[pp, None] + oz
            ok = (i2 >= 1) & (i2 <= nx) & (j2 >= 1) & (j2 <= nx) & (k2 >= 1) & (k2 <= nx)
            i2c, j2c, k2c = np.clip(i2, 1, nx), np.clip(j2, 1, nx), np.clip(k2, 1, nx)
            d2 = (x[pp, None] - radin[i2c - 1]) ** 2 + (y[pp, None] - radin[j2c - 1]) ** 2 + \
                 (z[pp, None] - radin[k2c - 1]) ** 2
            hh = h[pp, None]
            ok &= d2 <= 4.0 * hh * hh
            w = np.where(ok, _m4(np.sqrt(d2), hh, gauss), 0.0)
            norm = w.sum(1)
            has = norm > 0.0
            contrib = np.where(has[:, None], w * (mm[pp, None] / np.where(has, norm, 1.0)[:, None]), 0.0)
            cid = (i2c - 1) + nx * ((j2c - 1) + nx * (k2c - 1))
            u += np.bincount(cid.ravel(), weights=contrib.ravel(), minlength=nx ** 3)
            # no weight anywhere: the particle's mass goes to its own cell
            lone = pp[~has]
            inside = (ix[lone] >= 1) & (ix[lone] <= nx) & (jy[lone] >= 1) & (jy[lone] <= nx) & \
                     (kz[lone] >= 1) & (kz[lone] <= nx)
            lone = lone[inside]
            np.add.at(u, (ix[lone] - 1) + nx * ((jy[lone] - 1) + nx * (kz[lone] - 1)), mm[lone])
    return u


def _tsc_axis(v, rad, off, nx, dx, periodic):
    """TSC cell and the three weights of one coordinate (particles.f90:56-96)."""
    r1 = rad[1 - off] - 0.5 * dx
    rn = rad[nx - off] + 0.5 * dx
    if periodic:
        leng = rn - r1
        v = np.where(v < r1, v + leng, v)
        v = np.where(v >= rn, v - leng, v)
    i = np.floor((v - rad[1 - off]) / dx + 0.49999).astype(np.int64) + 1
    t0 = 1.5 - np.abs(rad[i - 1 - off] - v) / dx
    t1 = np.abs(rad[i - off] - v) / dx
    t2 = 1.5 - np.abs(rad[i + 1 - off] - v) / dx
    return i, (0.5 * t0 * t0, 0.75 - t1 * t1, 0.5 * t2 * t2)


def tsc_fp64(p, x, y, z, vx, vy, vz, m):
    """(u_mass, u2, u3, u4) of DENS_INTERP_TSC and VEL_INTERP_TSC in FP64
    (particles.f90:16-271; non-periodic cells outside 1..NX are dropped)."""
    from .oracle import grid_setup
    g, radx = grid_setup(p)
    nx, per = int(p.nx), bool(p.periodic)
    dx = float(g.dx)
    rad = np.asarray(radx, np.float64)
    off = int(g.rad_lo)
    x, y, z, vx, vy, vz, mm = (np.asarray(a, np.float64) for a in (x, y, z, vx, vy, vz, m))
    (ci, wx), (cj, wy), (ck, wz) = (_tsc_axis(v, rad, off, nx, dx, per) for v in (x, y, z))
    nc = nx ** 3
    um, s2, s3, s4, wt = (np.zeros(nc) for _ in range(5))
    for a in range(3):
        for b in range(3):
            for c in range(3):
                i3, j3, k3 = ci + c - 1, cj + b - 1, ck + a - 1
                if per:
                    i3, j3, k3 = ((t - 1) % nx + 1 for t in (i3, j3, k3))
                ok = (i3 >= 1) & (i3 <= nx) & (j3 >= 1) & (j3 <= nx) & (k3 >= 1) & (k3 <= nx)
                cid = ((i3 - 1) + nx * ((j3 - 1) + nx * (k3 - 1)))[ok]
                w = (wx[c] * wy[b] * wz[a])[ok]
                um += np.bincount(cid, weights=mm[ok] * w, minlength=nc)
                s2 += np.bincount(cid, weights=vx[ok] * w, minlength=nc)
                s3 += np.bincount(cid, weights=vy[ok] * w, minlength=nc)
                s4 += np.bincount(cid, weights=vz[ok] * w, minlength=nc)
                wt += np.bincount(cid, weights=w, minlength=nc)
    wei = np.where(wt == 0.0, 1.0, wt)
    return dict(u_mass=um, u2=s2 / wei, u3=s3 / wei, u4=s4 / wei)
