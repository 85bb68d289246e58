"""Topography and immersed boundaries, set up on the host.

The reference reads a topographic profile (2D) or an ASCII DEM (3D),
interpolates it on the mesh, turns the cells below it into no-slip walls
with a boundary layer of flag-5 cells above (topo.f), and, with immersed
boundaries, replaces the staircase by forcing points whose velocities are
interpolated every step so that the no-slip condition holds on the
interpolated surface (immb.f, interp.f:321-919), with cut-cell face factors
in the mass balances (ghost.f:2888-3345).

This module is the set-up part: it produces the flags, the forcing-point
tables and the face factors that the engine (and the oracle) read at create.
Everything here runs once per run on the host, in numpy, following the
reference's loops where their order matters (the profile searches, the
carried indices, the in-place flag updates).

Functions follow the reference file by file:

* ``interp_1d`` / ``interp_2d``: arrfil.f:367-511 (``interp``)
* ``mean_filter_2d``: arrfil.f:84-203
* ``read_profile``: topo.f:306-348 (``read_2Dprofile``)
* ``read_dem_ascii``: topo.f:350-469
* ``resize_dem``: topo.f:474-580
* ``Topography.set_profile``: topo.f:145-304, with ``set_flags`` topo.f:1031-1112
* ``Topography.flatten_vent_2d``: topo.f:828-854 (``flatten_dem_vent_2D``)
* ``Topography.interpolate_profile`` / ``interpolate_dem``: topo.f:904-1029
"""
from __future__ import annotations

import math

import numpy as np

FLUID, SLIP, NOSLIP, BL_CELL, FREE_IO, INLET = 1, 2, 4, 5, 8, 16
VENT, IMMB, FILLED1, FILLED2 = 64, 257, 512, 1024


def nint(x):
    """Fortran NINT: round half away from zero."""
    x = np.asarray(x, dtype=np.float64)
    return np.where(x >= 0.0, np.floor(x + 0.5), -np.floor(-x + 0.5)).astype(np.int64)


# ---------------------------------------------------------------------------
# arrfil.f
# ---------------------------------------------------------------------------
def _first_at_or_right(x1, x2):
    """For every x2[i], the 1-based index n of the first x1[n] >= x2[i]
    (0 where there is none), as the scans of interp_1d_array and interp_2d
    (arrfil.f:378-403, 440-471) assign it on ascending arrays."""
    x1 = np.asarray(x1, dtype=np.float64)
    x2 = np.asarray(x2, dtype=np.float64)
    t = np.zeros(x2.size, dtype=np.int64)
    lo = 0
    for n in range(x1.size):
        # the reference's inner loop runs from the first unassigned point
        # to the end and assigns every point at or left of x1[n]
        for i in range(lo, x2.size):
            if x1[n] >= x2[i]:
                t[i] = n + 1
                lo += 1
    return t


def interp_1d(x1, f1, x2):
    """Linear interpolation of the profile (x1, f1) at x2, arrfil.f:367-408.
    Returns (f2, t) with t the 1-based index of the profile point at or
    right of each x2; a point right of the whole profile is an error (the
    reference leaves it undefined and set_profile stops on it)."""
    x1 = np.asarray(x1, dtype=np.float64)
    f1 = np.asarray(f1, dtype=np.float64)
    t = _first_at_or_right(x1, x2)
    if np.any(t == 0):
        raise ValueError("topography: the computational domain exceeds the profile")
    f2 = np.empty(len(x2))
    for i, n in enumerate(t):
        if n == 1:
            f2[i] = f1[0]
        else:
            grad = (f1[n - 1] - f1[n - 2]) / (x1[n - 1] - x1[n - 2])
            f2[i] = f1[n - 2] + (x2[i] - x1[n - 2]) * grad
    return f2, t


def _weights(x1, x2, t):
    """alpha of interp_2d (arrfil.f:480-484): the weight of x1[t] against
    x1[t-1].  Where x2 falls on x1[t] exactly the weight is 1 whatever the
    point to the left (for t = 1 the reference reads outside x1 there and
    multiplies it by 0)."""
    a = np.empty(len(x2))
    for i, n in enumerate(t):
        d2 = x1[n - 1] - x2[i]
        if n == 1:
            if d2 != 0.0:
                raise ValueError("topography: the computational domain exceeds the DEM")
            a[i] = 1.0
        else:
            d1 = x2[i] - x1[n - 2]
            a[i] = d1 / (d1 + d2)
    return a


def interp_2d(x1, y1, f1, x2, y2):
    """Bilinear interpolation of f1 (indexed [i, j] on x1, y1) at the
    points of the mesh (x2, y2), arrfil.f:410-511.  Returns (f2, tx, ty)."""
    x1 = np.asarray(x1, dtype=np.float64)
    y1 = np.asarray(y1, dtype=np.float64)
    f1 = np.asarray(f1, dtype=np.float64)
    tx = _first_at_or_right(x1, x2)
    ty = _first_at_or_right(y1, y2)
    if np.any(tx == 0) or np.any(ty == 0):
        raise ValueError("topography: the computational domain exceeds the DEM")
    alpha = _weights(x1, x2, tx)
    beta = _weights(y1, y2, ty)
    ix, ixm = tx - 1, np.maximum(tx - 2, 0)
    iy, iym = ty - 1, np.maximum(ty - 2, 0)
    A = alpha[:, None]
    B = beta[None, :]
    tp1 = A * f1[np.ix_(ix, iy)] + (1.0 - A) * f1[np.ix_(ixm, iy)]
    tp2 = A * f1[np.ix_(ix, iym)] + (1.0 - A) * f1[np.ix_(ixm, iym)]
    f2 = B * tp1 + (1.0 - B) * tp2
    return f2, tx, ty


def mean_filter_2d(x1, y1, f1, window):
    """Subsample f1 on a uniform grid of spacing `window`, average each
    sample over the points within `window` of it, and interpolate back
    (arrfil.f:84-203).  Returns the filtered copy of f1."""
    x1 = np.asarray(x1, dtype=np.float64)
    y1 = np.asarray(y1, dtype=np.float64)
    f1 = np.asarray(f1, dtype=np.float64)
    cx_n, cy_n = x1.size, y1.size
    nsmx = int((x1[-1] - x1[0]) / window + 1)
    nsmy = int((y1[-1] - y1[0]) / window + 1)
    x2 = np.zeros(nsmx)
    y2 = np.zeros(nsmy)
    f2 = np.zeros((nsmx, nsmy))
    dcx = np.zeros((nsmx, 2), dtype=np.int64)
    dcy = np.zeros((nsmy, 2), dtype=np.int64)
    dcx[:, 0], dcy[:, 0] = cx_n, cy_n
    x2[0], y2[0] = x1[0], y1[0]
    for i in range(1, nsmx - 1):
        x2[i] = x2[i - 1] + window
    for j in range(1, nsmy - 1):
        y2[j] = y2[j - 1] + window
    x2[-1], y2[-1] = x1[-1], y1[-1]
    f2[0, 0] = f1[0, 0]
    f2[-1, -1] = f1[-1, -1]
    f2[0, -1] = f1[0, -1]
    f2[-1, 0] = f1[-1, 0]
    for i in range(1, nsmx - 1):
        sel = np.flatnonzero(np.abs(x1 - x2[i]) <= window)
        for c in sel:
            f2[i, 0] += f1[c, 0]
            f2[i, -1] += f1[c, -1]
        f2[i, 0] /= sel.size
        f2[i, -1] /= sel.size
        dcx[i] = (min(sel.min() + 1, cx_n), max(sel.max() + 1, 0))
    for j in range(1, nsmy - 1):
        sel = np.flatnonzero(np.abs(y1 - y2[j]) <= window)
        for c in sel:
            f2[0, j] += f1[0, c]
            f2[-1, j] += f1[-1, c]
        f2[0, j] /= sel.size
        f2[-1, j] /= sel.size
        dcy[j] = (min(sel.min() + 1, cy_n), max(sel.max() + 1, 0))
    for j in range(1, nsmy - 1):
        ysel = np.abs(y1 - y2[j]) <= window
        for i in range(1, nsmx - 1):
            xsel = np.abs(x1 - x2[i]) <= window
            acc, cnt = 0.0, 0
            # the reference sums row by row (cy outer, cx inner)
            for cy in range(dcy[j, 0] - 1, dcy[j, 1]):
                if not ysel[cy]:
                    continue
                for cx in range(dcx[i, 0] - 1, dcx[i, 1]):
                    if xsel[cx]:
                        acc += f1[cx, cy]
                        cnt += 1
            f2[i, j] = acc / cnt
    out, _, _ = interp_2d(x2, y2, f2, x1, y1)
    return out


# ---------------------------------------------------------------------------
# topography files
# ---------------------------------------------------------------------------
def read_profile(path, seatable=True):
    """2D profile file: the number of points, then one `x z` pair per line
    (topo.f:306-348); negative heights are raised to 0 with seatable."""
    with open(path) as f:
        toks = f.read().split()
    n = int(toks[0])
    vals = np.array([float(t.replace("d", "e").replace("D", "e")) for t in toks[1:1 + 2 * n]])
    xtop, ztop = vals[0::2].copy(), vals[1::2].copy()
    if seatable:
        ztop = np.maximum(ztop, 0.0)
    return xtop, ztop


def write_profile(path, xtop, ztop):
    with open(path, "w") as f:
        f.write(f"{len(xtop)}\n")
        for a, b in zip(xtop, ztop):
            f.write(f"{a:.6f} {b:.6f}\n")


def read_dem_ascii(path):
    """ASCII DEM (topo.f:350-469): six header records (columns, rows,
    x and y of the lower-left corner, cell size, no-data value), then the
    elevations row by row from north to south.  Returns (xdem, ydem, zdem)
    with zdem indexed [i, j], j = 0 the southern row."""
    with open(path) as f:
        toks = f.read().split()

    def num(t):
        return float(t.replace("d", "e").replace("D", "e"))

    # the header records may carry a keyword before the value
    vals, k = [], 0
    while len(vals) < 6:
        t = toks[k]
        k += 1
        try:
            vals.append(num(t))
        except ValueError:
            continue
    nxd, nyd = int(vals[0]), int(vals[1])
    xll, yll, dd = vals[2], vals[3], vals[4]
    z = np.array([num(t) for t in toks[k:k + nxd * nyd]], dtype=np.float64)
    if z.size != nxd * nyd:
        raise ValueError(f"DEM {path}: {z.size} elevations for {nxd} x {nyd}")
    zdem = z.reshape(nyd, nxd)[::-1, :].T.copy()  # rows north -> south
    xdem = xll + np.arange(nxd) * dd
    ydem = yll + np.arange(nyd) * dd
    return xdem, ydem, zdem


def write_dem_ascii(path, xll, yll, cellsize, zdem, nodata=-9999):
    """Write zdem [i, j] (j = 0 southern row) in the layout read_dem_ascii
    reads, rows from north to south."""
    nxd, nyd = zdem.shape
    with open(path, "w") as f:
        f.write(f"ncols {nxd}\nnrows {nyd}\nxllcorner {xll:.6f}\nyllcorner {yll:.6f}\n")
        f.write(f"cellsize {cellsize:.6f}\nNODATA_value {nodata}\n")
        for j in range(nyd - 1, -1, -1):
            f.write(" ".join(f"{v:.4f}" for v in zdem[:, j]) + "\n")


def resize_dem(xdem, ydem, zdem, cellsize, domain_x, domain_y, dxmax, dymax, center_x, center_y,
               alpha_x, alpha_y, filtersize, ismt, dx, dy):
    """Crop the DEM to the domain plus a margin, resample it at `cellsize`
    and low-pass filter it (topo.f:474-580).  Returns (xtop, ytop, ztop2d)."""
    newsizex = domain_x + 2.0 * max(dxmax, cellsize)
    newsizey = domain_y + 2.0 * max(dymax, cellsize)
    ntx = int(newsizex / cellsize) + 1
    nty = int(newsizey / cellsize) + 1
    xll = center_x - alpha_x * domain_x - dxmax
    yll = center_y - alpha_y * domain_y - dymax
    xtop = np.empty(ntx)
    ytop = np.empty(nty)
    xtop[0], ytop[0] = xll, yll
    for i in range(1, ntx):
        xtop[i] = xtop[i - 1] + cellsize
    for j in range(1, nty):
        ytop[j] = ytop[j - 1] + cellsize
    xur = xll + cellsize * (ntx - 1)
    yur = yll + cellsize * (nty - 1)
    if xll < xdem[0] or xur > xdem[-1] or yll < ydem[0] or yur > ydem[-1]:
        raise ValueError("resize_dem: the domain exceeds the DEM limits")
    ztop2d, _, _ = interp_2d(xdem, ydem, zdem, xtop, ytop)
    if filtersize >= cellsize:
        if ismt == 1:
            ztop2d = mean_filter_2d(xtop, ytop, ztop2d, filtersize)
        elif ismt in (2, 3):
            raise ValueError("topography: ismt = 2, 3 (gaussian and barnes filters) are not supported")
    return xtop, ytop, ztop2d


# ---------------------------------------------------------------------------
# topo.f: the topography on the mesh
# ---------------------------------------------------------------------------
def _round_cm(topo):
    """Heights to the centimetre, topo.f:180-186 (NINT(h * 1e2) * 1e-2)."""
    return nint(np.asarray(topo) * 1.0e2).astype(np.float64) * 1.0e-2


class Topography:
    """The topography of one run on the mesh of a Case.

    Holds the profile (2D: xtop, ztop; 3D: xtop, ytop, ztop2d), the index
    arrays of the reference (next, ord; nextx, nexty, ord2d) and, after
    set_profile, the cell flags below and just above the topography.  The
    mesh coordinates (x, xb, y, yb, z, zb) and the flags (fl, indexed
    [k, j, i]) are the Case's arrays, changed in place as the reference
    changes its module arrays."""

    def __init__(self, case):
        self.case = case
        d = case.deck
        self.is3d = case.is3d
        self.nx, self.ny, self.nz = case.nx, case.ny, case.nz
        self.itrans = bool(d["itrans"])
        path = d["dem_file"]
        if not self.is3d:
            self.xtop, self.ztop = read_profile(path, seatable=bool(d["seatable"]))
        else:
            if int(d["iavv"]) >= 1:
                raise ValueError("topography: iavv >= 1 (average_dem) is not supported")
            xdem, ydem, zdem = read_dem_ascii(path)
            dx, dy = case.dx[1:-1], case.dy[1:-1]
            self.xtop, self.ytop, self.ztop2d = resize_dem(
                xdem, ydem, zdem, float(d["cellsize"]), case.domain_x, case.domain_y,
                case.dxmax, case.dymax, float(d["center_x"]), float(d["center_y"]),
                float(d["alpha_x"]), float(d["alpha_y"]), float(d["filtersize"]), int(d["ismt"]), dx, dy)
            # compute_UTM_coords, topo.f:731-751: the mesh moves so that the
            # centre cell sits at (center_x, center_y)
            tx = float(d["center_x"]) - case.x[case.iv - 1]
            ty = float(d["center_y"]) - case.y[case.jv - 1]
            case.x += tx
            case.xb += tx
            case.y += ty
            case.yb += ty
        self.kv = 0

    # set_profile, topo.f:145-304, then set_flags
    def set_profile(self):
        c = self.case
        nx, ny, nz = self.nx, self.ny, self.nz
        if not self.is3d:
            if self.xtop.max() < c.x.max():
                raise ValueError("topography: the computational domain exceeds the topography")
            topo, self.next = interp_1d(self.xtop, self.ztop, c.x)
            topo = _round_cm(topo)
            transl = topo.min() - c.zb[0] if self.itrans else 0.0
            c.z += transl
            c.zb += transl
            self.ord = np.zeros(nx, dtype=np.int64)
            for i in range(nx):
                below = np.flatnonzero(c.zb <= topo[i])
                self.ord[i] = below[-1] + 1 if below.size else 0
            self.dist = (c.z[:, None] - topo[None, :]).reshape(nz, 1, nx)
            self.kv = int(self.ord[c.iv - 1])
        else:
            if self.xtop.max() < c.x.max() or self.ytop.max() < c.y.max():
                raise ValueError("topography: the computational domain exceeds the topography")
            topo2d, self.nextx, self.nexty = interp_2d(self.xtop, self.ytop, self.ztop2d, c.x, c.y)
            topo2d = _round_cm(topo2d)
            transl = topo2d.min() - c.zb[0] if self.itrans else 0.0
            c.z += transl
            c.zb += transl
            # ord2d[i, j]: the last cell whose bottom face is at or below the topography
            cnt = (c.zb[None, None, :] <= topo2d[:, :, None])
            last = np.where(cnt.any(axis=2), nz - np.argmax(cnt[:, :, ::-1], axis=2), 0)
            self.ord2d = last.astype(np.int64)
            self.dist = c.z[:, None, None] - topo2d.T[None, :, :]
            self.kv = int(self.ord2d[c.iv - 1, c.jv - 1])
        self.set_flags()

    # set_flags, topo.f:1031-1112
    def set_flags(self):
        c = self.case
        nx, ny, nz = self.nx, self.ny, self.nz
        fl = c.flag3.reshape(-1)
        if not self.is3d:
            qcol = self.ord.reshape(1, nx)
        else:
            qcol = self.ord2d.T  # [j, i]
        flv = c.flag3
        kk = np.arange(1, nz + 1)[:, None, None]
        q = qcol[None, :, :]
        under = kk <= q
        flv[under & (flv != INLET)] = NOSLIP
        flv[(~under) & (flv == NOSLIP)] = FLUID
        # the boundary layer: rows q+1 .. q+3, columns i-3 .. i+3 (and
        # j-3 .. j+3), by flat index as the reference computes it (an offset
        # past the end of a row lands in the next row); only fluid cells
        # change, so the order of the updates does not matter
        ntot = nx * ny * nz
        jj_, ii_ = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
        qv = qcol.astype(np.int64)
        for dk in (1, 2, 3):
            for dj in (range(-3, 4) if self.is3d else (0,)):
                for di in range(-3, 4):
                    m = (ii_ + di) + nx * ((jj_ + dj) + ny * (qv + dk - 1))
                    m = m[(m >= 0) & (m < ntot)]
                    hit = m[fl[m] == FLUID]
                    fl[hit] = BL_CELL

    # flatten_dem_vent_2D, topo.f:828-854
    def flatten_vent_2d(self, xvent, vent_radius, quota):
        zq = self.case.zb[quota - 1]
        n = self.xtop.size
        for i in range(n):
            if (self.xtop[i] - xvent) ** 2 < vent_radius ** 2:
                self.ztop[i] = zq
                if i + 1 < n:
                    self.ztop[i + 1] = zq
        self.set_profile()

    # interpolate_profile, topo.f:904-968: the topography on a (staggered)
    # mesh, the last row at or below it, and the forced points
    def interpolate_profile(self, cx, cz):
        nx, nz = self.nx, self.nz
        topo, self.next = interp_1d(self.xtop, self.ztop, cx)
        topo = _round_cm(topo)
        ordv = np.zeros(nx, dtype=np.int64)
        for i in range(nx):
            below = np.flatnonzero(np.asarray(cz) <= topo[i])
            ordv[i] = below[-1] + 1 if below.size else 0
        self.ord = ordv
        ff = np.zeros(nx * nz, dtype=bool)
        for i in range(2, nx):
            o, om, op = ordv[i - 1], ordv[i - 2], ordv[i]
            if o - om > 0 and topo[i] - topo[i - 2] >= 0:
                ks = range(om, o + 1)
            elif op - o < 0:
                ks = range(op, o + 1)
            else:
                ks = (o,)
            for k in ks:
                ff[(i - 1) + (k - 1) * nx] = True
        return topo, ff

    # interpolate_dem, topo.f:970-1029
    def interpolate_dem(self, cx, cy, cz):
        nx, ny, nz = self.nx, self.ny, self.nz
        topo2d, self.nextx, self.nexty = interp_2d(self.xtop, self.ytop, self.ztop2d, cx, cy)
        cz = np.asarray(cz)
        cnt = (cz[None, None, :] <= topo2d[:, :, None])
        ord2d = np.where(cnt.any(axis=2), nz - np.argmax(cnt[:, :, ::-1], axis=2), 0).astype(np.int64)
        self.ord2d = ord2d
        # forced cells (topo.f:1004-1023): in the interior columns, the rows
        # 2 .. ord2d - 1 above the lowest of the eight neighbours' ord2d,
        # and the row ord2d itself
        ff = np.zeros((nz, ny, nx), dtype=bool)
        o = ord2d[1:-1, 1:-1]
        nb = np.minimum.reduce([ord2d[:-2, 1:-1], ord2d[:-2, :-2], ord2d[1:-1, :-2], ord2d[2:, :-2],
                                ord2d[2:, 1:-1], ord2d[2:, 2:], ord2d[1:-1, 2:], ord2d[:-2, 2:]])
        kk = np.arange(1, nz + 1)[:, None, None]
        band = (kk >= 2) & (kk <= (o.T - 1)[None]) & (kk > nb.T[None])
        ff[:, 1:-1, 1:-1] = band
        ii, jj = np.meshgrid(np.arange(2, nx), np.arange(2, ny), indexing="ij")
        oo = o.astype(np.int64)
        ok = oo >= 1
        ff[oo[ok] - 1, jj[ok] - 1, ii[ok] - 1] = True
        ff = ff.reshape(-1)
        return topo2d, ff


# ---------------------------------------------------------------------------
# immb.f: forcing points
# ---------------------------------------------------------------------------
# neighbour directions of the 3D forcing points (immb.f:937-952): 1 W, 2 SW,
# 3 S, 4 SE, 5 E, 6 NE, 7 N, 8 NW
_DI = (0, -1, -1, 0, 1, 1, 1, 0, -1)
_DJ = (0, 0, -1, -1, -1, 0, 1, 1, 1)


class ForcingPoint:
    """One forcing point (immb.f:31-43): mesh indices (1-based), the
    interpolation type, the offset of the fluid neighbour used by the 3D
    interpolation, and the no-slip point on the topography."""
    __slots__ = ("i", "j", "k", "int", "di", "dj", "dk", "nx_", "ny_", "nz_", "q", "qq")

    def __init__(self, i, j, k, kind, di=0, dj=0, dk=0, nsl=(0.0, 0.0, 0.0)):
        self.i, self.j, self.k, self.int = i, j, k, kind
        self.di, self.dj, self.dk = di, dj, dk
        self.nx_, self.ny_, self.nz_ = nsl
        self.q = 0   # 1-based flat index of the first interpolation neighbour (3D)
        self.qq = 0  # of the second


def _sol2(a11, a12, a21, a22, b1, b2):
    """immb.f:896-907 (Cramer's rule, second unknown)."""
    return (a11 * b2 - b1 * a21) / (a11 * a22 - a12 * a21)


class ImmersedBoundaries:
    """Forcing points, flags and cut-cell face factors of one run:
    set_forcing (immb.f:73-516), local_forcing (ghost.f:2888-3050),
    fill_cells (ghost.f:3052-3261) and face_fractions (ghost.f:3263-3321)."""

    def __init__(self, topo: Topography):
        self.t = topo
        self.case = c = topo.case
        self.nx, self.ny, self.nz = c.nx, c.ny, c.nz
        if not c.is3d:
            self._set_forcing_2d()
        else:
            self._set_forcing_3d()
        self._local_forcing()
        self._fill_cells()
        self._face_fractions()

    # -- 2D ------------------------------------------------------------------
    def _set_forcing_2d(self):
        t, c = self.t, self.case
        nx, nz = self.nx, self.nz
        fl = c.flag3[:, 0, :]  # view [k, i]
        x, xb, z, zb = c.x, c.xb, c.z, c.zb
        topo_x, forcex = t.interpolate_profile(xb, z)
        topo_c, forcez = t.interpolate_profile(x, zb)
        extfx = np.zeros(nx * nz, dtype=bool)
        extfz = np.zeros(nx * nz, dtype=bool)

        def setfill(i, k):
            if fl[k - 1, i - 1] not in (INLET, VENT):
                fl[k - 1, i - 1] = FILLED1

        for k in range(2, nz + 1):
            for i in range(2, nx):
                ijk = (k - 1) * nx + i - 1
                imjk = ijk - 1
                ijkm = ijk - nx
                if forcez[ijk] and forcex[ijk] and z[k - 1] > topo_x[i - 2]:
                    extfx[imjk] = True
                    setfill(i, k)
                if forcez[ijk] and forcex[imjk] and z[k - 1] > topo_x[i - 1]:
                    extfx[ijk] = True
                    setfill(i, k)
                if forcex[imjk] and forcex[ijk] and forcez[ijkm] and zb[k - 1] > topo_c[i - 1]:
                    extfz[ijk] = True
                    setfill(i, k)
        nfpx = int(forcex.sum() + extfx.sum())
        nfpz = int(forcez.sum() + extfz.sum())
        # along x
        topo_x, forcex = t.interpolate_profile(xb, z)
        fptx = self._forcing2d(xb, z, topo_x)
        for k in range(2, nz + 1):
            for i in range(2, nx):
                if extfx[(k - 1) * nx + i - 1]:
                    fptx.append(self._ext_forcing2d(i, k, xb, z, topo_x, fptx))
        self._mark_immb_2d(fptx)
        # along z
        topo_c, forcez = t.interpolate_profile(x, zb)
        fptz = self._forcing2d(x, zb, topo_c)
        for k in range(2, nz + 1):
            for i in range(2, nx):
                if extfz[(k - 1) * nx + i - 1]:
                    fptz.append(self._ext_forcing2d(i, k, x, zb, topo_c, fptz))
        self._mark_immb_2d(fptz)
        if len(fptx) != nfpx or len(fptz) != nfpz:
            raise ValueError(f"immersed boundaries: {len(fptx)}/{nfpx} x and {len(fptz)}/{nfpz} z forcing "
                             "points (the reference leaves the rest undefined)")
        self.fptx, self.fpty, self.fptz = fptx, [], fptz
        self.topo_x, self.topo_c = topo_x, topo_c

    def _mark_immb_2d(self, fpts):
        fl = self.case.flag3[:, 0, :]
        for p in fpts:
            f = fl[p.k - 1, p.i - 1]
            if p.k > 1 and f not in (INLET, VENT, FILLED1):
                fl[p.k - 1, p.i - 1] = IMMB

    def _forcing2d(self, cx, cz, topo):
        """forcing2d, immb.f:589-910: the forcing points of each column along
        an increasing, decreasing or flat stretch of the profile."""
        t = self.t
        nx = self.nx
        ordv, nxt = t.ord, t.next
        xtop, ztop = t.xtop, t.ztop
        out = []

        def segs(a, b):
            # the profile segments n-1 .. n for n = next(a) .. next(b)
            return range(int(nxt[a - 1]), int(nxt[b - 1]) + 1)

        def nsl_row(n1, n2, k, rising):
            hit = None
            for n in segs(n1, n2):
                if rising:
                    ok = ztop[n - 2] <= cz[k - 1] and ztop[n - 1] >= cz[k - 1]
                else:
                    ok = ztop[n - 2] >= cz[k - 1] and ztop[n - 1] <= cz[k - 1]
                if ok:
                    grad = (xtop[n - 1] - xtop[n - 2]) / (ztop[n - 1] - ztop[n - 2])
                    hit = (xtop[n - 2] + (cz[k - 1] - ztop[n - 2]) * grad, cz[k - 1])
            return hit

        def add(i, k, kind, nsl):
            fp = ForcingPoint(i, 0, k, kind)
            if nsl is not None:
                fp.nx_, fp.nz_ = nsl
            out.append(fp)

        for i in range(2, nx):
            o, om, op = int(ordv[i - 1]), int(ordv[i - 2]), int(ordv[i])
            if o - om > 0 and topo[i] - topo[i - 2] >= 0:
                # increasing_profile, immb.f:633-746 (the last match wins, as
                # the reference's loops overwrite)
                kref = om
                norm = (cx[i - 2] - cx[i - 1], cz[om] - cz[om - 1])
                hits = [h for h in self._all_diag(norm, i - 1, i, i, kref, cx, cz)]
                add(i, kref, -3, hits[-1] if hits else None)
                for k in range(om + 1, o):
                    add(i, k, -2, nsl_row(i - 1, i, k, True))
                norm = (topo[i - 2] - topo[i - 1], cx[i - 1] - cx[i - 2])
                hits = [h for h in self._all_diag(norm, i - 1, i, i, o, cx, cz)]
                add(i, o, -1, hits[-1] if hits else None)
            elif op - o < 0:
                # decreasing_profile, immb.f:748-862
                norm = (topo[i - 1] - topo[i], cx[i] - cx[i - 1])
                hits = [h for h in self._all_diag(norm, i, i + 1, i, o, cx, cz)]
                add(i, o, 1, hits[-1] if hits else None)
                for k in range(o - 1, op, -1):
                    add(i, k, 2, nsl_row(i, i + 1, k, False))
                norm = (cx[i] - cx[i - 1], cz[op] - cz[op - 1])
                hits = [h for h in self._all_diag(norm, i, i + 1, i, op, cx, cz)]
                add(i, op, 3, hits[-1] if hits else None)
            else:
                # stationnary_profile, immb.f:864-881
                add(i, o, 0, (cx[i - 1], topo[i - 1]))
        return out

    def _all_diag(self, norm, n1, n2, i, kref, cx, cz):
        t = self.t
        xtop, ztop, nxt = t.xtop, t.ztop, t.next
        for n in range(int(nxt[n1 - 1]), int(nxt[n2 - 1]) + 1):
            dxt = xtop[n - 1] - xtop[n - 2]
            dzt = ztop[n - 1] - ztop[n - 2]
            dxs = xtop[n - 1] - cx[i - 1]
            dzs = ztop[n - 1] - cz[kref - 1]
            with np.errstate(divide="ignore", invalid="ignore"):
                s = _sol2(norm[0], dxt, norm[1], dzt, dxs, dzs)
            if 0 <= s <= 1:
                yield (s * xtop[n - 2] + (1 - s) * xtop[n - 1], s * ztop[n - 2] + (1 - s) * ztop[n - 1])

    def _ext_forcing2d(self, i, k, cx, cz, topo, fpts):
        """ext_forcing2d, immb.f:518-587."""
        t = self.t
        xtop, ztop, nxt = t.xtop, t.ztop, t.next
        droite = any(f.i == i + 1 and f.k == k for f in fpts)
        gauche = any(f.i == i - 1 and f.k == k for f in fpts)
        fp = ForcingPoint(i, 0, k, 20)
        if droite and not gauche:
            fp.int = 21
            for n in range(int(nxt[i - 1]), int(nxt[i]) + 1):
                if ztop[n - 2] <= cz[k - 1] and ztop[n - 1] >= cz[k - 1]:
                    grad = (xtop[n - 1] - xtop[n - 2]) / (ztop[n - 1] - ztop[n - 2])
                    fp.nx_, fp.nz_ = xtop[n - 2] + (cz[k - 1] - ztop[n - 2]) * grad, cz[k - 1]
        elif gauche and not droite:
            fp.int = 22
            for n in range(int(nxt[i - 2]), int(nxt[i - 1]) + 1):
                if ztop[n - 2] >= cz[k - 1] and ztop[n - 1] <= cz[k - 1]:
                    grad = (xtop[n - 1] - xtop[n - 2]) / (ztop[n - 1] - ztop[n - 2])
                    fp.nx_, fp.nz_ = xtop[n - 2] + (cz[k - 1] - ztop[n - 2]) * grad, cz[k - 1]
        else:
            fp.nx_, fp.nz_ = cx[i - 1], topo[i - 1]
        return fp

    # -- 3D ------------------------------------------------------------------
    def _set_forcing_3d(self):
        t, c = self.t, self.case
        nx, ny, nz = self.nx, self.ny, self.nz
        fl = c.flag3.reshape(-1)
        x, xb, y, yb, z, zb = c.x, c.xb, c.y, c.yb, c.z, c.zb
        tx, forcex = t.interpolate_dem(xb, y, z)
        ty, forcey = t.interpolate_dem(x, yb, z)
        tc, forcez = t.interpolate_dem(x, y, zb)
        n = nx * ny * nz
        extf = [np.zeros(n, dtype=bool) for _ in range(3)]

        def idx(i, j, k):
            return (i - 1) + nx * (j - 1) + nx * ny * (k - 1)

        # one or two faces above the topography (immb.f:231-359): every
        # interior cell's pattern bds depends only on the topography, so the
        # cells are classified at once
        K, J, I = np.meshgrid(np.arange(2, nz), np.arange(2, ny), np.arange(2, nx), indexing="ij")
        zk, zbk, zbkm = z[K - 1], zb[K - 1], zb[K - 2]
        bds = ((zk > tx[I - 1, J - 1]) * 1 + (zk > tx[I - 2, J - 1]) * 2 + (zbk > tc[I - 1, J - 1]) * 4
               + (zbkm >= tc[I - 1, J - 1]) * 8 + (zk > ty[I - 1, J - 1]) * 16 + (zk > ty[I - 1, J - 2]) * 32)
        if np.any(bds == 8):
            raise ValueError("set_forcing: inconsistent immersed boundary (immb.f:302)")
        m_all = (I - 1) + nx * (J - 1) + nx * ny * (K - 1)
        # per pattern: the (axis, cell offset) pairs forced externally
        rules = {1: ((0, 0),), 2: ((0, -1),), 4: ((2, 0),), 16: ((1, 0),), 32: ((1, -nx),),
                 17: ((0, 0), (1, 0)), 18: ((0, -1), (1, 0)), 34: ((0, -1), (1, -nx)),
                 33: ((0, 0), (1, -nx)), 48: ((1, 0), (1, -nx)), 3: ((0, 0), (0, -1))}
        for pat, rule in rules.items():
            m = m_all[bds == pat]
            if m.size == 0:
                continue
            for axis, off in rule:
                extf[axis][m + off] = True
            keep = (fl[m] != INLET) & (fl[m] != VENT)
            fl[m[keep]] = FILLED1 if len(rule) == 1 else FILLED2
        nfp = [int(forcex.sum() + extf[0].sum()), int(forcey.sum() + extf[1].sum()),
               int(forcez.sum() + extf[2].sum())]
        fpts = []
        meshes = ((xb, y, z), (x, yb, z), (x, y, zb))
        for axis in range(3):
            cx, cy, cz = meshes[axis]
            topo2d, _ = t.interpolate_dem(cx, cy, cz)
            lst = []
            for m in np.flatnonzero(extf[axis]):
                i, j, k = m % nx + 1, (m // nx) % ny + 1, m // (nx * ny) + 1
                lst.append(self._ext_forcing3d(i, j, k, cx, cy, cz, topo2d, axis + 1))
            lst.extend(self._forcing3d(cx, cy, cz, topo2d))
            for p in lst:
                if p.i > 1 and p.j > 1 and p.k > 1:
                    mm = idx(p.i, p.j, p.k)
                    if fl[mm] not in (INLET, VENT, FILLED1, FILLED2):
                        fl[mm] = IMMB
            if len(lst) != nfp[axis]:
                raise ValueError(f"immersed boundaries: {len(lst)} forcing points along axis {axis + 1}, "
                                 f"{nfp[axis]} counted (the reference leaves the rest undefined)")
            fpts.append(lst)
            if axis == 0:
                self.topo_x = topo2d
            elif axis == 1:
                self.topo_y = topo2d
            else:
                self.topo_c = topo2d
        self.fptx, self.fpty, self.fptz = fpts

    def _gamma(self, i, j, k, index, cz, topo2d):
        num = cz[k - 1] - topo2d[i - 1, j - 1]
        den = topo2d[i - 1 + _DI[index], j - 1 + _DJ[index]] - topo2d[i - 1, j - 1]
        with np.errstate(divide="ignore", invalid="ignore"):
            return np.float64(num) / np.float64(den)

    def _forcing3d(self, cx, cy, cz, topo2d):
        """forcing3d, immb.f:913-1069."""
        o2 = self.t.ord2d
        nx, ny = self.nx, self.ny
        out = []
        for i in range(2, nx):
            for j in range(2, ny):
                o = int(o2[i - 1, j - 1])
                # rows at or below every neighbour's ord2d have no candidate
                lo = min(int(o2[i - 1 + _DI[n], j - 1 + _DJ[n]]) for n in range(1, 9))
                for k in range(max(2, lo + 1), o):
                    g = [-1.0] * 9
                    for n in range(1, 9):
                        if o2[i - 1 + _DI[n], j - 1 + _DJ[n]] < k:
                            g[n] = self._gamma(i, j, k, n, cz, topo2d)
                    if max(g[1:]) > -1:
                        # mingam, immb.f:1045-1067: the neighbour whose gamma
                        # is closest to 1/2 (the first of equals)
                        ming, gint = 1.0, 0
                        for n in range(1, 9):
                            if abs(0.5 - g[n]) < ming:
                                ming, gint = abs(0.5 - g[n]), n
                        fp = ForcingPoint(i, j, k, gint, _DI[gint], _DJ[gint], 0)
                        gg = g[gint]
                        fp.nx_ = gg * cx[i - 1] + (1.0 - gg) * cx[i - 1 + _DI[gint]]
                        fp.ny_ = gg * cy[j - 1] + (1.0 - gg) * cy[j - 1 + _DJ[gint]]
                        fp.nz_ = cz[k - 1]
                        out.append(fp)
                if o < 1:
                    # a column whose topography lies below the first face
                    # (interpolate_dem does not round to the centimetre as
                    # set_profile does, so the translated mesh can leave one
                    # there): the reference writes this point past the end of
                    # its table (the count of topo.f:1021-1022 skips it) and
                    # never reads it back
                    continue
                fp = ForcingPoint(i, j, o, 0, 0, 0, 1, (cx[i - 1], cy[j - 1], topo2d[i - 1, j - 1]))
                out.append(fp)
        return out

    def _ext_forcing3d(self, i, j, k, cx, cy, cz, topo2d, axis):
        """ext_forcing3d, immb.f:1071-1261."""
        o2 = self.t.ord2d
        g = [-1.0] * 9
        gext = [0.0] * 5
        maxg = 1.0
        gmin = 0
        gint, fpint = 0, 0
        if k > o2[i - 1, j - 1]:
            for n in range(1, 9):
                if o2[i - 1 + _DI[n], j - 1 + _DJ[n]] >= k:
                    g[n] = self._gamma(i, j, k, n, cz, topo2d)
            if axis != 1:
                gext[1] = g[1] * g[5]
            gext[2] = g[2] * g[6]
            if axis != 2:
                gext[3] = g[3] * g[7]
            gext[4] = g[4] * g[8]
            for l in range(1, 5):
                if gext[l] < 0 and -gext[l] < maxg:
                    gmin, maxg = l, -gext[l]
            if min(gext[1:]) < 0 and gmin:
                a, b = gmin, gmin + 4
                if g[a] < 0:
                    gint, fpint = b, 20 + gmin
                else:
                    gint, fpint = a, 24 + gmin
        if k == o2[i - 1, j - 1] + 1:
            maxg_z = (cz[k - 1] - topo2d[i - 1, j - 1]) / (cz[k] - topo2d[i - 1, j - 1])
        else:
            maxg_z = 1.0
        if maxg < 1 and maxg < maxg_z:
            d = fpint - 20
            fp = ForcingPoint(i, j, k, fpint, _DI[d], _DJ[d], 0)
            gg = g[gint]
            fp.nx_ = (1.0 - gg) * cx[i - 1] + gg * cx[i - 1 + _DI[gint]]
            fp.ny_ = (1.0 - gg) * cy[j - 1] + gg * cy[j - 1 + _DJ[gint]]
            fp.nz_ = cz[k - 1]
        else:
            fp = ForcingPoint(i, j, k, 20, 0, 0, 1, (cx[i - 1], cy[j - 1], topo2d[i - 1, j - 1]))
        return fp

    # -- ghost.f -------------------------------------------------------------
    def _local_forcing(self):
        """local_forcing, ghost.f:2888-3050: the forcing point of each cell
        along each axis (1-based into the axis's list, 0 for none) and, in
        3D, the flat indices of the interpolation neighbours."""
        nx, ny, nz = self.nx, self.ny, self.nz
        n = nx * ny * nz
        self.num = [np.zeros(n, dtype=np.int32) for _ in range(3)]
        for axis, lst in enumerate((self.fptx, self.fpty, self.fptz)):
            for npt, p in enumerate(lst, start=1):
                if p.i == 0 or p.k == 0 or (self.case.is3d and p.j == 0):
                    raise ValueError("local_forcing: control num (ghost.f:2930)")
                if not self.case.is3d:
                    m = (p.i - 1) + nx * (p.k - 1)
                else:
                    m = (p.i - 1) + nx * (p.j - 1) + nx * ny * (p.k - 1)
                    q = (p.i + p.di - 1) + nx * (p.j + p.dj - 1) + nx * ny * (p.k + p.dk - 1)
                    qq = (p.i + 2 * p.di - 1) + nx * (p.j + 2 * p.dj - 1) + nx * ny * (p.k + 2 * p.dk - 1)
                    p.q = q + 1
                    if p.int % 2 != 0 or p.int == 0:
                        p.qq = qq + 1
                # a later point of the same cell and axis replaces an earlier one
                self.num[axis][m] = npt

    def _fill_cells(self):
        """fill_cells, ghost.f:3052-3261: the faces of each fluid cell that lie
        above the topography (bd, bit 1 E, 2 W, 4 T, 8 B, 16 N, 32 S) and its
        fluid volume fraction vf; a cell with none becomes filled_cell_1."""
        c = self.case
        nx, ny, nz = self.nx, self.ny, self.nz
        fl = c.flag3.reshape(-1)
        n = nx * ny * nz
        is3d = c.is3d
        z, zb = c.z, c.zb
        m = np.arange(n)
        i, j, k = m % nx + 1, (m // nx) % ny + 1, m // (nx * ny) + 1
        # raw neighbours, clamped at the mesh edge as myijk clamps them
        ip = np.where(i < nx, m + 1, m)
        im = np.where(i > 1, m - 1, m)
        jp = np.where(j < ny, m + nx, m)
        jm = np.where(j > 1, m - nx, m)
        km = np.where(k > 1, m - nx * ny, m)
        zk, zbk = z[k - 1], zb[k - 1]
        zbkm = np.where(k > 1, zb[np.maximum(k - 2, 0)], -np.inf)
        if not is3d:
            tx, tc = self.topo_x, self.topo_c
            faces = [(zk > tx[i - 1], ip, 1), (zk > tx[np.maximum(i - 2, 0)], im, 2),
                     (zbk > tc[i - 1], None, 4), (zbkm >= tc[i - 1], km, 8)]
            full = 4
        else:
            tx, ty, tc = self.topo_x, self.topo_y, self.topo_c
            faces = [(zk > tx[i - 1, j - 1], ip, 1), (zk > tx[np.maximum(i - 2, 0), j - 1], im, 2),
                     (zbk > tc[i - 1, j - 1], None, 4), (zbkm >= tc[i - 1, j - 1], km, 8),
                     (zk > ty[i - 1, j - 1], jp, 16), (zk > ty[i - 1, np.maximum(j - 2, 0)], jm, 32)]
            full = 6
        fluid = (fl & 1) == 1
        allup = np.ones(n, dtype=bool)
        for cond, _, _ in faces:
            allup &= cond
        # a fluid cell whose faces all lie above the topography and whose
        # neighbours are not filled (and cannot become filled: only cells
        # with a face below the topography can) has every face open and
        # vf = 1; the others are visited in the reference's order, because a
        # cell that turns filled changes the count of the cells after it
        cand = fluid & ~allup
        near = cand.copy()
        filled = (fl == FILLED1) | (fl == FILLED2)
        for _, nb, _ in faces:
            if nb is not None:
                near |= fluid & (filled[nb] | cand[nb])
        bd = np.zeros(n, dtype=np.int32)
        vf = np.zeros(n, dtype=np.float64)
        easy = fluid & ~near
        bd[easy] = sum(bit for _, _, bit in faces)
        vf[easy] = float(full) / full
        conds = [np.asarray(cnd) for cnd, _, _ in faces]
        for mm in np.flatnonzero(near):
            v, b = 0.0, 0
            for (cond, nb, bit), cc in zip(faces, conds):
                if not cc[mm]:
                    continue
                if nb is None:
                    b += bit
                    v += 1.0
                    continue
                f = fl[nb[mm]]
                if f == FILLED1:
                    v += 2.0
                elif is3d and f == FILLED2:
                    v += 1.0
                else:
                    b += bit
                    v += 1.0
            v = v / full
            bd[mm] = b
            vf[mm] = v
            if v == 0.0:
                fl[mm] = FILLED1
        self.bd, self.vf = bd, vf

    def _face_fractions(self):
        """face_fractions, ghost.f:3263-3321: the per-face factors b_e .. b_b
        (kept here as the bits of bd, default all six set) and ivf = 1 / vf.
        The reference leaves the routine (RETURN, not CYCLE) at the first
        fluid cell that is a forcing point along both x and z, after zeroing
        that cell's x and z factors; the cells after it keep the defaults
        (all faces open, ivf = 1), and so do they here."""
        c = self.case
        fl = c.flag3.reshape(-1)
        n = fl.size
        faces = np.full(n, 63, dtype=np.int32)
        ivf = np.ones(n, dtype=np.float64)
        fluid = (fl & 1) == 1
        both = np.flatnonzero(fluid & (self.num[0] != 0) & (self.num[2] != 0))
        stop = int(both[0]) if both.size else n
        sel = np.flatnonzero(fluid[:stop])
        faces[sel] = self.bd[sel]
        with np.errstate(divide="ignore"):
            ivf[sel] = np.where(self.vf[sel] > 0.0, 1.0 / np.where(self.vf[sel] > 0.0, self.vf[sel], 1.0), 0.0)
        if stop < n:
            faces[stop] &= ~(1 | 2 | 4 | 8)
        self.stopped_at = stop if stop < n else -1
        self.faces, self.ivf = faces, ivf
