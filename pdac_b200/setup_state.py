"""Host-side run set-up: mesh, cell flags, atmosphere, vent and initial state.

This is the once-per-run part of PDAC that precedes the time loop
(pdac.f:108-281).  It is host logic, restated in numpy from:
  grid_setup / flic        grid.f:206-483
  set_atmosphere           atmosphere.f:81-142, compute_profile :150-230,
                           hydrostatic :240-264
  locate_vent_2D           vent.f:130-246
  set_atmc / specified_flow / cnvert / set_ventc
                           setup.f:204-275, 397-498, 280-390; vent.f:443-581
The result is a :class:`Case` holding the metric, flags, hydrostatic
profile, vent cell list and an initial :class:`State` in the reference
layout, plus the ``pdac_cfg`` structure for the C ABI.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import abi
from .deck import Deck, MAX_NGAS

# cell flags, grid.f:45-58
FLUID, SLIP, NOSLIP, FREE_IO, INLET, ZERO_GRAD, VENT = 1, 2, 4, 8, 16, 32, 64
BL_CELL = 5  # boundary-layer cell, grid.f:48 (no-slip bit + fluid bit)


def _nint(x):
    """Fortran NINT of a non-negative value (half away from zero)."""
    return int(math.floor(x + 0.5))

# setup.f:563-571 (g/mol) and 608
GMW = np.array([32.0, 28.0, 44.0, 2.0, 18.0, 28.96442, 64.0]) * 1.0e-3
RGAS = 8.31432


def hcapg(tg, icpc=2, tref=298.0):
    """Per-species specific heats [J/(kg K)], hcapgs.f:33-85 (vectorised)."""
    t1 = np.full_like(np.asarray(tg, dtype=np.float64), tref) if icpc <= 1 else np.asarray(tg, dtype=np.float64)
    t2 = t1 * t1
    t3 = t1 * t2
    cp = np.stack([
        (2.811e1 - 3.68e-6 * t1 + 1.746e-5 * t2 - 1.065e-8 * t3),
        (3.115e1 - 1.357e-2 * t1 + 2.680e-5 * t2 - 1.168e-8 * t3),
        (1.980e1 + 7.344e-2 * t1 - 5.602e-5 * t2 + 1.715e-8 * t3),
        (2.714e1 + 9.274e-3 * t1 - 1.381e-5 * t2 + 7.645e-9 * t3),
        (3.224e1 + 1.924e-3 * t1 + 1.055e-5 * t2 - 3.596e-9 * t3),
        (3.0413e1 - 1.059e-2 * t1 + 2.458e-5 * t2 - 1.135e-8 * t3),
        (2.385e1 + 6.699e-2 * t1 - 4.961e-5 * t2 + 1.328e-8 * t3)])
    cp = cp / GMW.reshape((7,) + (1,) * t1.ndim)
    if icpc == 0:
        cp[4] = 1810.0
        cp[5] = 1004.0
    return cp


def mole(ygc, gas_type):
    """Mass to molar fractions, eosg.f:38-68; ygc has shape (ngas, ...)."""
    g = GMW[np.asarray(gas_type) - 1].reshape((-1,) + (1,) * (ygc.ndim - 1))
    mol = np.zeros(ygc.shape[1:])
    for ig in range(ygc.shape[0]):
        mol = mol + ygc[ig] / g[ig]
    molinv = np.where(np.abs(mol) <= 1e-10, 0.0, 1.0 / np.where(mol == 0, 1.0, mol))
    return np.stack([ygc[ig] / g[ig] * molinv for ig in range(ygc.shape[0])])


def mas(xgc, gas_type):
    """Molar to mass fractions, eosg.f:70-99; xgc has shape (ngas, ...)."""
    g = GMW[np.asarray(gas_type) - 1].reshape((-1,) + (1,) * (xgc.ndim - 1))
    mass = np.zeros(xgc.shape[1:])
    for ig in range(xgc.shape[0]):
        mass = mass + xgc[ig] * g[ig]
    massinv = np.where(np.abs(mass) < 1e-10, 0.0, 1.0 / np.where(mass == 0, 1.0, mass))
    return np.stack([xgc[ig] * g[ig] * massinv for ig in range(xgc.shape[0])])


def _powi(x, n):
    """x**n for an integer n by repeated squaring, as Fortran evaluates an
    integer power."""
    r, b, e = 1.0, x, abs(n)
    while e:
        if e & 1:
            r = r * b
        b = b * b
        e >>= 1
    return r if n >= 0 else 1.0 / r


def _fnint(x):
    """Fortran NINT: nearest integer, halves away from zero."""
    return int(math.floor(abs(x) + 0.5)) * (1 if x >= 0 else -1)


def generate_grid(nd, domain_size, alpha, demin, demax, n0, maxbeta):
    """generate_grid, grid.f:485-786: nd cell sizes between demin (a band
    of n0 cells around the relative position alpha) and demax, growing at a
    constant rate found by adjusting it until the cells fill domain_size,
    rounded to 1e-4 of the length unit."""
    if demin == demax:
        return np.full(nd, float(demin))
    if nd < domain_size / demax:
        raise ValueError("grid_generator: insufficient number of cells")
    if nd > domain_size / demin:
        raise ValueError("grid_generator: number of cells is too big")
    if domain_size * alpha < demin:
        alpha = 0.0
    if domain_size * (1.0 - alpha) < demin:
        alpha = 1.0
    if alpha == 0.0:
        n01, n02 = 0, n0
        l1, l2 = 0.0, domain_size - n02 * demin
    elif alpha == 1.0:
        n01, n02 = n0, 0
        l1, l2 = domain_size - n01 * demin, 0.0
    else:
        n01 = _fnint(n0 / 2.0)
        n02 = n0 - n01
        l1 = (domain_size * alpha) - n01 * demin
        l2 = (domain_size * (1.0 - alpha)) - n02 * demin
    der = demax / demin
    beta, dbeta, minbeta = 1.2, 0.99, 1.0 + 1.0e-5
    print_mesh, already = False, False

    def side(l, n0s, frac_alpha, m, lcomp):
        if l < 0:
            return int(frac_alpha * domain_size / demin), 0.0, 0, 0
        if (l / demax) > (nd - n0s):
            raise ValueError("grid: insufficient number of cells")
        if lcomp < l:
            return n0s, l, m, int((l - lcomp) / demax)
        return n0s, l, int(math.log(1.0 + (beta - 1.0) * (l / demin + 1.0)) / math.log(beta) - 1), 0

    while not print_mesh:
        m = int(math.log(der) / math.log(beta))
        frac = (_powi(beta, m + 1) - 1.0) / (beta - 1.0)
        lcomp = demin * (frac - 1.0)
        n01, l1, m1, n11 = side(l1, n01, alpha, m, lcomp)
        n02, l2, m2, n12 = side(l2, n02, 1.0 - alpha, m, lcomp)
        if (l2 + l1) / demax > nd - n01 - n02:
            raise ValueError("grid: insufficient number of cells")
        tot = (n01 + m1 + n11) + (n02 + m2 + n12)
        if tot < nd:
            if beta * dbeta < minbeta:
                print_mesh = True
            else:
                if already:
                    dbeta = dbeta + (1.0 - dbeta) / 2.0
                    already = False
                beta = beta * dbeta
        elif tot > nd:
            if not already:
                dbeta = dbeta + (1.0 - dbeta) / 2.0
                already = True
            beta = beta / dbeta
        else:
            if (1.0 - dbeta) <= 1.0e-15:
                print_mesh = True
            else:
                already = True
                beta = beta / dbeta

    def refit(l, n1, m1_, realexp):
        while True:
            ntilde = (l - n1 * demax) / demin + 1.0
            b1 = beta
            if ntilde > 1.0:
                for _ in range(50):
                    num = (m1_ * (math.pow(b1, m1_ + 1.0) if realexp else _powi(b1, m1_ + 1)) + 1.0) / ntilde
                    b1 = (1.0 - num) / (1.0 - (m1_ + 1.0) * _powi(b1, m1_) / ntilde)
            if demin * _powi(b1, m1_) > demax:
                if m1_ == 0 or b1 > maxbeta:
                    return n1, m1_, b1
                n1, m1_ = n1 + 1, m1_ - 1
            else:
                return n1, m1_, b1

    n11, m1, beta1 = refit(l1, n11, m1, False)
    n12, m2, beta2 = refit(l2, n12, m2, True)   # the reference raises beta2 to the real m2 + 1.D0
    center = n11 + m1 + n01
    delta = np.full(nd, float(demax))
    for i in range(1, m1 + 1):
        delta[center - n01 - i] = demin * _powi(beta1, i)
    delta[center - n01:center + n02] = demin
    for i in range(1, m2 + 1):
        delta[center + n02 + i - 1] = demin * _powi(beta2, i)
    return np.array([_fnint(v * 10000.0) / 10000.0 for v in delta])


def thermal_eosg(tg, p, xgc, gas_type):
    """Ideal-gas density, eosg.f:114-137."""
    mg = np.zeros_like(np.asarray(tg, dtype=np.float64))
    for ig, gt in enumerate(gas_type):
        mg = mg + xgc[ig] * GMW[gt - 1]
    return p / (RGAS * tg) * mg


def hydrostatic(zb, z, grad, tb, pb, gravz):
    """atmosphere.f:240-264."""
    erreair = RGAS / GMW[5]
    if grad != 0.0:
        cost = gravz / (erreair * grad)
        t = tb + grad * (z - zb)
        p = pb * (t / tb) ** cost
    else:
        cost = gravz / (erreair * tb)
        t = tb
        p = pb * math.exp(cost * (z - zb))
    return t, p


def atmosphere_profile(deck, z):
    """set_atmosphere + compute_profile, atmosphere.f:81-230."""
    names = ("troposphere", "tropopause", "lower_stratosphere", "upper_stratosphere", "ozone_layer",
             "lower_mesosphere", "upper_mesosphere")
    layers = []
    ptop, ttop = deck["p_ground"], deck["t_ground"]
    gz = deck["gravz"]
    for li, nm in enumerate(names):
        zbot = layers[li - 1]["ztop"] if li > 0 else 0.0
        ztop = deck[f"{nm}_z"]
        gradt = deck[f"{nm}_grad"]
        pbot, tbot = ptop, ttop
        ttop, ptop = hydrostatic(zbot, ztop, gradt, tbot, pbot, gz)
        layers.append(dict(ztop=ztop, gradt=gradt, ptop=ptop, ttop=ttop))
    nz = len(z)
    p_atm = np.zeros(nz)
    t_atm = np.zeros(nz)
    if z[0] <= layers[0]["ztop"]:
        lidx = 1
    else:
        lidx = 2
        while lidx <= len(layers) and not (z[0] > layers[lidx - 2]["ztop"]):
            lidx += 1
    for k in range(nz):
        za = z[k]
        if za > 0.0:
            if not deck["stratification"]:
                zbot, pbot, tbot, gradt = 0.0, deck["p_ground"], deck["t_ground"], 0.0
            else:
                if za > layers[lidx - 1]["ztop"]:
                    lidx += 1
                if lidx == 1:
                    zbot, pbot, tbot = 0.0, deck["p_ground"], deck["t_ground"]
                else:
                    zbot = layers[lidx - 2]["ztop"]
                    pbot = layers[lidx - 2]["ptop"]
                    tbot = layers[lidx - 2]["ttop"]
                gradt = layers[lidx - 1]["gradt"]
            ta, pa = hydrostatic(zbot, za, gradt, tbot, pbot, gz)
        else:
            ta, pa = deck["t_ground"], deck["p_ground"]
        t_atm[k] = ta
        p_atm[k] = pa
    return p_atm, t_atm


class State(dict):
    """Prognostic fields in the reference layout (flat numpy float64 arrays)."""

    def copy(self):
        return State({k: v.copy() for k, v in self.items()})


class Case:
    """A fully set-up run: metric, flags, atmosphere, vent, state, cfg."""

    def __init__(self, deck: Deck, precision=abi.PREC_FP64):
        self.deck = deck
        bad = deck.check()
        if bad:
            raise ValueError("unsupported options: " + ", ".join(bad))
        self.is3d = deck.is3d
        self.nx = int(deck["nx"])
        self.ny = int(deck["ny"]) if self.is3d else 1
        self.nz = int(deck["nz"])
        self.ncell = self.nx * self.ny * self.nz
        self.nsolid = int(deck["nsolid"])
        self.ngas = int(deck["ngas"])
        self.precision = precision
        self.gas_type = deck.gas_types()
        self._grid()
        self._flags()
        # pdac.f:138-191: import_topography, locate_vent, export_topography,
        # set_forcing; the atmosphere (setup, pdac.f:267) sees the mesh as
        # the topography left it
        self.topography = None
        self.ib = None
        if int(deck["itp"]) >= 1:
            from .topography import Topography
            self.topography = Topography(self)
            self.topography.set_profile()
        self._vent()
        self._export_topography()
        if int(deck["itp"]) >= 1 and int(deck["immb"]) == 1:
            from .topography import ImmersedBoundaries
            self.ib = ImmersedBoundaries(self.topography)
            self.flag = self.flag3.reshape(-1).copy()
        self.p_atm, self.t_atm = atmosphere_profile(deck, self.z)
        self.state = self._initial_state()

    # grid.f:206-345
    def _grid(self):
        d = self.deck
        if d["grigen"] == 1:
            # grid_setup (grid.f:244-256): generated non-uniform mesh
            if any(d[k] != 0 for k in ("npx", "nmx", "npy", "nmy", "npz", "nmz")):
                raise ValueError("grigen=1 with added cells (npx, nmx, ...) is not supported")
            self.dx = generate_grid(self.nx, d["domain_x"], d["alpha_x"], d["dxmin"], d["dxmax"], max(d["n0x"], 1),
                                    d["maxbeta"])
            self.dy = (generate_grid(self.ny, d["domain_y"], d["alpha_y"], d["dymin"], d["dymax"], max(d["n0y"], 1),
                                     d["maxbeta"]) if self.is3d else np.zeros(1))
            self.dz = generate_grid(self.nz, d["domain_z"], d["alpha_z"], d["dzmin"], d["dzmax"], max(d["n0z"], 1),
                                    d["maxbeta"])
        elif d["grigen"] != 0:
            raise ValueError("grigen=2 (generate_nu_grid) is not supported")
        elif d["iuni"] == 1:
            self.dx = np.full(self.nx, float(d["dx0"]))
            self.dy = np.full(self.ny, float(d["dy0"])) if self.is3d else np.zeros(1)
            self.dz = np.full(self.nz, float(d["dz0"]))
        elif d["grigen"] == 0:
            self.dx = np.asarray(d.delta_x, dtype=np.float64)
            self.dy = np.asarray(d.delta_y, dtype=np.float64) if self.is3d else np.zeros(1)
            self.dz = np.asarray(d.delta_z, dtype=np.float64)
        nx, nz = self.nx, self.nz
        self.xb = np.zeros(nx)
        self.x = np.zeros(nx)
        self.x[0] = -0.5 * self.dx[0] + self.xb[0]
        for i in range(1, nx):
            self.xb[i] = self.xb[i - 1] + self.dx[i]
            self.x[i] = self.xb[i] - 0.5 * self.dx[i]
        ny = self.ny
        self.yb = np.zeros(ny)
        self.y = np.zeros(ny)
        if self.is3d:
            self.y[0] = -0.5 * self.dy[0]
            for j in range(1, ny):
                self.yb[j] = self.yb[j - 1] + self.dy[j]
                self.y[j] = self.yb[j] - 0.5 * self.dy[j]
        self.zb = np.zeros(nz)
        self.z = np.zeros(nz)
        self.zb[0] = float(d["zzero"])
        self.z[0] = -0.5 * self.dz[0] + self.zb[0]
        for k in range(1, nz):
            self.zb[k] = self.zb[k - 1] + self.dz[k]
            self.z[k] = self.zb[k] - 0.5 * self.dz[k]
        self.itc = int(d["itc"]) if not self.is3d else 0
        # mesh centre cell and domain extent of a prescribed mesh without
        # added cells (grid.f:229-239); the topography needs them
        self.iv = _nint(nx / 2.0)
        self.jv = _nint(ny / 2.0) if self.is3d else 1
        self.domain_x, self.dxmax = float(np.sum(self.dx)), float(np.max(self.dx))
        self.domain_y = float(np.sum(self.dy)) if self.is3d else 0.0
        self.dymax = float(np.max(self.dy)) if self.is3d else 0.0

    def idx(self, i, j, k):
        """1-based (i, j, k) -> flat 0-based index."""
        return (i - 1) + self.nx * ((j - 1) + self.ny * (k - 1))

    # flic, grid.f:375-483
    def _flags(self):
        d = self.deck
        nx, ny, nz = self.nx, self.ny, self.nz
        fl = np.full((nz, ny, nx), FLUID, dtype=np.int32)
        if not self.is3d:
            fl[0, 0, 1:nx - 1] = 2 ** (d["bottom"] - 1)
            fl[nz - 1, 0, 1:nx - 1] = 2 ** (d["top"] - 1)
            fl[:, 0, 0] = 2 ** (d["west"] - 1)
            fl[:, 0, nx - 1] = 2 ** (d["east"] - 1)
        else:
            fl[0, 1:ny - 1, 1:nx - 1] = 2 ** (d["bottom"] - 1)
            fl[nz - 1, 1:ny - 1, 1:nx - 1] = 2 ** (d["top"] - 1)
            fl[:, :, 0] = 2 ** (d["west"] - 1)
            fl[:, :, nx - 1] = 2 ** (d["east"] - 1)
            fl[:, 0, :] = 2 ** (d["south"] - 1)
            fl[:, ny - 1, :] = 2 ** (d["north"] - 1)
        for b in d.blocks:
            ys = slice(b["ylo"] - 1, b["yhi"]) if self.is3d else slice(0, 1)
            fl[b["zlo"] - 1:b["zhi"], ys, b["xlo"] - 1:b["xhi"]] = 2 ** (b["typ"] - 1)
            if self.is3d and b["typ"] == 8:
                fl[b["zlo"] - 1:b["zhi"], ys, b["xlo"] - 1:b["xhi"]] = 129
        self.flag3 = fl

    # locate_vent_2D, vent.f:130-246 (3D square vents are given as type-5 blocks)
    def _vent(self):
        d = self.deck
        self.vent = []  # dicts: ijk (0-based), frac, dist
        if d["ivent"] < 1:
            self.flag = self.flag3.reshape(-1).copy()
            return
        if self.is3d:
            raise ValueError("circular vents in 3D (locate_vent_3D) are not supported; use a FIXED_FLOWS block")
        nx, nz = self.nx, self.nz
        fl = self.flag3[:, 0, :]
        xvent = d["xvent"]
        iv = _nint(nx / 2.0)
        in_center = bool(d["vent_in_center"]) and self.topography is None  # vent.f:79
        if xvent == -99999.0:
            xvent = self.x[iv - 1] if in_center else self.xb[iv - 1]
        iiv = 1
        for i in range(1, nx + 1):
            if self.x[i - 1] <= xvent:
                iiv = i
        if iiv == 1 or self.itc == 1:
            iiv = 2
        xvent = self.xb[iiv - 2]
        if self.topography is None:
            kkv = 1
            for k in range(1, nz):
                if fl[k - 1, iiv - 1] in (SLIP, NOSLIP):
                    kkv = k
            quota = kkv
        else:
            # the vent sits on the topography, which is flattened around it
            # (vent.f:165-178, flatten_dem_vent_2D topo.f:828-854)
            quota = int(self.topography.ord[iiv - 1])
            self.topography.flatten_vent_2d(xvent, d["vent_radius"], quota)
            fl = self.flag3[:, 0, :]
        vr = d["vent_radius"]
        iwest, ieast = 2, 2
        for i in range(2, nx + 1):
            if self.xb[i - 2] <= (xvent - vr):
                iwest = i
            if self.xb[i - 2] < (xvent + vr):
                ieast = i
        nvt = ieast - iwest + 1
        for nv, i in enumerate(range(iwest, ieast + 1), start=1):
            for k in range(1, quota):
                fl[k - 1, i - 1] = NOSLIP
            k = quota
            frac = 1.0
            if nv == nvt:
                if self.itc == 1:
                    frac = 1.0 - (self.xb[ieast - 1] - self.xb[iwest - 2] - vr) / self.dx[ieast - 1]
                else:
                    frac = 1.0 - (self.xb[ieast - 1] - self.xb[iwest - 2] - 2.0 * vr) / self.dx[ieast - 1]
            fl[k - 1, i - 1] = VENT
            self.vent.append(dict(ijk=self.idx(i, 1, k), i=i, k=k, frac=frac, dist=self.x[i - 1] - xvent))
            for kk in range(quota + 1, nz):
                fl[kk - 1, i - 1] = FLUID
        self.flag3[:, 0, :] = fl
        self.flag = self.flag3.reshape(-1).copy()

    # export_topography, topo.f:1114-1181, which pdac.f:180 calls for every
    # run: a fluid cell up to three rows above the last no-slip cell below it
    # in its column becomes a boundary-layer cell (flag 5).  Such cells take
    # first-order fluxes, because the MUSCL corrections and the limiters test
    # flag == fluid (flux_*.f, iter.f:634-897, tilde.f:955-1248).  The
    # reference carries the row of the last no-slip cell from one column to
    # the next (j, then i, then k, i fastest among the columns), so a column
    # with no no-slip cell (a vent column) uses the previous column's; before
    # the first no-slip cell the reference leaves it undefined, and it is 0
    # here.  The level of the last no-slip cell's bottom face is kept per
    # column as topo_c (the discrete topography the immersed boundaries
    # start from).
    def _export_topography(self):
        nx, ny, nz = self.nx, self.ny, self.nz
        fl = self.flag3.reshape(nz, ny * nx)
        ncol = ny * nx
        kk = np.arange(1, nz + 1, dtype=np.int64)[:, None]
        noslip = fl == NOSLIP
        # row (1-based) of the last no-slip cell at or below each cell, 0 if none
        below = np.maximum.accumulate(np.where(noslip, kk, 0), axis=0)
        last = below[-1]
        has = last > 0
        # the value carried into each column from the columns before it
        src = np.maximum.accumulate(np.where(has, np.arange(ncol), -1))
        carried_out = np.where(src >= 0, last[np.maximum(src, 0)], 0)
        carried_in = np.concatenate(([0], carried_out[:-1]))
        q = np.where(below > 0, below, carried_in[None, :])
        bl = (fl == FLUID) & (kk <= q + 3)
        fl[bl] = BL_CELL
        self.flag3 = fl.reshape(nz, ny, nx)
        self.flag = self.flag3.reshape(-1).copy()
        zb = np.asarray(self.zb, dtype=np.float64)
        self.topo_c = np.where(has, zb[np.maximum(last - 1, 0)], 0.0).reshape(ny, nx)

    def _initial_state(self):
        d = self.deck
        n, ns, ng = self.ncell, self.nsolid, self.ngas
        kk = np.repeat(np.arange(self.nz), self.nx * self.ny)
        st = State()
        for name in abi.STATE_CELL:
            st[name] = np.zeros(n)
        for name in abi.STATE_SOLID:
            st[name] = np.zeros(n * ns)
        for name in abi.STATE_GAS:
            st[name] = np.zeros(n * ng)
        rl = np.array(d["density"][:ns], dtype=np.float64)
        # set_atmc, setup.f:204-275
        st["p"][:] = self.p_atm[kk]
        st["tg"][:] = self.t_atm[kk]
        st["ep"][:] = d["void_fraction"]
        atm = d.atm_ygc()
        Y = st["ygc"].reshape(ng, n)
        for ig, gt in enumerate(self.gas_type):
            Y[ig, :] = atm[gt - 1]
        RL = st["rlk"].reshape(ns, n)
        TS = st["ts"].reshape(ns, n)
        for s in range(ns):
            RL[s] = rl[s] * (1.0 - st["ep"]) / ns
            TS[s] = st["tg"]
        moving = np.isin(self.flag, (FLUID, FREE_IO, ZERO_GRAD))
        st["ug"][moving] = d["wind_x"]
        st["wg"][moving] = d["wind_z"]
        if self.is3d:
            st["vg"][moving] = d["wind_y"]
        for name, src in (("us", "ug"), ("ws", "wg"), ("vs", "vg")):
            A = st[name].reshape(ns, n)
            for s in range(ns):
                A[s, moving] = st[src][moving]
        # specified_flow, setup.f:397-498
        for b in d.blocks:
            if b["typ"] not in (1, 5):
                continue
            for k in range(b["zlo"], b["zhi"] + 1):
                for j in (range(b["ylo"], b["yhi"] + 1) if self.is3d else (1,)):
                    for i in range(b["xlo"], b["xhi"] + 1):
                        c = self.idx(i, j, k)
                        st["ug"][c] = b["ug"]
                        if self.is3d:
                            st["vg"][c] = b["vg"]
                        st["wg"][c] = b["wg"]
                        st["tg"][c] = b["tg"]
                        st["p"][c] = b["p"]
                        st["ep"][c] = 1.0 - sum(s_["eps"] for s_ in b["solids"])
                        for ig, gt in enumerate(self.gas_type):
                            Y[ig, c] = b["ygc"][gt - 1]
                        for s, sd in enumerate(b["solids"]):
                            TS[s, c] = sd["t"]
                            st["us"][s * n + c] = sd["u"]
                            if self.is3d:
                                st["vs"][s * n + c] = sd["v"]
                            st["ws"][s * n + c] = sd["w"]
                            RL[s, c] = sd["eps"] * rl[s]
                        if Y[:, c].sum() != 1.0:
                            Y[ng - 1, c] = 1.0 - Y[:ng - 1, c].sum()
        # set_ventc, vent.f:443-581 (uniform inlet; iali 4 = velocity profile)
        if d["ivent"] >= 1:
            vy = d.vent_ygc()
            for v in self.vent:
                c = v["ijk"]
                st["ug"][c] = d["u_gas"]
                st["wg"][c] = d["w_gas"]
                st["tg"][c] = d["t_gas"]
                st["ep"][c] = 1.0 - sum(d["ep_solid"][:ns])
                st["p"][c] = d["p_gas"]
                for ig, gt in enumerate(self.gas_type):
                    Y[ig, c] = vy[gt - 1]
                for s in range(ns):
                    st["us"][s * n + c] = d["u_solid"][s]
                    st["ws"][s * n + c] = d["w_solid"][s]
                    TS[s, c] = d["t_solid"][s]
                    RL[s, c] = d["ep_solid"][s] * rl[s]
                if Y[:, c].sum() != 1.0:
                    Y[ng - 1, c] = 1.0 - Y[:ng - 1, c].sum()
                if d["iali"] == 4:
                    ra = min(v["dist"] / d["vent_radius"], 1.0)
                    if d["inlet_profile"] == 1:
                        bet = (1.0 if (not self.is3d and self.itc == 0) else 2.0) / (d["wrat"] - 1.0)
                        fac = d["wrat"] * (1.0 - ra ** bet)
                    else:
                        fac = 0.5 * (1.0 - math.tanh(0.25 * d["rbyb"] * (ra - 1.0 / ra))) if ra > 0 else 1.0
                    st["ug"][c] = d["u_gas"] * fac
                    st["wg"][c] = d["w_gas"] * fac
                    for s in range(ns):
                        st["us"][s * n + c] = d["u_solid"][s] * fac
                        st["ws"][s * n + c] = d["w_solid"][s] * fac
                elif d["iali"] in (1, 2, 3) and v["frac"] != 1.0:
                    raise ValueError("vent antialiasing iali=1..3 on partial cells is not supported")
        # cnvert, setup.f:280-390 (itd <= 1)
        X = mole(Y, self.gas_type)
        st["xgc"][:] = X.reshape(-1)
        if d["density_specified"]:
            # setup.f:319-327: the temperature slot holds a density, turned
            # into the temperature of the thermal equation of state
            mass = np.zeros(n)
            for ig, gt in enumerate(self.gas_type):
                mass = mass + X[ig] * GMW[gt - 1]
            tem = st["p"] * mass / RGAS / st["tg"]
            st["tg"][:] = tem
            for s in range(ns):
                TS[s] = tem
        st["rog"][:] = thermal_eosg(st["tg"], st["p"], X, self.gas_type)
        st["rgp"][:] = st["rog"] * st["ep"]
        cp = hcapg(st["tg"], d["icpc"], d["tref"])
        hc = np.zeros(n)
        for ig, gt in enumerate(self.gas_type):
            hc = hc + cp[gt - 1] * Y[ig]
        st["cg"][:] = hc
        st["sieg"][:] = (st["tg"] - 0.0) * st["cg"] + 0.0
        cps = np.array(d["specific_heat"][:ns], dtype=np.float64)
        SI = st["sies"].reshape(ns, n)
        for s in range(ns):
            SI[s] = (TS[s] - 0.0) * cps[s] + 0.0
        return st

    # ---- C ABI configuration ---------------------------------------------
    def cfg(self):
        """Build a ``pdac_cfg``; the returned object keeps its arrays alive."""
        d = self.deck
        c = abi.PdacCfg()
        c.job_type = 3 if self.is3d else 2
        c.nx, c.ny, c.nz = self.nx, self.ny, self.nz
        c.itc = self.itc
        c.nsolid, c.ngas = self.nsolid, self.ngas
        for ig, gt in enumerate(self.gas_type):
            c.gas_type[ig] = gt
        c.dt = d["dt"]
        c.rungekut = d["rungekut"]
        c.time_integration = d["time_integration"]
        c.alpha, c.alphagrav = d["alpha"], d["alphagrav"]
        c.omega, c.delg = d["omega"], d["delg"]
        c.inmax, c.maxout = d["inmax"], d["maxout"]
        c.cstop = int(bool(d["cstop"]))
        c.muscl, c.lv, c.lm = d["muscl"], d["vel_limiter"], d["mass_limiter"]
        c.beta, c.flim = d["beta"], d["flim"]
        c.update_eosg = int(bool(d["update_eosg"]))
        c.implicit_fluxes = int(bool(d["implicit_fluxes"]))
        c.implicit_enthalpy = int(bool(d["implicit_enthalpy"]))
        c.optimization = int(d["optimization"])
        c.pmodel, c.drag_model, c.icpc = d["pmodel"], d["drag_model"], d["icpc"]
        c.tref = d["tref"]
        c.gas_viscosity = int(bool(d["gas_viscosity"]))
        c.part_viscosity = int(bool(d["part_viscosity"]))
        c.repulsive_model = d["repulsive_model"]
        c.iturb, c.modturbo, c.iss, c.cmut = int(d["iturb"]), int(d["modturbo"]), int(d["iss"]), float(d["cmut"])
        c.gravx, c.gravy, c.gravz = d["gravx"], d["gravy"], d["gravz"]
        for s in range(self.nsolid):
            c.dk[s] = d["diameter"][s] * 1.0e-6
            c.rl[s] = d["density"][s]
            c.phis[s] = d["sphericity"][s]
            c.cmus[s] = d["viscosity"][s]
            c.cps[s] = d["specific_heat"][s]
            c.kap[s] = d["thermal_conductivity"][s]
            c.plim[s] = d["twophase_limit"][s]
        c.void_fraction = d["void_fraction"]
        for g, v in enumerate(d.atm_ygc()):
            c.atm_ygc[g] = v
        c.irand = d["irand"]
        c.isink = int(d["isink"])
        c.rprox, c.rdist = float(d["rprox"]), float(d["rdist"])
        c.center_x, c.center_y = float(d["center_x"]), float(d["center_y"])
        c.compute_mixture = int(bool(d["compute_mixture"]))
        c.formatted_output = int(bool(d["formatted_output"]))
        c.precision = self.precision
        keep = dict(dx=np.ascontiguousarray(self.dx), dy=np.ascontiguousarray(self.dy),
                    dz=np.ascontiguousarray(self.dz), flag=np.ascontiguousarray(self.flag, dtype=np.int32),
                    p_atm=np.ascontiguousarray(self.p_atm), t_atm=np.ascontiguousarray(self.t_atm),
                    vent=np.array([v["ijk"] for v in self.vent] or [0], dtype=np.int32))
        c.dx, c.dy, c.dz = abi.dptr(keep["dx"]), abi.dptr(keep["dy"]), abi.dptr(keep["dz"])
        c.flag = abi.iptr(keep["flag"])
        c.p_atm, c.t_atm = abi.dptr(keep["p_atm"]), abi.dptr(keep["t_atm"])
        c.nvent = len(self.vent)
        c.vent_ijk = abi.iptr(keep["vent"])
        for name in ("x", "xb", "y", "yb", "z", "zb"):
            keep[name] = np.ascontiguousarray(getattr(self, name), dtype=np.float64)
            setattr(c, name, abi.dptr(keep[name]))
        # the ground level under each column for the roughness length of the
        # sub-grid model (turbo.f:72-101): export_topography's, or the
        # immersed boundaries' interpolated profile / DEM when they replaced it
        # (immb.f:117-119, 227-230); i fastest
        if self.ib is not None:
            tc = np.asarray(self.ib.topo_c, dtype=np.float64)
            tc = tc.T.reshape(-1) if tc.ndim == 2 else tc.reshape(-1)
        else:
            tc = np.asarray(self.topo_c, dtype=np.float64).reshape(-1)
        keep["topo_c"] = np.ascontiguousarray(tc)
        c.topo_c = abi.dptr(keep["topo_c"])
        c.zrough = float(d["zrough"])
        c.immb = 0
        if self.ib is not None:
            ib = self.ib
            c.immb = 1
            keep["ib_faces"] = np.ascontiguousarray(ib.faces, dtype=np.int32)
            keep["ib_ivf"] = np.ascontiguousarray(ib.ivf, dtype=np.float64)
            c.ib_faces, c.ib_ivf = abi.iptr(keep["ib_faces"]), abi.dptr(keep["ib_ivf"])
            for a, lst in enumerate((ib.fptx, ib.fpty, ib.fptz)):
                keep[f"ib_num{a}"] = np.ascontiguousarray(ib.num[a], dtype=np.int32)
                fp = np.array([[p.i, p.j, p.k, p.int, p.q - 1, p.qq - 1] for p in lst] or [[0, 0, 0, 0, -1, -1]],
                              dtype=np.int32)
                nsl = np.array([[p.nx_, p.ny_, p.nz_] for p in lst] or [[0.0, 0.0, 0.0]], dtype=np.float64)
                keep[f"ib_fp{a}"], keep[f"ib_nsl{a}"] = np.ascontiguousarray(fp), np.ascontiguousarray(nsl)
                c.ib_num[a] = abi.iptr(keep[f"ib_num{a}"])
                c.ib_nfp[a] = len(lst)
                c.ib_fp[a] = abi.iptr(keep[f"ib_fp{a}"])
                c.ib_nsl[a] = abi.dptr(keep[f"ib_nsl{a}"])
        c._keep = keep
        return c

    def fluid_count(self):
        return int(np.count_nonzero(self.flag & 1))
