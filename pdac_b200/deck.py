"""PDAC input deck: Fortran namelists and cards with the reference defaults.

Restates the reader of input.f: the namelists ``control, model, mesh,
boundaries, topography, inlet, dome, atmosphere, particles, numeric``
(input.f:159-209), their defaults (input.f:219-468), the ``MESH`` and
``FIXED_FLOWS`` cards (input.f:788-886) and the derived values of
check_input / initc (input.f:912-1105).  Defaults that the reference writes
as single-precision literals (``omega = 1.1``, ``maxbeta = 1.2`` ...) are
kept at the value the Fortran compiler stores, i.e. rounded through float32.
"""
from __future__ import annotations

import re

import numpy as np


def f32(x):
    """A Fortran REAL(4) literal promoted to REAL(8)."""
    return float(np.float32(x))


MAX_NSOLID = 8
MAX_NGAS = 7
GAS_NAMES = ("O2", "N2", "CO2", "H2", "H2O", "Air", "SO2")


def _defaults():
    d = {}
    d["control"] = dict(
        run_name="pdac_run_2d", job_type="2D", restart_mode="from_scratch", time=0.0, tstop=100.0,
        dt=0.01, lpr=0, imr=0, isrt=0, imrt=0, tpr=1.0, tdump=20.0, nfil=0, formatted_output=False,
        formatted_input=False, max_seconds=f32(40000.0), tau=0.0, tau1=0.0, tau2=0.0, ift=1, cstop=False)
    d["model"] = dict(
        icpc=2, irex=1, compute_mixture=False, isink=0, gas_viscosity=True, part_viscosity=True,
        density_specified=False, iss=0, repulsive_model=1, iturb=1, modturbo=1, pmodel=2, drag_model=1,
        cmut=0.1, gravx=0.0, gravy=0.0, gravz=-9.81, ngas=2, rprox=f32(0.0), rdist=f32(25000.0), tref=298.0)
    d["mesh"] = dict(
        nx=100, nz=100, ny=1, npx=0, npz=0, npy=0, nmx=0, nmz=0, nmy=0, n0x=1, n0y=1, n0z=1, itc=0,
        grigen=0, maxbeta=f32(1.2), mesh_partition=1, iuni=0, dz0=20.0, dx0=20.0, dy0=20.0,
        dxmin=10.0, dymin=10.0, dzmin=10.0, dxmax=100.0, dymax=100.0, dzmax=100.0,
        alpha_x=0.5, alpha_y=0.5, alpha_z=0.0, center_x=0.0, center_y=0.0,
        domain_x=10.0e3, domain_y=10.0e3, domain_z=10.0e3, zzero=0.0)
    d["boundaries"] = dict(west=2, east=2, bottom=3, top=4, south=2, north=2, immb=0, ibl=0, ord=0)
    d["topography"] = dict(
        dem_file="topo.dat", itp=0, ismt=1, iavv=0, min_angle=0.0, max_angle=0.0, nocrater=False,
        itrans=True, seatable=True, rim_quota=1000.0, filtersize=100, cellsize=10, zrough=1.0,
        write_improfile=True)
    d["inlet"] = dict(
        ivent=0, iali=4, irand=0, ipro=0, isl=0, inlet_profile=2, mass_flow_rate=0.0,
        vent_in_center=True, rad_file="profile.rad", xvent=-99999.0, yvent=-99999.0,
        vent_radius=100.0, base_radius=200.0, crater_radius=500.0, u_gas=0.0, v_gas=0.0,
        w_gas=0.0, wrat=1.0, rbyb=11.2, p_gas=1.01325e5, t_gas=288.15,
        u_solid=[0.0] * MAX_NSOLID, v_solid=[0.0] * MAX_NSOLID, w_solid=[0.0] * MAX_NSOLID,
        ep_solid=[0.0] * MAX_NSOLID, t_solid=[288.15] * MAX_NSOLID,
        vent_O2=0.0, vent_N2=0.0, vent_CO2=0.0, vent_H2=0.0, vent_H2O=1.0, vent_Air=0.0, vent_SO2=0.0)
    d["dome"] = dict(idome=0, idw=0, domegeom=1)
    d["atmosphere"] = dict(
        wind_x=0.0, wind_y=0.0, wind_z=0.0, stratification=True, p_ground=1.01325e5,
        t_ground=288.15, void_fraction=1.0 - 1.0e-10, max_packing=f32(0.6413),
        atm_O2=0.0, atm_N2=0.0, atm_CO2=0.0, atm_H2=0.0, atm_H2O=0.0, atm_Air=1.0, atm_SO2=0.0,
        troposphere_z=1.1e4, tropopause_z=2.0e4, lower_stratosphere_z=3.2e4,
        upper_stratosphere_z=4.7e4, ozone_layer_z=5.1e4, lower_mesosphere_z=7.1e4,
        upper_mesosphere_z=8.0e4, troposphere_grad=-6.5e-3, tropopause_grad=0.0,
        lower_stratosphere_grad=1.0e-3, upper_stratosphere_grad=2.8e-3, ozone_layer_grad=0.0,
        lower_mesosphere_grad=-2.8e-3, upper_mesosphere_grad=-2.0e-3)
    d["particles"] = dict(
        nsolid=2, diameter=[100.0] * MAX_NSOLID, density=[2700.0] * MAX_NSOLID,
        sphericity=[1.0] * MAX_NSOLID, viscosity=[0.5] * MAX_NSOLID,
        specific_heat=[1.2e3] * MAX_NSOLID, thermal_conductivity=[2.0] * MAX_NSOLID,
        twophase_limit=[1.0e-8] * MAX_NSOLID)
    d["numeric"] = dict(
        rungekut=1, beta=0.25, mass_limiter=2, vel_limiter=2, muscl=0, inmax=8, maxout=500,
        delg=1.0e-8, omega=f32(1.1), optimization=1, implicit_fluxes=False, implicit_enthalpy=False,
        update_eosg=False, rlim=1.0e-8, flim=1.0e-6, alpha=1.0, alphagrav=0.0, ctu=0,
        time_integration=0, adapt_dt=False, lim_type=2)
    return d


NAMELIST_ORDER = ("control", "model", "mesh", "boundaries", "topography", "inlet", "dome",
                  "atmosphere", "particles", "numeric")


def _parse_value(tok):
    t = tok.strip()
    if not t:
        return None
    up = t.upper()
    if up in (".TRUE.", "T", ".T."):
        return True
    if up in (".FALSE.", "F", ".F."):
        return False
    if (t[0] == t[-1]) and t[0] in "'\"":
        return t[1:-1]
    num = t.replace("d", "e").replace("D", "e")
    try:
        if re.fullmatch(r"[+-]?\d+", num):
            return int(num)
        return float(num)
    except ValueError:
        return t


def _split_values(s):
    out, cur, q = [], "", None
    for ch in s:
        if q:
            cur += ch
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
            cur += ch
        elif ch in ",":
            out.append(cur)
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur)
    vals = []
    for item in out:
        item = item.strip()
        if not item:
            continue
        m = re.fullmatch(r"(\d+)\*(.+)", item)
        if m:
            vals.extend([_parse_value(m.group(2))] * int(m.group(1)))
        else:
            vals.extend(_parse_value(x) for x in item.split())
    return vals


class _ListReader:
    """Fortran list-directed input over the records (lines) after the
    namelists: each read() is one READ statement."""

    def __init__(self, lines):
        self.lines = list(lines)
        self.pos = 0

    @staticmethod
    def _items(line):
        out, cur, q = [], "", None
        for ch in line:
            if q:
                if ch == q:
                    q = None
                else:
                    cur += ch
            elif ch in "'\"":
                q = ch
            elif ch == "," or ch.isspace():
                if cur:
                    out.append(cur)
                cur = ""
            elif ch == "/":
                if cur:
                    out.append(cur)
                out.append("/")
                cur = ""
                break
            else:
                cur += ch
        if cur:
            out.append(cur)
        return out

    def find_card(self, name):
        """READ(unit,*) card until TRIM(card) == name; False at the end."""
        while self.pos < len(self.lines):
            items = self._items(self.lines[self.pos])
            self.pos += 1
            if items and items[0] == name:
                return True
        return False

    def read(self, count):
        vals = []
        while len(vals) < count:
            if self.pos >= len(self.lines):
                raise ValueError("input ended inside a card")
            items = self._items(self.lines[self.pos])
            self.pos += 1
            for it in items:
                if it == "/" or len(vals) >= count:
                    break
                m = re.fullmatch(r"(\d+)\*(.*)", it)
                rep, tok = (int(m.group(1)), m.group(2)) if m else (1, it)
                v = float(tok.replace("d", "e").replace("D", "e"))
                vals.extend([v] * rep)
            if items and items[-1] == "/":
                break
        return vals[:count]


class Deck:
    """All namelist groups plus the MESH and FIXED_FLOWS cards of one run."""

    def __init__(self):
        self.nml = _defaults()
        self.delta_x = None
        self.delta_y = None
        self.delta_z = None
        self.blocks = []  # FIXED_FLOWS blocks: dicts

    # ---- namelist access -------------------------------------------------
    def __getitem__(self, key):
        for g in NAMELIST_ORDER:
            if key in self.nml[g]:
                return self.nml[g][key]
        raise KeyError(key)

    def set(self, group, **kw):
        for k, v in kw.items():
            if k not in self.nml[group]:
                raise KeyError(f"{k} is not in namelist &{group}")
            cur = self.nml[group][k]
            if isinstance(cur, list) and not isinstance(v, list):
                cur = list(cur)
                cur[0] = v
                v = cur
            elif isinstance(cur, list):
                full = list(cur)
                full[: len(v)] = v
                v = full
            self.nml[group][k] = v
        return self

    @property
    def is3d(self):
        return str(self["job_type"]).upper().strip() == "3D"

    # ---- parsing ---------------------------------------------------------
    @classmethod
    def parse(cls, text):
        d = cls()
        lines = text.splitlines()
        pos = 0
        body = []
        # namelists
        for group in NAMELIST_ORDER:
            while pos < len(lines) and not lines[pos].strip().lower().startswith("&" + group):
                pos += 1
            if pos >= len(lines):
                raise ValueError(f"namelist &{group} not found")
            pos += 1
            body = []
            while pos < len(lines) and not lines[pos].strip().startswith("/"):
                body.append(lines[pos].split("!")[0])
                pos += 1
            pos += 1
            d._assign(group, " ".join(body))
        rest = [ln.strip() for ln in lines[pos:]]
        d._cards(rest)
        return d

    def _assign(self, group, body):
        parts = re.split(r"([A-Za-z_][A-Za-z0-9_]*(?:\(\s*\d+\s*\))?)\s*=", body)
        it = iter(parts[1:])
        for name, val in zip(it, it):
            m = re.fullmatch(r"([A-Za-z_][A-Za-z0-9_]*)(?:\(\s*(\d+)\s*\))?", name.strip())
            key, index = m.group(1), m.group(2)
            vals = _split_values(val)
            g = self.nml[group]
            lk = {k.lower(): k for k in g}
            if key.lower() not in lk:
                continue  # variables of the reference this engine does not read
            k = lk[key.lower()]
            if isinstance(g[k], list):
                arr = list(g[k])
                start = int(index) - 1 if index else 0
                for q, v in enumerate(vals):
                    arr[start + q] = float(v) if isinstance(v, (int, float)) and not isinstance(v, bool) else v
                g[k] = arr
            else:
                v = vals[0] if vals else None
                if isinstance(g[k], float) and isinstance(v, int) and not isinstance(v, bool):
                    v = float(v)
                g[k] = v

    def _cards(self, lines):
        """The MESH and FIXED_FLOWS cards (input.f:786-890), read as the
        reference's list-directed READs do: every READ starts at a new
        record (line), takes values separated by commas or blanks (r*v
        repeats, '/' ends the READ), continues on the next records when the
        current one runs out and drops the rest of its last record."""
        nx, ny, nz = self["nx"], self["ny"], self["nz"]
        rd = _ListReader(lines)
        # MESH card: READ(iunit,*) card until TRIM(card) == 'MESH'
        if not rd.find_card("MESH"):
            raise ValueError("MESH card not found")
        if self["iuni"] == 0 and self["grigen"] == 0:
            self.delta_x = np.array(rd.read(nx), dtype=float)
            if self.is3d:
                self.delta_y = np.array(rd.read(ny), dtype=float)
            self.delta_z = np.array(rd.read(nz), dtype=float)
        if not rd.find_card("FIXED_FLOWS"):
            raise ValueError("FIXED_FLOWS card not found")
        nb = int(rd.read(1)[0])
        ns = self["nsolid"]
        for _ in range(nb):
            if self.is3d:
                typ, x0, x1, y0, y1, z0, z1 = (int(v) for v in rd.read(7))
            else:
                typ, x0, x1, z0, z1 = (int(v) for v in rd.read(5))
                y0 = y1 = 0
            blk = dict(typ=typ, xlo=x0, xhi=x1, ylo=y0, yhi=y1, zlo=z0, zhi=z1)
            if typ in (1, 5, 8):
                if self.is3d:
                    ugv, vgv, wgv, pv, epv, tgv = rd.read(6)
                else:
                    ugv, wgv, pv, epv, tgv = rd.read(5)
                    vgv = 0.0
                per = 5 if self.is3d else 4
                sv_all = rd.read(per * ns)
                sol = []
                for q in range(ns):
                    sv = sv_all[q * per:(q + 1) * per]
                    if self.is3d:
                        sol.append(dict(u=sv[0], v=sv[1], w=sv[2], eps=sv[3], t=sv[4]))
                    else:
                        sol.append(dict(u=sv[0], v=0.0, w=sv[1], eps=sv[2], t=sv[3]))
                conc = rd.read(MAX_NGAS)
                blk.update(ug=ugv, vg=vgv, wg=wgv, p=pv, ep=epv, tg=tgv, solids=sol, ygc=conc)
            self.blocks.append(blk)

    # ---- writing ---------------------------------------------------------
    def to_text(self):
        out = []

        def fmt(v):
            if isinstance(v, bool):
                return ".TRUE." if v else ".FALSE."
            if isinstance(v, str):
                return f"'{v}'"
            if isinstance(v, int):
                return str(v)
            return repr(float(v)).replace("e", "D") if "e" in repr(float(v)) else repr(float(v)) + "D0"

        for g in NAMELIST_ORDER:
            out.append(f" &{g}")
            for k, v in self.nml[g].items():
                if isinstance(v, list):
                    out.append(f"  {k} = " + ", ".join(fmt(x) for x in v) + ",")
                else:
                    out.append(f"  {k} = {fmt(v)},")
            out.append(" /")
        out.append("MESH")
        if self["iuni"] == 0 and self["grigen"] == 0:
            out.append(" ".join(repr(float(x)) for x in self.delta_x))
            if self.is3d:
                out.append(" ".join(repr(float(x)) for x in self.delta_y))
            out.append(" ".join(repr(float(x)) for x in self.delta_z))
        out.append("FIXED_FLOWS")
        out.append(str(len(self.blocks)))
        for b in self.blocks:
            if self.is3d:
                out.append(f"{b['typ']} {b['xlo']} {b['xhi']} {b['ylo']} {b['yhi']} {b['zlo']} {b['zhi']}")
            else:
                out.append(f"{b['typ']} {b['xlo']} {b['xhi']} {b['zlo']} {b['zhi']}")
            if b["typ"] in (1, 5, 8):
                if self.is3d:
                    out.append(" ".join(repr(float(b[k])) for k in ("ug", "vg", "wg", "p", "ep", "tg")))
                    out.append(" ".join(repr(float(s[k])) for s in b["solids"] for k in ("u", "v", "w", "eps", "t")))
                else:
                    out.append(" ".join(repr(float(b[k])) for k in ("ug", "wg", "p", "ep", "tg")))
                    out.append(" ".join(repr(float(s[k])) for s in b["solids"] for k in ("u", "w", "eps", "t")))
                out.append(" ".join(repr(float(x)) for x in b["ygc"]))
        return "\n".join(out) + "\n"

    # ---- derived quantities (check_input / initc) ---------------------------
    def atm_ygc(self):
        return [float(self[f"atm_{g}"]) for g in GAS_NAMES]

    def vent_ygc(self):
        if self["ivent"] >= 1:
            return [float(self[f"vent_{g}"]) for g in GAS_NAMES]
        return [0.0] * MAX_NGAS

    def gas_types(self):
        """gas_check, setup.f:621-669: present species in reference order."""
        present = []
        for igg in range(MAX_NGAS):
            on = self.atm_ygc()[igg] != 0.0
            if self["ivent"] > 0 and self.vent_ygc()[igg] != 0.0:
                on = True
            for b in self.blocks:
                if "ygc" in b and b["ygc"][igg] != 0.0:
                    on = True
            if on:
                present.append(igg + 1)
        if len(present) != self["ngas"]:
            raise ValueError(f"wrong number of gas species: {len(present)} present, ngas={self['ngas']}")
        return present

    def check(self):
        """Options of the reference that this engine does not implement."""
        bad = []
        if self["iturb"] not in (0, 1, 2):
            bad.append("iturb other than 0, 1 or 2")
        if self["iturb"] >= 1 and self["modturbo"] not in (1, 2):
            bad.append("modturbo other than 1 or 2")
        if self["iss"] not in (0, 1):
            bad.append("iss>1")
        if self["ctu"] != 0:
            bad.append("ctu>0 (corner transport upwind)")
        if self["implicit_fluxes"] and self["alpha"] != 1.0:
            # the previous-visit interphase terms of alpha < 1 are not
            # defined when tilde runs inside the sweeps
            bad.append("implicit_fluxes with alpha other than 1")
        if self["time_integration"] not in (0, 1):
            bad.append("time_integration other than 0 or 1")
        elif self["time_integration"] == 1 and self["pmodel"] not in (1, 2):
            # compute_rhs (explicit_solver.f:632-642) defines the face volume
            # fractions only for pmodel 1 and 2
            bad.append("time_integration=1 with pmodel other than 1 or 2")
        if self["irex"] > 1:
            bad.append("irex>1 (reactions)")
        if self["itp"] not in (0, 1):
            bad.append("itp other than 0 or 1")
        elif self["itp"] == 1:
            if self["grigen"] != 0:
                bad.append("topography (itp=1) on a generated mesh (grigen>0)")
            if self.is3d and self["iavv"] != 0:
                bad.append("iavv>0 (average_dem)")
            if self.is3d and self["ismt"] != 1 and self["filtersize"] >= self["cellsize"]:
                bad.append("ismt=2, 3 (gaussian and barnes DEM filters)")
            if self["immb"] not in (0, 1):
                bad.append("immb other than 0 or 1")
            elif self["immb"] == 1 and self["time_integration"] == 1:
                bad.append("immersed boundaries with the explicit solver (time_integration=1)")
        if self["isink"] < 0:
            bad.append("isink<0")
        if self["idome"] != 0:
            bad.append("idome>0")
        if self["ibl"] != 0:
            bad.append("ibl>0")
        if self["ipro"] != 0 or self["iali"] not in (0, 1, 2, 3, 4):
            bad.append("ipro>0 or iali=5")
        if self["optimization"] not in (1, 2, 3):
            bad.append("optimization other than 1, 2 or 3")
        elif self["optimization"] == 3 and self.is3d and self["nsolid"] == 2:
            # opt3_inner_loop, the matrix-precomputing variant of 3D with two classes
            bad.append("optimization=3 in 3D with two particle classes")
        return bad
