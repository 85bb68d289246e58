"""Synthetic input decks for the benchmark and test workloads.

Each builder returns a :class:`~pdac_b200.deck.Deck` with the reference's
namelist defaults overridden as the workload states.  No public dataset is
involved; all inputs are generated here.
"""
from __future__ import annotations

from .deck import Deck


def plume_2d(nx=128, nz=192, dxz=10.0, dt=0.01, vent_radius=50.0, w_gas=100.0, t_gas=1100.0,
             diameters=(50.0, 500.0), density=2500.0, ep_solid=(0.01, 0.01), muscl=1,
             limiter=2, irand=1, delg=1.0e-8, maxout=500, iali=0):
    """2D cylindrical (r, z) volcanic plume on a uniform staggered grid.

    Defaults are the 128 x 192, 10 m, two-class, 500-step workload: air
    atmosphere hydrostatic from 288 K with a 6.5 K/km lapse rate, axis vent of
    radius 50 m injecting water vapour at 1100 K and 100 m/s, classes of 50 and
    500 um (2500 kg/m3) at volume fraction 0.01 each, second-order MUSCL.
    """
    d = Deck()
    ns = len(diameters)
    d.set("control", job_type="2D", dt=dt, tstop=1.0e9)
    d.set("model", iturb=0, ngas=2, gravz=-9.81, pmodel=2, drag_model=1)
    d.set("mesh", nx=nx, nz=nz, ny=1, itc=1, iuni=1, dx0=dxz, dz0=dxz, grigen=0)
    d.set("boundaries", west=2, east=4, bottom=3, top=4)
    d.set("atmosphere", stratification=True, t_ground=288.0, troposphere_grad=-6.5e-3,
          p_ground=1.01325e5, atm_Air=1.0)
    d.set("inlet", ivent=1, iali=iali, irand=irand, vent_radius=vent_radius, w_gas=w_gas, t_gas=t_gas,
          vent_H2O=1.0, ep_solid=list(ep_solid), w_solid=[w_gas] * ns, t_solid=[t_gas] * ns)
    d.set("particles", nsolid=ns, diameter=list(diameters), density=[density] * ns)
    d.set("numeric", muscl=muscl, vel_limiter=limiter, mass_limiter=limiter, delg=delg, maxout=maxout)
    d.delta_x = None
    d.delta_z = None
    return d


def small_2d(nx=12, nz=16, **kw):
    """A tiny version of the 2D plume for parity tests (vent radius 20 m)."""
    kw.setdefault("vent_radius", 20.0)
    return plume_2d(nx=nx, nz=nz, **kw)


WORKLOADS = {
    "plume2d_128x192": dict(builder="plume_2d", kw={}, steps=500),
}
