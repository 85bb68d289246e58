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


def plume_3d(nx=256, ny=256, nz=192, dxyz=20.0, dt=0.02, vent_cells=5, w_gas=150.0, t_gas=1000.0,
             diameters=(30.0, 250.0, 1000.0), density=2400.0, ep_solid=(0.005, 0.01, 0.005), muscl=1,
             limiter=2, delg=1.0e-8, maxout=500):
    """3D Cartesian plume over flat ground on a uniform grid.

    Defaults are the 256 x 256 x 192, 20 m, three-class, 300-step workload: the
    same stratified air atmosphere, a square vent of 5 x 5 cells at the domain
    centre (a FIXED_FLOWS inlet block in the ground row) injecting water vapour
    at 1000 K and 150 m/s with classes of 30, 250 and 1000 um (2400 kg/m3) at
    volume fractions 0.005, 0.01 and 0.005.  Lateral and top boundaries are
    free in/outflow, the ground is a no-slip wall.
    """
    d = Deck()
    ns = len(diameters)
    d.set("control", job_type="3D", dt=dt, tstop=1.0e9)
    d.set("model", iturb=0, ngas=2, gravz=-9.81, pmodel=2, drag_model=1)
    d.set("mesh", nx=nx, ny=ny, nz=nz, itc=0, iuni=1, dx0=dxyz, dy0=dxyz, dz0=dxyz, grigen=0)
    d.set("boundaries", west=4, east=4, south=4, north=4, bottom=3, top=4)
    d.set("atmosphere", stratification=True, t_ground=288.0, troposphere_grad=-6.5e-3,
          p_ground=1.01325e5, atm_Air=1.0)
    d.set("particles", nsolid=ns, diameter=list(diameters), density=[density] * ns)
    d.set("numeric", muscl=muscl, vel_limiter=limiter, mass_limiter=limiter, delg=delg, maxout=maxout)
    lo_i = nx // 2 - vent_cells // 2 + 1
    lo_j = ny // 2 - vent_cells // 2 + 1
    d.blocks = [dict(typ=5, xlo=lo_i, xhi=lo_i + vent_cells - 1, ylo=lo_j, yhi=lo_j + vent_cells - 1, zlo=1, zhi=1,
                     ug=0.0, vg=0.0, wg=w_gas, p=1.01325e5, ep=1.0 - sum(ep_solid), tg=t_gas,
                     solids=[dict(u=0.0, v=0.0, w=w_gas, eps=e, t=t_gas) for e in ep_solid],
                     ygc=[0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0])]
    return d


def small_3d(nx=10, ny=9, nz=12, **kw):
    """A tiny version of the 3D plume for parity tests (2 x 2 vent)."""
    kw.setdefault("vent_cells", 2)
    return plume_3d(nx=nx, ny=ny, nz=nz, **kw)


WORKLOADS = {
    "plume2d_128x192": dict(builder="plume_2d", kw={}, steps=500),
    "plume3d_256x256x192": dict(builder="plume_3d", kw={}, steps=300),
}


def _explicit(deck):
    deck.set("numeric", time_integration=1)
    return deck


def plume_2d_rk3(**kw):
    """The 2D plume advanced by the explicit SSP-RK3 solver (time_integration
    = 1, explicit_solver.f) at dt = 5 ms.  At the semi-implicit deck's 10 ms
    the explicit stages drive a cell near the vent out of the range where
    the caloric equation of state converges after about 20 steps (the
    oracle counts one failure at step 21), and from there on the state
    depends on round-off."""
    kw.setdefault("dt", 0.005)
    return _explicit(plume_2d(**kw))


def plume_3d_rk3(**kw):
    """The 3D plume advanced by the explicit SSP-RK3 solver.  Its explicit
    stages need dt = 1 ms on this grid (the 20 ms of the semi-implicit deck
    does not keep the dilute particle phases stable), so that is the
    default."""
    kw.setdefault("dt", 0.001)
    return _explicit(plume_3d(**kw))


def small_2d_rk3(**kw):
    """small_2d with the explicit SSP-RK3 solver."""
    return _explicit(small_2d(**kw))


def small_3d_rk3(**kw):
    """small_3d with the explicit SSP-RK3 solver at dt = 1 ms."""
    kw.setdefault("dt", 0.001)
    return _explicit(small_3d(**kw))


def _les(deck):
    deck.set("model", iturb=1, modturbo=1, iss=1)
    return deck


def small_2d_les(**kw):
    """small_2d with the Smagorinsky sub-grid model (iturb = 1, the
    reference's default) and the particle sub-grid stress (iss = 1)."""
    return _les(small_2d(**kw))


def small_3d_les(**kw):
    """small_3d with the sub-grid models of small_2d_les."""
    return _les(small_3d(**kw))


def small_2d_rk3_les(**kw):
    """small_2d_rk3 with the sub-grid models of small_2d_les."""
    return _les(small_2d_rk3(**kw))


def _dynamic(deck):
    deck.set("model", iturb=1, modturbo=2, iss=1)
    return deck


def small_3d_dyn(**kw):
    """small_3d with the dynamic Smagorinsky model (modturbo = 2, turbo.f:180-349)
    and the particle sub-grid stress."""
    return _dynamic(small_3d(**kw))


def small_3d_rk3_dyn(**kw):
    """small_3d_rk3 with the sub-grid models of small_3d_dyn."""
    return _dynamic(small_3d_rk3(**kw))


def small_2d_sink(**kw):
    """small_2d with the ground sink (isink = 1) on the ring 10 m < r < 60 m
    around the axis."""
    d = small_2d(**kw)
    d.set("model", isink=1, rprox=10.0, rdist=60.0)
    return d


def small_3d_sink(**kw):
    """small_3d with the ground sink on the ring 20 m < r < 70 m around the
    domain centre (100 m, 80 m)."""
    d = small_3d(**kw)
    d.set("model", isink=1, rprox=20.0, rdist=70.0)
    d.set("mesh", center_x=100.0, center_y=80.0)
    return d


def _implicit(deck, fluxes, enthalpy):
    deck.set("numeric", implicit_fluxes=fluxes, implicit_enthalpy=enthalpy)
    return deck


def small_2d_implicit(fluxes=True, enthalpy=True, **kw):
    """small_2d with tilde (implicit_fluxes) and / or ftem (implicit_enthalpy)
    inside the outer sweeps of iter (iter.f:211-226, 362-379)."""
    return _implicit(small_2d(**kw), fluxes, enthalpy)


def small_3d_implicit(fluxes=True, enthalpy=True, **kw):
    """small_3d with the implicit modes of small_2d_implicit."""
    return _implicit(small_3d(**kw), fluxes, enthalpy)


def small_2d_mixture(formatted=False, **kw):
    """small_2d with the mixture fields (compute_mixture) and, optionally,
    text output files (formatted_output)."""
    d = small_2d(**kw)
    d.set("model", compute_mixture=True)
    d.set("control", formatted_output=formatted)
    return d


def small_3d_mixture(formatted=False, **kw):
    """small_3d with the options of small_2d_mixture."""
    d = small_3d(**kw)
    d.set("model", compute_mixture=True)
    d.set("control", formatted_output=formatted)
    return d


def small_2d_opt(optimization=2, **kw):
    """small_2d with the reference's optimized inner loop (optimization = 2,
    opt_inner_loop, iter.f:1255-1547) and a no-slip east wall.  The loop's
    density stencils keep the loop-entry value in slots remapped to the cell
    itself, which only the MUSCL corrections of fluid cells next to a wall
    read; the rows above the ground are boundary-layer cells with
    first-order fluxes, so the side wall is where the variant shows."""
    d = small_2d(**kw)
    d.set("numeric", optimization=optimization)
    d.set("boundaries", east=3)
    return d


def small_3d_opt(optimization=2, **kw):
    """small_3d with the optimized inner loop of small_2d_opt and no-slip
    walls on the x sides."""
    d = small_3d(**kw)
    d.set("numeric", optimization=optimization)
    d.set("boundaries", west=3, east=3)
    return d


# ---- topography and immersed boundaries ------------------------------------
def write_hill_profile(path, x_end, x_hill, height, sigma, dx=5.0):
    """A 2D topographic profile (topo.f:306-348 layout): one Gaussian hill
    of the given height and width centred at x_hill on flat ground at 0,
    sampled every dx from -dx to x_end + dx."""
    import numpy as np

    from .topography import write_profile
    xs = np.arange(-dx, x_end + 2 * dx, dx)
    zs = height * np.exp(-0.5 * ((xs - x_hill) / sigma) ** 2)
    write_profile(path, xs, zs)
    return path


def write_hills_dem(path, nx, ny, dxy, n_hills=8, seed=0, h_range=(100.0, 600.0), s_range=(300.0, 1200.0),
                    vent_xy=None, vent_flat=0.0, dem_cell=None, margin=3):
    """A seeded ASCII DEM (the layout read_dem_ascii reads) that is the sum
    of n_hills Gaussian hills with heights drawn from h_range and widths
    from s_range, centred at uniformly drawn points of the nx x ny mesh of
    spacing dxy (mesh coordinates: cell centres at (i - 1.5) dxy).  With
    vent_flat > 0 the ground is flat (at 0) within that radius of vent_xy
    and rises to the full hills at twice the radius (the flattened crater
    floor the vent sits on).  The DEM covers
    the mesh with `margin` DEM cells to spare on every side."""
    import numpy as np

    from .topography import write_dem_ascii
    rng = np.random.default_rng(seed)
    dem_cell = dem_cell or dxy
    lx, ly = nx * dxy, ny * dxy
    x0, y0 = -dxy - margin * dem_cell, -dxy - margin * dem_cell
    nxd = int(np.ceil((lx + 2 * dxy + 2 * margin * dem_cell) / dem_cell)) + 1
    nyd = int(np.ceil((ly + 2 * dxy + 2 * margin * dem_cell) / dem_cell)) + 1
    xs = x0 + dem_cell * np.arange(nxd)
    ys = y0 + dem_cell * np.arange(nyd)
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    Z = np.zeros_like(X)
    for _ in range(n_hills):
        h = rng.uniform(*h_range)
        s = rng.uniform(*s_range)
        cx, cy = rng.uniform(0.0, lx), rng.uniform(0.0, ly)
        Z += h * np.exp(-0.5 * ((X - cx) ** 2 + (Y - cy) ** 2) / s ** 2)
    if vent_flat > 0.0 and vent_xy is not None:
        # a crater floor at ground level within vent_flat of the vent, rising
        # smoothly to the full hills at twice that distance
        r = np.sqrt((X - vent_xy[0]) ** 2 + (Y - vent_xy[1]) ** 2)
        t = np.clip((r - vent_flat) / vent_flat, 0.0, 1.0)
        Z *= t * t * (3.0 - 2.0 * t)
    write_dem_ascii(path, x0, y0, dem_cell, Z)
    return path


def plume_2d_topo(dem_file, immb=1, nx=128, nz=192, **kw):
    """The 2D plume over a topographic profile read from dem_file (itp = 1),
    with immersed boundaries (immb = 1, the default) or the staircase of
    no-slip cells (immb = 0)."""
    d = plume_2d(nx=nx, nz=nz, **kw)
    d.set("topography", itp=1, dem_file=str(dem_file))
    d.set("boundaries", immb=immb)
    return d


def small_2d_topo(tmpdir, immb=1, nx=24, nz=24, height=60.0, **kw):
    """A 24 x 24 (10 m) 2D plume with a 60 m Gaussian hill 150 m from the
    axis, the profile written under tmpdir."""
    import os
    kw.setdefault("vent_radius", 20.0)
    path = write_hill_profile(os.path.join(str(tmpdir), "hill.dat"), x_end=nx * 10.0, x_hill=150.0,
                              height=height, sigma=40.0)
    return plume_2d_topo(path, immb=immb, nx=nx, nz=nz, **kw)


def plume_3d_topo(dem_file, immb=1, nx=384, ny=384, nz=256, dxyz=15.0, dt=0.01, w_gas=120.0, t_gas=1100.0,
                  diameters=None, ep_total=0.03, density=2500.0, **kw):
    """The large 3D workload over synthetic topography: the DEM in dem_file
    (write_hills_dem), immersed boundaries, five classes from 20 to 2000 um
    (log-spaced, 2500 kg/m3) sharing a total volume fraction of 0.03, and
    the vent (5 x 5 cells at the centre) at 1100 K and 120 m/s."""
    import numpy as np
    if diameters is None:
        diameters = tuple(float(v) for v in np.geomspace(20.0, 2000.0, 5))
    ns = len(diameters)
    d = plume_3d(nx=nx, ny=ny, nz=nz, dxyz=dxyz, dt=dt, w_gas=w_gas, t_gas=t_gas, diameters=diameters,
                 density=density, ep_solid=tuple([ep_total / ns] * ns), **kw)
    # the DEM is resampled at the mesh spacing; the hills are smooth, so the
    # low-pass filter of resize_dem is off (filtersize < cellsize): it would
    # also raise the crater floor around the vent
    d.set("topography", itp=1, dem_file=str(dem_file), cellsize=dxyz, filtersize=0.5 * dxyz)
    d.set("boundaries", immb=immb)
    # the DEM is given in mesh coordinates (cell centres at (i - 1.5) dxyz):
    # compute_UTM_coords (topo.f:731-751) then leaves the mesh where it is
    d.set("mesh", center_x=(nx // 2 - 1.5) * dxyz, center_y=(ny // 2 - 1.5) * dxyz)
    return d


def _vent_centre(n, cells, d):
    """Mesh coordinate of the centre of the vent block of plume_3d (cells
    nx // 2 - cells // 2 + 1 .. + cells - 1 along an axis of n cells)."""
    lo = n // 2 - cells // 2 + 1
    return (lo + 0.5 * (cells - 1) - 1.5) * d


def small_3d_topo(tmpdir, immb=1, nx=16, ny=14, nz=14, dxyz=20.0, seed=3, **kw):
    """A 16 x 14 x 14 (20 m) 3D plume over three seeded hills of 40-100 m
    with a flat crater floor around the 2 x 2 vent."""
    import os
    kw.setdefault("vent_cells", 2)
    cx = _vent_centre(nx, kw["vent_cells"], dxyz)
    cy = _vent_centre(ny, kw["vent_cells"], dxyz)
    path = write_hills_dem(os.path.join(str(tmpdir), "hills.asc"), nx, ny, dxyz, n_hills=3, seed=seed,
                           h_range=(40.0, 100.0), s_range=(40.0, 90.0), vent_xy=(cx, cy), vent_flat=3 * dxyz)
    d = plume_3d(nx=nx, ny=ny, nz=nz, dxyz=dxyz, **kw)
    d.set("topography", itp=1, dem_file=path, cellsize=dxyz / 2, filtersize=dxyz / 4)
    d.set("boundaries", immb=immb)
    d.set("mesh", center_x=(nx // 2 - 1.5) * dxyz, center_y=(ny // 2 - 1.5) * dxyz)
    return d


def plume_3d_hills(nx=384, ny=384, nz=256, dxyz=15.0, seed=0, immb=1, dem_dir=None, **kw):
    """The large 3D workload with its synthetic topography written out: the
    sum of 8 seeded Gaussian hills (heights 100-600 m, widths 300-1200 m on
    the 384-cell mesh, both scaled with nx / 384 on smaller meshes so that a
    reduced case keeps the shape of the terrain) with a flat crater floor of
    four cells' radius around the vent, as an ASCII DEM under dem_dir
    (default: the system temporary directory), read back through the
    topography path (itp = 1) with immersed boundaries."""
    import os
    import tempfile
    dem_dir = dem_dir or os.path.join(tempfile.gettempdir(), "pdac_b200_dem")
    os.makedirs(dem_dir, exist_ok=True)
    cx = _vent_centre(nx, 5, dxyz)
    cy = _vent_centre(ny, 5, dxyz)
    path = os.path.join(dem_dir, f"hills_{nx}x{ny}_{dxyz:g}m_seed{seed}_v2.asc")
    sc = nx / 384.0
    if not os.path.exists(path):
        write_hills_dem(path, nx, ny, dxyz, n_hills=8, seed=seed, h_range=(100.0 * sc, 600.0 * sc),
                        s_range=(300.0 * sc, 1200.0 * sc), vent_xy=(cx, cy), vent_flat=4 * dxyz)
    return plume_3d_topo(path, immb=immb, nx=nx, ny=ny, nz=nz, dxyz=dxyz, **kw)
