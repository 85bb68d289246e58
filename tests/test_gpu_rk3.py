"""Parity of the CUDA explicit SSP-RK3 solver (time_integration = 1,
explicit_solver.f) with the CPU FP64 oracle, call by call and over whole
steps, in 2D and 3D.

Tolerances (relative L-infinity against each field's scale):
  * initialize_fieldn (n-level copies, viscosity, heat exchange, interphase
    matrix, stresses): 1e-12 -- the only differences are last-ulp
    differences of pow/exp/sqrt between the CUDA and glibc math libraries;
  * explicit_iter and whole steps: 1e-9, the bound for FP64 fields.
Particle temperature and enthalpy are compared where the class is present
(rlk > 1e-5), as in the semi-implicit tests.
"""
import numpy as np
import pytest

from helpers import STEP_FIELDS, compare_state, rel_linf

pytestmark = pytest.mark.gpu

TOL_EXPLICIT = 1e-12
TOL_STEP = 1e-9
FIELDS_3D = STEP_FIELDS + ("vg", "vs")


def _pair(builder, **kw):
    from pdac_b200.setup_state import Case
    from pdac_b200.engine import Engine
    import pyoracle
    deck = builder(**kw)
    deck.set("numeric", time_integration=1)
    case = Case(deck)
    return case, Engine(case), pyoracle.Oracle(case)


def _state_check(eng, ora, names, tol, where):
    case = eng.case
    fluid = (case.flag & 1) == 1
    got = {n: eng.get(n) for n in set(names) | {"rlk"}}
    ref = {n: ora.get(n) for n in set(names) | {"rlk"}}
    errs, bad = compare_state(got, ref, names, tol, case.nsolid, case.ncell, cells=fluid)
    assert not bad, f"{where}: {bad}"


def _array_check(eng, ora, names, tol, where):
    bad = {}
    for n in names:
        e = rel_linf(eng.get(n), ora.get(n))
        if not e <= tol:
            bad[n] = e
    assert not bad, f"{where}: {bad}"


def _vis_check(eng, ora, d3, tol, where):
    """The engine keeps the viscous terms in one array, block (phase * 3 +
    axis); the oracle in gvisx/y/z and pvisx/y/z."""
    case = eng.case
    n, ns = case.ncell, case.nsolid
    vis = eng.get("vis").reshape(ns + 1, 3, n)
    axes = (0, 1, 2) if d3 else (0, 2)
    for ax in axes:
        name = "xyz"[ax]
        g = ora.get("gvis" + name)
        p = ora.get("pvis" + name).reshape(ns, n)
        e = max([rel_linf(vis[0, ax], g)] + [rel_linf(vis[1 + s, ax], p[s]) for s in range(ns)])
        assert e <= tol, f"{where}: vis {name} {e}"


def _run_calls(case, eng, ora, d3, steps):
    fields = FIELDS_3D if d3 else STEP_FIELDS
    dt = case.deck["dt"]
    fieldn_arrays = ["pn", "epn", "rgpn", "siegn", "rlkn", "siesn", "rgpgcn", "ugn", "wgn", "usn", "wsn",
                     "mug", "kapg", "appu", "appw", "hv"]
    if d3:
        fieldn_arrays += ["vgn", "vsn", "appv"]
    for sweep in range(1, steps + 1):
        eng.boundary(sweep); ora.boundary(sweep)
        _state_check(eng, ora, fields, TOL_EXPLICIT, f"boundary {sweep}")
        eng.initialize_fieldn(); ora.initialize_fieldn()
        _array_check(eng, ora, fieldn_arrays, TOL_EXPLICIT, f"initialize_fieldn {sweep}")
        _vis_check(eng, ora, d3, TOL_EXPLICIT, f"initialize_fieldn {sweep}")
        eng.explicit_iter(dt); ora.explicit_iter(dt)
        _state_check(eng, ora, fields, TOL_STEP, f"explicit_iter {sweep}")
        eng.ygas(dt); ora.ygas(dt)
        _state_check(eng, ora, ("ygc", "xgc"), TOL_STEP, f"ygas {sweep}")


def test_calls_rk3_2d():
    from pdac_b200 import configs
    case, eng, ora = _pair(configs.small_2d)
    _run_calls(case, eng, ora, False, 3)


def test_calls_rk3_3d():
    from pdac_b200 import configs
    case, eng, ora = _pair(configs.small_3d, dt=0.001)
    _run_calls(case, eng, ora, True, 3)


@pytest.mark.parametrize("d3", [False, True])
def test_steps_rk3(d3):
    """Ten whole steps through pdac_gpu_step; fields compared every step."""
    from pdac_b200 import configs
    if d3:
        case, eng, ora = _pair(configs.small_3d, nx=16, ny=14, nz=18, dt=0.001, vent_cells=4)
    else:
        case, eng, ora = _pair(configs.plume_2d, nx=48, nz=64, dt=0.005)
    fields = FIELDS_3D if d3 else STEP_FIELDS
    for s in range(1, 11):
        assert eng.step(s) == 0
        ora.step(s)
        _state_check(eng, ora, fields, TOL_STEP, f"step {s}")


def test_rk3_rejected_on_semi_implicit_context():
    """initialize_fieldn / explicit_iter on a time_integration = 0 context
    return PDAC_ERR_CONFIG and leave the context usable."""
    from pdac_b200 import configs
    from pdac_b200.setup_state import Case
    from pdac_b200.engine import Engine, PdacError
    case = Case(configs.small_2d())
    eng = Engine(case)
    with pytest.raises(PdacError):
        eng.initialize_fieldn()
    with pytest.raises(PdacError):
        eng.explicit_iter(case.deck["dt"])
    eng.step(1)
    assert np.all(np.isfinite(eng.get("p")))
