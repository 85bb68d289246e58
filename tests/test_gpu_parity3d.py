"""Parity of the 3D CUDA path with the CPU FP64 oracle, phase by phase and
over whole steps.  Tolerances as for 2D (relative L-infinity against each
field's scale): 1e-12 for the explicit passes, 1e-9 after iter and for steps.
"""
import numpy as np
import pytest

from helpers import STEP_FIELDS, compare_state, frame_mismatches, rel_linf

pytestmark = pytest.mark.gpu

TOL_EXPLICIT = 1e-12
TOL_STEP = 1e-9
STEP_FIELDS3 = STEP_FIELDS + ("vg", "vs")


def _pair(deck_builder, **kw):
    from pdac_b200.setup_state import Case
    from pdac_b200.engine import Engine
    import pyoracle
    case = Case(deck_builder(**kw))
    return case, Engine(case), pyoracle.Oracle(case, order=pyoracle.ORDER_COLORED)


def _check(eng, ora, names, tol, where, alias=None):
    case = eng.case
    fluid = (case.flag & 1) == 1
    worst = {}
    for n in names:
        a = eng.get(n)
        b = ora.get((alias or {}).get(n, n))
        if n in STEP_FIELDS3:
            got, ref = {n: a, "rlk": eng.get("rlk")}, {n: b, "rlk": ora.get("rlk")}
            errs, _ = compare_state(got, ref, (n,), tol, case.nsolid, case.ncell, cells=fluid)
            worst[n] = errs[n]
        else:
            worst[n] = rel_linf(a, b)
    bad = {n: e for n, e in worst.items() if not e <= tol}
    assert not bad, f"{where}: {bad}"


def test_phases_small_3d():
    from pdac_b200 import configs
    case, eng, ora = _pair(configs.small_3d)
    dt = case.deck["dt"]
    for sweep in (1, 2, 3):
        eng.boundary(sweep); ora.boundary(sweep)
        _check(eng, ora, STEP_FIELDS3, TOL_EXPLICIT, f"boundary {sweep}")
        bad_frame, _ = frame_mismatches(eng.download(), ora.get_state(), STEP_FIELDS3, case, TOL_EXPLICIT)
        assert not bad_frame, f"boundary {sweep}: frame values differ: {bad_frame[:10]}"
        eng.fieldn(); ora.fieldn()
        _check(eng, ora, ("rugn", "rvgn", "rwgn", "rusn", "rvsn", "rwsn", "mug", "kapg", "rgpgcn"),
               TOL_EXPLICIT, "fieldn")
        eng.tilde(dt); ora.tilde(dt)
        _check(eng, ora, ("mf",), TOL_EXPLICIT, "tilde fluxes", alias={"mf": "mf3"})
        _check(eng, ora, ("rug", "rvg", "rwg", "rus", "rvs", "rws", "appu", "appv", "appw"), TOL_EXPLICIT, "tilde")
        n1 = eng.iter(dt); n2 = ora.iter(dt)
        assert n1 == n2, f"outer sweeps differ: gpu {n1} oracle {n2}"
        _check(eng, ora, STEP_FIELDS3, TOL_STEP, f"iter {sweep}")
        eng.ygas(dt); ora.ygas(dt)
        _check(eng, ora, ("ygc", "xgc"), TOL_STEP, "ygas")
        eng.htilde(dt); ora.htilde(dt)
        _check(eng, ora, ("rhg", "rhs"), TOL_STEP, "htilde")
        eng.ftem(dt); ora.ftem(dt)
        _check(eng, ora, STEP_FIELDS3, TOL_STEP, f"ftem {sweep}")


def test_steps_3d():
    """10 whole steps of a 24 x 20 x 28 version of the 3D plume."""
    from pdac_b200 import configs
    case, eng, ora = _pair(configs.small_3d, nx=24, ny=20, nz=28, vent_cells=4)
    fluid = (case.flag & 1) == 1
    for s in range(1, 11):
        n1 = eng.step(s)
        n2 = ora.step(s)
        got = eng.download()
        ref = ora.get_state()
        errs, bad = compare_state(got, ref, STEP_FIELDS3, TOL_STEP, case.nsolid, case.ncell, cells=fluid)
        assert n1 == n2, f"step {s}: outer sweeps gpu {n1} oracle {n2}"
        assert not bad, f"step {s} (nit {n1}): {bad}"
        bad_frame, _ = frame_mismatches(got, ref, STEP_FIELDS3, case, TOL_STEP)
        assert not bad_frame, f"step {s}: frame values differ: {bad_frame[:10]}"
