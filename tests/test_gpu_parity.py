"""Parity of the CUDA engine with the CPU FP64 oracle, phase by phase.

Both run the same deck from the same initial state; the oracle runs the
corrector in the engine's colour order.  Tolerances (relative L-infinity
against each field's scale):
  * explicit phases (boundary, fieldn, tilde, ygas, htilde, ftem): 1e-12;
    the only differences are last-ulp differences of pow/exp/sqrt between
    the CUDA and glibc math libraries;
  * iter and whole steps: 1e-9, the per-step bound for FP64 fields.
"""
import numpy as np
import pytest

from helpers import STEP_FIELDS, compare_state, frame_mismatches, rel_linf

pytestmark = pytest.mark.gpu

TOL_EXPLICIT = 1e-12
TOL_STEP = 1e-9


def _pair(deck_builder, **kw):
    from pdac_b200.setup_state import Case
    from pdac_b200.engine import Engine
    import pyoracle
    case = Case(deck_builder(**kw))
    return case, Engine(case), pyoracle.Oracle(case, order=pyoracle.ORDER_COLORED)


@pytest.fixture(scope="module")
def small():
    from pdac_b200 import configs
    return _pair(configs.small_2d, nx=12, nz=16)


def _check_arrays(eng, ora, names, tol, where):
    case = eng.case
    fluid = (case.flag & 1) == 1
    worst = {}
    for n in names:
        a, b = eng.get(n), ora.get(n)
        if n in STEP_FIELDS:
            got, ref = {n: a, "rlk": eng.get("rlk")}, {n: b, "rlk": ora.get("rlk")}
            errs, _ = compare_state(got, ref, (n,), tol, case.nsolid, case.ncell, cells=fluid)
            worst[n] = errs[n]
            continue
        e = rel_linf(a, b)
        worst[n] = e
    bad = {n: e for n, e in worst.items() if not e <= tol}
    assert not bad, f"{where}: {bad}"


def test_phases_small_2d(small):
    case, eng, ora = small
    dt = case.deck["dt"]
    for sweep in (1, 2, 3):
        eng.boundary(sweep); ora.boundary(sweep)
        _check_arrays(eng, ora, STEP_FIELDS, TOL_EXPLICIT, f"boundary {sweep}")
        bad_frame, _ = frame_mismatches(eng.download(), ora.get_state(), STEP_FIELDS, case, TOL_EXPLICIT)
        assert not bad_frame, f"boundary {sweep}: frame values differ: {bad_frame[:10]}"
        eng.fieldn(); ora.fieldn()
        _check_arrays(eng, ora, ("rugn", "rwgn", "rusn", "rwsn", "mug", "kapg", "rgpgcn"), TOL_EXPLICIT, "fieldn")
        eng.tilde(dt); ora.tilde(dt)
        _check_arrays(eng, ora, ("ugfe", "ugft", "wgfe", "wgft", "usfe", "usft", "wsfe", "wsft"), TOL_EXPLICIT, "tilde fluxes")
        _check_arrays(eng, ora, ("rug", "rwg", "rus", "rws", "appu", "appw"), TOL_EXPLICIT, "tilde")
        n1 = eng.iter(dt); n2 = ora.iter(dt)
        assert n1 == n2, f"outer sweeps differ: gpu {n1} oracle {n2}"
        _check_arrays(eng, ora, STEP_FIELDS, TOL_STEP, f"iter {sweep}")
        eng.ygas(dt); ora.ygas(dt)
        _check_arrays(eng, ora, ("ygc", "xgc"), TOL_STEP, "ygas")
        eng.htilde(dt); ora.htilde(dt)
        _check_arrays(eng, ora, ("rhg", "rhs"), TOL_STEP, "htilde")
        eng.ftem(dt); ora.ftem(dt)
        _check_arrays(eng, ora, STEP_FIELDS, TOL_STEP, f"ftem {sweep}")


def test_steps_full_2d():
    """20 whole steps of the 128 x 192 workload, fields compared every step."""
    from pdac_b200 import configs
    case, eng, ora = _pair(configs.plume_2d)
    for s in range(1, 21):
        n1 = eng.step(s)
        n2 = ora.step(s)
        got = eng.download()
        ref = ora.get_state()
        fluid = (case.flag & 1) == 1
        errs, bad = compare_state(got, ref, STEP_FIELDS, TOL_STEP, case.nsolid, case.ncell, cells=fluid)
        assert n1 == n2, f"step {s}: outer sweeps gpu {n1} oracle {n2}"
        assert not bad, f"step {s} (nit {n1}): {bad}"
        bad_frame, _ = frame_mismatches(got, ref, STEP_FIELDS, case, TOL_STEP)
        assert not bad_frame, f"step {s}: frame values differ: {bad_frame[:10]}"
