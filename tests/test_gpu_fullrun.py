"""Whole runs on the GPU against the oracle, checked the way the reference's runs
are checked: phase-mass totals (the fluid-cell sums of residuals.f:14-130)
to 1e-12 relative after every step, and for a run with the ground sink the
deposited mass per class (the columns' massl, sink.f) to 1e-6 relative and
the runout, the largest distance from the vent axis at which the particle
volume fraction of the first fluid row exceeds 1e-6, exactly."""
import numpy as np
import pytest

from sink_decks import seeded_case

pytestmark = pytest.mark.gpu


def _pair(case):
    import pyoracle
    from pdac_b200.engine import Engine
    return Engine(case), pyoracle.Oracle(case, order=pyoracle.ORDER_COLORED)


@pytest.mark.parametrize("builder,steps", [("small_2d", 30), ("small_3d", 12), ("small_2d_rk3", 30)])
def test_phase_mass_totals(builder, steps):
    from pdac_b200 import configs
    from pdac_b200.setup_state import Case
    case = Case(getattr(configs, builder)())
    eng, ora = _pair(case)
    for s in range(1, steps + 1):
        assert eng.step(s) == ora.step(s)
        a, b = eng.mass_totals(), ora.mass_totals()
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=0, err_msg=f"step {s}")
    eng.close()


def _runout(case, rlk, threshold=1e-6):
    """Largest cell-centre distance from the axis (2D) of a first-row fluid
    cell whose total particle volume fraction exceeds threshold."""
    n, nx = case.ncell, case.nx
    x, xb = [], 0.0
    for i, d in enumerate(case.dx):
        if i == 0:
            x.append(-0.5 * d)
        else:
            xb = xb + d
            x.append(xb - 0.5 * d)
    best = 0.0
    for i in range(nx):
        c = i + nx * 1  # k = 2, the first row above the ground
        if not case.flag[c] & 1:
            continue
        eps = sum(rlk[q * n + c] / case.deck["density"][q] for q in range(case.nsolid))
        if eps > threshold:
            best = max(best, x[i])
    return best


def test_deposit_and_runout():
    case = seeded_case("small_2d_sink", irand=0)
    eng, ora = _pair(case)
    for s in range(1, 11):
        assert eng.step(s) == ora.step(s)
    ntr, ns = case.nx, case.nsolid
    ma, mb = eng.get("massl").reshape(ns, ntr), ora.get("massl").reshape(ns, ntr)
    dep_a, dep_b = ma.sum(axis=1), mb.sum(axis=1)
    assert np.all(dep_b != 0.0)
    np.testing.assert_allclose(dep_a, dep_b, rtol=1e-6, atol=0)
    ra = _runout(case, eng.download()["rlk"])
    rb = _runout(case, ora.get_state()["rlk"])
    assert ra == rb and ra > 0.0
    eng.close()


@pytest.mark.parametrize("sink", [False, True])
def test_config0_full_run_500_steps(sink):
    """The 2D workload (128 x 192, two classes, 500 steps of 10 ms) run
    through to the end on the engine.  Every step is checked against the
    oracle started from the engine's state of the step before: the same
    number of outer sweeps, phase-mass totals to 1e-12 relative and the
    fields within 1e-9 (relative L-infinity over the fluid cells).  The two
    agree bit for bit after every one of the 500 steps (no step needs the
    oracle restarted; the run reaches maxout in 18 steps), so this is also
    a comparison of two free-running runs.  At the end the runout agrees
    exactly and, with the ground sink over the whole ground (isink = 1,
    0 < r < 1e9 m), the mass taken out per class over the 500 steps agrees
    to 1e-6 relative."""
    from helpers import STEP_FIELDS, compare_state
    from pdac_b200 import configs
    from pdac_b200.setup_state import Case
    d = configs.plume_2d()
    if sink:
        d.set("model", isink=1, rprox=0.0, rdist=1.0e9)
    case = Case(d)
    eng, ora = _pair(case)
    fluid = (case.flag & 1) == 1
    resynced = []
    for s in range(1, 501):
        n1, n2 = eng.step(s), ora.step(s)
        assert n1 == n2, f"step {s}: outer sweeps {n1} vs {n2}"
        np.testing.assert_allclose(eng.mass_totals(), ora.mass_totals(), rtol=1e-12, atol=0, err_msg=f"step {s}")
        got, ref = eng.download(), ora.get_state()
        if any(not np.array_equal(got[k], ref[k]) for k in got):
            errs, bad = compare_state(got, ref, STEP_FIELDS, 1e-9, case.nsolid, case.ncell, cells=fluid)
            assert not bad, f"step {s} (nit {n1}): {bad}"
            ora.set_state(got)
            resynced.append(s)
    assert not resynced, f"steps that did not end bit for bit: {resynced[:10]}"
    ra = _runout(case, eng.download()["rlk"])
    rb = _runout(case, ora.get_state()["rlk"])
    assert ra == rb and ra > 0.0
    if sink:
        ns = case.nsolid
        dep_a = eng.get("massl").reshape(ns, case.nx).sum(axis=1)
        dep_b = ora.get("massl").reshape(ns, case.nx).sum(axis=1)
        assert np.all(dep_b != 0.0)  # the sink term's sign: mass taken out is negative (sink.f:123-167)
        np.testing.assert_allclose(dep_a, dep_b, rtol=1e-6, atol=0)
    eng.close()
