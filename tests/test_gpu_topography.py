"""Topography and immersed boundaries on the engine against the oracle.

Decks: a 2D cylindrical plume with a 60 m Gaussian hill 150 m from the axis
(profile file, itp = 1) and a 3D plume over three seeded Gaussian hills
(ASCII DEM, itp = 1) with a flat crater floor around the vent, each with
the staircase of no-slip cells (immb = 0) and with immersed boundaries
(immb = 1: forcing points, cut-cell face factors, hn fills).

Phase by phase from the same state, the boundary pass (whose cells the
engine runs in dependency levels), fieldn and tilde (with the flux masks
and forcing terms) agree with the oracle to 1e-12 over every cell, the
corrector takes the same number of outer sweeps, and whole steps agree to
1e-9 over the fluid cells, every step restarting the oracle from the
engine's state (the same scheme as the other multi-step parity tests).
"""
import numpy as np
import pytest

from helpers import STEP_FIELDS, compare_state, frame_mismatches, rel_linf

pytestmark = pytest.mark.gpu

TOL_EXPLICIT = 1e-12
TOL_STEP = 1e-9
CASES = [("small_2d_topo", 0), ("small_2d_topo", 1), ("small_3d_topo", 0), ("small_3d_topo", 1)]


def _case(tmp_path, builder, immb):
    from pdac_b200 import configs
    from pdac_b200.setup_state import Case
    return Case(getattr(configs, builder)(tmp_path, immb=immb))


def _all_cells(case, got, ref, names, tol, where):
    """Fluid cells (the immersed ones among them) by relative L-infinity,
    every other cell (walls below the topography, filled cells, the frame)
    value by value under the free in/outflow rule of frame_mismatches."""
    fluid = (case.flag & 1) == 1
    errs, bad = compare_state(got, ref, names, tol, case.nsolid, case.ncell, cells=fluid)
    assert not bad, f"{where}: fluid cells {bad}"
    bad_frame, _ = frame_mismatches(got, ref, names, case, tol)
    assert not bad_frame, f"{where}: other cells {bad_frame[:10]}"


@pytest.mark.parametrize("builder,immb", CASES)
def test_phases(tmp_path, builder, immb):
    import pyoracle
    from pdac_b200.engine import Engine
    case = _case(tmp_path, builder, immb)
    if immb:
        assert case.ib is not None and np.any(case.flag == 257) and np.any(case.flag == 512)
    eng = Engine(case)
    ora = pyoracle.Oracle(case, order=pyoracle.ORDER_COLORED)
    dt = case.deck["dt"]
    fields3 = STEP_FIELDS + (("vg", "vs") if case.is3d else ())
    for s in range(1, 4):
        ora.set_state(eng.download())
        eng.boundary(s); ora.boundary(s)
        _all_cells(case, eng.download(), ora.get_state(), fields3, TOL_EXPLICIT, f"boundary {s}")
        eng.fieldn(); ora.fieldn()
        eng.tilde(dt); ora.tilde(dt)
        tnames = ("rug", "rwg", "rus", "rws") + (("rvg", "rvs") if case.is3d else ())
        bad = {n: rel_linf(eng.get(n), ora.get(n)) for n in tnames}
        bad = {n: e for n, e in bad.items() if not e <= TOL_EXPLICIT}
        assert not bad, f"tilde {s}: {bad}"
        n1, n2 = eng.iter(dt), ora.iter(dt)
        assert n1 == n2, f"step {s}: outer sweeps {n1} vs {n2}"
        eng.ygas(dt); ora.ygas(dt)
        eng.htilde(dt); ora.htilde(dt)
        eng.ftem(dt); ora.ftem(dt)
        fluid = (case.flag & 1) == 1
        errs, badf = compare_state(eng.download(), ora.get_state(), fields3, TOL_STEP, case.nsolid, case.ncell,
                                   cells=fluid)
        assert not badf, f"step {s}: {badf}"
    eng.close()


@pytest.mark.parametrize("builder,immb,steps", [("small_2d_topo", 1, 30), ("small_3d_topo", 1, 12),
                                                ("small_2d_topo", 0, 30)])
def test_steps(tmp_path, builder, immb, steps):
    """Whole steps (pdac_gpu_step): equal outer sweeps and fields within 1e-9
    every step, the oracle restarted from the engine's state; the phase-mass
    totals agree to 1e-12."""
    import pyoracle
    from pdac_b200.engine import Engine
    case = _case(tmp_path, builder, immb)
    eng = Engine(case)
    ora = pyoracle.Oracle(case, order=pyoracle.ORDER_COLORED)
    fluid = (case.flag & 1) == 1
    fields3 = STEP_FIELDS + (("vg", "vs") if case.is3d else ())
    for s in range(1, steps + 1):
        ora.set_state(eng.download())
        n1, n2 = eng.step(s), ora.step(s)
        assert n1 == n2, f"step {s}: outer sweeps {n1} vs {n2}"
        errs, bad = compare_state(eng.download(), ora.get_state(), fields3, TOL_STEP, case.nsolid, case.ncell,
                                  cells=fluid)
        assert not bad, f"step {s}: {bad}"
        np.testing.assert_allclose(eng.mass_totals(), ora.mass_totals(), rtol=1e-12, atol=0, err_msg=f"step {s}")
    eng.close()


def test_hills_five_classes(tmp_path):
    """The large workload's deck (seeded Gaussian hills, immersed boundaries,
    five particle classes: the six-phase inner loop) on a 40 x 40 x 32 mesh:
    whole steps with equal outer sweeps and fields within 1e-9, the oracle
    restarted from the engine's state every step."""
    import pyoracle
    from pdac_b200 import configs
    from pdac_b200.engine import Engine
    from pdac_b200.setup_state import Case
    case = Case(configs.plume_3d_hills(nx=40, ny=40, nz=32, dem_dir=str(tmp_path)))
    assert case.nsolid == 5 and case.ib is not None
    eng = Engine(case)
    ora = pyoracle.Oracle(case, order=pyoracle.ORDER_COLORED)
    fluid = (case.flag & 1) == 1
    fields3 = STEP_FIELDS + ("vg", "vs")
    for s in range(1, 7):
        ora.set_state(eng.download())
        n1, n2 = eng.step(s), ora.step(s)
        assert n1 == n2, f"step {s}: outer sweeps {n1} vs {n2}"
        errs, bad = compare_state(eng.download(), ora.get_state(), fields3, TOL_STEP, case.nsolid, case.ncell,
                                  cells=fluid)
        assert not bad, f"step {s}: {bad}"
    eng.close()


def test_forcing_point_checks_reject_bad_tables(tmp_path):
    """An immersed cell without a forcing point (the reference stops there,
    bdry.f:111-113) is rejected at create with PDAC_ERR_CONFIG, by the
    engine as by the oracle."""
    import pyoracle
    from pdac_b200 import abi
    from pdac_b200.engine import Engine, PdacError
    case = _case(tmp_path, "small_2d_topo", 1)
    # an immersed cell loses its forcing points
    m = int(np.flatnonzero(case.flag == 257)[0])
    for a in range(3):
        case.ib.num[a][m] = 0
    with pytest.raises(PdacError) as e:
        Engine(case)
    assert e.value.status == abi.PDAC_ERR_CONFIG
    with pytest.raises(RuntimeError, match="config"):
        pyoracle.Oracle(case)


@pytest.mark.parametrize("builder,immb", [("small_2d_topo", 1), ("small_3d_topo", 1), ("small_3d_topo", 0)])
def test_sub_grid_model_with_ground_roughness(tmp_path, builder, immb):
    """iturb = 2 (turbo.f:72-101): the mixing length of every cell equals the
    oracle's bit for bit, and four steps with the static model and the
    particle sub-grid stress agree over the fluid cells to 1e-9, the
    model's viscosities included, with the same sweep counts."""
    import pyoracle
    from pdac_b200 import configs
    from pdac_b200.engine import Engine
    from pdac_b200.setup_state import Case
    d = getattr(configs, builder)(tmp_path, immb=immb)
    d.set("model", iturb=2, modturbo=1, iss=1)
    d.set("topography", zrough=2.0)
    case = Case(d)
    eng = Engine(case)
    ora = pyoracle.Oracle(case, order=pyoracle.ORDER_COLORED)
    assert np.array_equal(eng.get("smag"), ora.get("smag"))
    fields = STEP_FIELDS + (("vg", "vs") if case.is3d else ())
    fluid = (case.flag & 1) == 1
    for s in range(1, 5):
        n1, n2 = eng.step(s), ora.step(s)
        assert n1 == n2, f"step {s}: outer sweeps gpu {n1} oracle {n2}"
        got, ref = eng.download(), ora.get_state()
        errs, bad = compare_state(got, ref, fields, TOL_STEP, case.nsolid, case.ncell, cells=fluid)
        assert not bad, f"step {s}: {bad}"
        for name in ("mugt", "kapgt", "must"):
            e = rel_linf(eng.get(name), ora.get(name))
            assert e <= TOL_STEP, f"step {s}: {name} {e}"
    eng.close()

