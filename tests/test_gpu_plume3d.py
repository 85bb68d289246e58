"""The 3D plume deck (20 m cells, 5 x 5 vent at 1000 K and 150 m/s, three
particle classes) on a 64 x 64 x 48 grid for 25 steps, engine against the
coloured oracle every step.

At this size the deck reproduces what the 256 x 256 x 192 benchmark grid
shows at the same step numbers: in steps 9 and 23 a few cells next to the
vent edge never reach |dg| <= conv, and the corrector stops at maxout (500
sweeps, nit = 501; iter.f:428-450).  The oracle does the same: the outer
sweep counts are equal in every step, the unconverged cells are the same
cells, and the fields agree to 1e-9 (relative L-infinity over the fluid
cells) after every step.
"""
import numpy as np
import pytest

from helpers import STEP_FIELDS, compare_state

pytestmark = pytest.mark.gpu

TOL = 1e-9
FIELDS3 = STEP_FIELDS + ("vg", "vs")


def test_plume3d_64x64x48_25_steps():
    import pyoracle
    from pdac_b200 import configs
    from pdac_b200.engine import Engine
    from pdac_b200.setup_state import Case
    case = Case(configs.plume_3d(nx=64, ny=64, nz=48))
    eng = Engine(case)
    ora = pyoracle.Oracle(case, order=pyoracle.ORDER_COLORED)
    fluid = (case.flag & 1) == 1
    maxout_steps = []
    for s in range(1, 26):
        n1, n2 = eng.step(s), ora.step(s)
        assert n1 == n2, f"step {s}: outer sweeps engine {n1} oracle {n2}"
        g, o = eng.unconverged_cells(), ora.unconverged_cells()
        assert np.array_equal(g, o), f"step {s}: unconverged cells differ"
        if n1 > case.deck["maxout"]:
            maxout_steps.append(s)
            assert g.size > 0
        errs, bad = compare_state(eng.download(), ora.get_state(), FIELDS3, TOL, case.nsolid, case.ncell, cells=fluid)
        assert not bad, f"step {s} (nit {n1}): {bad}"
    assert maxout_steps == [9, 23], maxout_steps
    eng.close()
