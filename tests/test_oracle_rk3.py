"""The CPU oracle of the explicit SSP-RK3 solver (explicit_solver.f).

Besides the regression fixtures (test_golden.py), the final ODE solve of
explicit_iter (explicit_solver.f:1116-1143) is checked to set the new
densities of every fluid cell to the rhs3 mass rows (the n-level density
plus dt (k1 + k2 + 4 k3) / 6, clipped at zero for the particles), and a few
whole steps to stay finite.
"""
import numpy as np
import pytest

from pdac_b200 import configs
from pdac_b200.setup_state import Case


def _oracle(deck):
    import pyoracle
    case = Case(deck)
    return case, pyoracle.Oracle(case)


@pytest.mark.parametrize("builder", ["small_2d_rk3", "small_3d_rk3"])
def test_final_density_is_rhs3_mass_row(builder):
    case, o = _oracle(getattr(configs, builder)())
    o.boundary(1)
    o.initialize_fieldn()
    o.explicit_iter(case.deck["dt"])
    n = case.ncell
    neq = (5 if case.is3d else 4) * (case.nsolid + 1)
    rhs3 = o.get("rhs3").reshape(n, neq)
    fluid = (case.flag & 1) == 1
    np.testing.assert_array_equal(o.get("rgp")[fluid], rhs3[fluid, 0])
    rlk = o.get("rlk").reshape(case.nsolid, n)
    for s in range(case.nsolid):
        np.testing.assert_array_equal(rlk[s][fluid], np.maximum(0.0, rhs3[fluid, 1 + s]))


@pytest.mark.parametrize("builder", ["small_2d_rk3", "small_3d_rk3"])
def test_steps_stay_finite(builder):
    case, o = _oracle(getattr(configs, builder)())
    for s in range(1, 6):
        o.step(s)
    for name, a in o.get_state().items():
        if a is not None:
            assert np.all(np.isfinite(a)), name
