"""The implicit-flux options of the semi-implicit path on the GPU against
the oracle: implicit_fluxes runs tilde at the start of every outer sweep of
iter (iter.f:211-226) and none before it (prog.f:246-251), so the
predictor sees the zeroed tilde terms of allocate_fluxes (tilde.f:56-102);
implicit_enthalpy runs ftem (after htilde with implicit_fluxes) at the end
of every sweep (iter.f:362-379) instead of after ygas.  The engine must take
the same number of sweeps as the oracle and agree to the step tolerance 1e-9
(relative L-infinity)."""
import pytest

from helpers import STEP_FIELDS, compare_state

pytestmark = pytest.mark.gpu

# With implicit_enthalpy the sweeps of these decks do not converge: each
# sweep's ftem moves the temperatures the next sweep's equation of state
# reads, and the coupled iteration runs to maxout in the oracle as on the
# GPU.  A non-contracting iteration amplifies last-bit differences of the
# caloric inversion (the first five sweeps are bit-identical); maxout = 20
# keeps the comparison within the step tolerance.
CASES = [
    ("small_2d_implicit", dict(fluxes=True, enthalpy=False, dt=0.002)),
    ("small_2d_implicit", dict(fluxes=False, enthalpy=True, maxout=20)),
    ("small_2d_implicit", dict(fluxes=True, enthalpy=True, dt=0.002, maxout=20)),
    ("small_3d_implicit", dict(fluxes=True, enthalpy=True, dt=0.001, maxout=20)),
]


@pytest.mark.parametrize("builder,kw", CASES, ids=["2d-fluxes", "2d-enthalpy", "2d-both", "3d-both"])
def test_implicit_modes_match_oracle(builder, kw):
    import pyoracle
    from pdac_b200 import configs
    from pdac_b200.engine import Engine
    from pdac_b200.setup_state import Case
    case = Case(getattr(configs, builder)(**kw))
    eng = Engine(case)
    ora = pyoracle.Oracle(case, order=pyoracle.ORDER_COLORED)
    fields = STEP_FIELDS + (("vg", "vs") if case.is3d else ())
    fluid = (case.flag & 1) == 1
    for s in range(1, 4):
        n1, n2 = eng.step(s), ora.step(s)
        assert n1 == n2, (s, n1, n2)
        errs, bad = compare_state(eng.download(), ora.get_state(), fields, 1e-9, case.nsolid, case.ncell, cells=fluid)
        assert not bad, (s, bad)
    eng.close()


def test_static_iter_rejects_the_implicit_modes():
    from pdac_b200 import configs
    from pdac_b200.engine import Engine, PdacError
    from pdac_b200.setup_state import Case
    import ctypes as C
    eng = Engine(Case(configs.small_2d_implicit()))
    eng.boundary(1)
    eng.fieldn()
    nit = C.c_int(0)
    st = eng.L.pdac_gpu_iter_static(eng.h, C.c_double(0.01), C.byref(nit))
    assert st == 1  # PDAC_ERR_CONFIG
    eng.close()
