"""Failure statuses of the C ABI, each provoked on the host: no GPU fault,
trap or hang is involved (the corrector and the caloric inversion stop
after maxout sweeps and 2000 iterations whatever the values).

* PDAC_ERR_NONFINITE: a NaN or Inf in a host buffer is refused at upload;
  a NaN vent factor handed to pdac_gpu_set_vent_factors reaches the state
  and the step reports it.
* PDAC_ERR_MAXOUT: iter ends without convergence after maxout sweeps with
  cstop set (iter.f:449); without cstop the step returns PDAC_OK with
  nit = maxout + 1 and the unconverged cells the reference reports
  (iter.f:428-447), the same cells as the oracle's.
* PDAC_ERR_EOS: an enthalpy no temperature satisfies (ftem.f:191-193).
"""
import ctypes as C

import numpy as np
import pytest

from helpers import STEP_FIELDS, compare_state

pytestmark = pytest.mark.gpu


def _engine(case, upload=True):
    from pdac_b200.engine import Engine
    return Engine(case, upload=upload)


@pytest.mark.parametrize("field,value", [("p", np.nan), ("rlk", np.inf), ("xgc", -np.inf)])
def test_upload_refuses_non_finite_values(field, value):
    from pdac_b200 import abi, configs
    from pdac_b200.engine import PdacError
    from pdac_b200.setup_state import Case
    case = Case(configs.small_2d())
    eng = _engine(case, upload=False)
    bad = {k: np.array(v, copy=True) for k, v in case.state.items()}
    fluid = np.flatnonzero(case.flag & 1)
    bad[field][fluid[len(fluid) // 2]] = value
    with pytest.raises(PdacError) as e:
        eng.upload(bad)
    assert e.value.status == abi.PDAC_ERR_NONFINITE
    assert field in str(e.value)
    eng.upload(case.state)  # a clean state is accepted afterwards
    assert eng.step(1) >= 1
    eng.close()


def test_step_reports_a_non_finite_state():
    from pdac_b200 import abi, configs
    from pdac_b200.engine import PdacError
    from pdac_b200.setup_state import Case
    d = configs.small_2d()
    d.set("numeric", maxout=5)
    case = Case(d)
    eng = _engine(case)
    eng.set_vent_factors(np.full(len(case.vent), np.nan))
    with pytest.raises(PdacError) as e:
        eng.step(1)
    assert e.value.status == abi.PDAC_ERR_NONFINITE
    eng.close()


def _maxout_case(cstop, is3d):
    from pdac_b200 import configs
    from pdac_b200.setup_state import Case
    d = configs.small_3d(nx=14, ny=12, nz=16) if is3d else configs.small_2d(nx=16, nz=20)
    d.set("numeric", maxout=2)
    d.set("control", cstop=cstop)
    return Case(d)


@pytest.mark.parametrize("is3d", [False, True])
def test_maxout_without_cstop_matches_the_oracle(is3d):
    import pyoracle
    case = _maxout_case(False, is3d)
    eng = _engine(case)
    ora = pyoracle.Oracle(case, order=pyoracle.ORDER_COLORED)
    fields = STEP_FIELDS + (("vg", "vs") if is3d else ())
    for s in (1, 2):
        n1, n2 = eng.step(s), ora.step(s)
        assert n1 == n2 == 3, (n1, n2)
        g, o = eng.unconverged_cells(), ora.unconverged_cells()
        assert g.size > 0
        assert np.array_equal(g, o), f"step {s}: gpu {g[:10]} oracle {o[:10]}"
        fluid = (case.flag & 1) == 1
        errs, bad = compare_state(eng.download(), ora.get_state(), fields, 1e-9, case.nsolid, case.ncell, cells=fluid)
        assert not bad, bad
    eng.close()


@pytest.mark.parametrize("is3d", [False, True])
def test_maxout_with_cstop_stops_the_step(is3d):
    import pyoracle
    from pdac_b200 import abi
    from pdac_b200.engine import PdacError
    case = _maxout_case(True, is3d)
    eng = _engine(case)
    with pytest.raises(PdacError) as e:
        eng.step(1)
    assert e.value.status == abi.PDAC_ERR_MAXOUT
    assert "max number of iters" in str(e.value)
    ora = pyoracle.Oracle(case)
    nit = C.c_int(0)
    assert ora.L.pdac_oracle_step(ora.h, 1, C.byref(nit)) == abi.PDAC_ERR_MAXOUT
    eng.close()


def test_converged_iter_lists_no_cells():
    from pdac_b200 import configs
    from pdac_b200.setup_state import Case
    case = Case(configs.small_2d())
    eng = _engine(case)
    eng.step(1)
    assert eng.unconverged_cells().size == 0
    eng.close()


@pytest.mark.parametrize("is3d", [False, True])
def test_impossible_enthalpy_is_an_eos_failure(is3d):
    """A negative gas enthalpy in a block of fluid cells has no positive
    temperature: caloric_eosg fails there (eosg.f:139-223) and ftem reports
    more than one failure (ftem.f:191-193), in the engine and the oracle."""
    import pyoracle
    from pdac_b200 import abi, configs
    from pdac_b200.engine import PdacError
    from pdac_b200.setup_state import Case
    case = Case(configs.small_3d() if is3d else configs.small_2d())
    st = {k: np.array(v, copy=True) for k, v in case.state.items()}
    fluid = np.flatnonzero(case.flag & 1)
    mid = fluid[len(fluid) // 2:len(fluid) // 2 + 4]
    st["sieg"][mid] = -1.0e6
    eng = _engine(case, upload=False)
    eng.upload(st)
    with pytest.raises(PdacError) as e:
        eng.step(1)
    assert e.value.status == abi.PDAC_ERR_EOS
    ora = pyoracle.Oracle(case)
    ora.set_state(st)
    nit = C.c_int(0)
    assert ora.L.pdac_oracle_step(ora.h, 1, C.byref(nit)) == abi.PDAC_ERR_EOS
    eng.close()
