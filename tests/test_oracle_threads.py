"""The oracle's 3D cell loops on several host threads give the same bits as
on one thread, and its report of the corrector's end without convergence
(iter.f:428-450) follows the reference.

Each multi-threaded loop writes every value from exactly one cell (the one
that writes it last in the serial order) and the corrector runs one colour's
cells at a time, so equality is exact; the grids are large enough (more than
4096 cells) that the loops really split.
"""
import numpy as np
import pytest

import pyoracle
from pdac_b200 import abi, configs
from pdac_b200.setup_state import Case


def _run(builder, threads, steps, **kw):
    pyoracle.set_threads(threads)
    try:
        case = Case(builder(**kw))
        o = pyoracle.Oracle(case, order=pyoracle.ORDER_COLORED)
        nits = [o.step(s) for s in range(1, steps + 1)]
        return o.get_state(), nits, o.unconverged_cells(), o.mass_totals()
    finally:
        pyoracle.set_threads(0)


@pytest.mark.parametrize("builder,kw", [
    (configs.plume_3d, dict(nx=24, ny=20, nz=28, vent_cells=4)),
    (configs.small_3d_les, dict(nx=20, ny=18, nz=24)),
])
def test_threads_give_the_same_bits(builder, kw):
    a = _run(builder, 1, 4, **kw)
    b = _run(builder, 4, 4, **kw)
    assert a[1] == b[1], f"outer sweeps {a[1]} vs {b[1]}"
    for k in a[0]:
        assert np.array_equal(a[0][k], b[0][k]), k
    assert np.array_equal(a[2], b[2])
    assert np.array_equal(a[3], b[3])


def test_lexicographic_order_is_unaffected_by_threads():
    kw = dict(nx=24, ny=20, nz=28, vent_cells=4)
    res = []
    for th in (1, 4):
        pyoracle.set_threads(th)
        case = Case(configs.plume_3d(**kw))
        o = pyoracle.Oracle(case, order=pyoracle.ORDER_LEXICOGRAPHIC)
        nits = [o.step(s) for s in (1, 2, 3)]
        res.append((o.get_state(), nits))
    pyoracle.set_threads(0)
    assert res[0][1] == res[1][1]
    for k in res[0][0]:
        assert np.array_equal(res[0][0][k], res[1][0][k]), k


def _maxout_case(cstop):
    d = configs.small_3d(nx=14, ny=12, nz=16)
    d.set("numeric", maxout=2)
    d.set("control", cstop=cstop)
    return Case(d)


def test_maxout_without_cstop_reports_the_unconverged_cells():
    """nit = maxout + 1 and the cells of the last sweep that ran the inner
    loop are listed (iter.f:428-447); the run goes on (cstop = .FALSE.)."""
    case = _maxout_case(False)
    o = pyoracle.Oracle(case)
    nit = o.step(1)
    assert nit == 3
    cells = o.unconverged_cells()
    assert cells.size > 0
    assert np.all(np.diff(cells) > 0)
    assert np.all((case.flag[cells] & 1) == 1)


def test_maxout_with_cstop_stops_the_step():
    case = _maxout_case(True)
    o = pyoracle.Oracle(case)
    L = o.L
    nit = pyoracle.C.c_int(0)
    st = L.pdac_oracle_step(o.h, 1, pyoracle.C.byref(nit))
    assert st == abi.PDAC_ERR_MAXOUT
    assert nit.value == 3


def test_converged_iter_reports_no_cells():
    case = Case(configs.small_3d())
    o = pyoracle.Oracle(case)
    nit = o.step(1)
    assert nit <= case.deck["maxout"]
    assert o.unconverged_cells().size == 0
