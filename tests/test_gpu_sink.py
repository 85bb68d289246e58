"""The ground sink on the GPU (isink > 0, sink.f:46-167): parity of the
sink, of the columns' lost mass and of the state with the oracle over
several steps; the massl file in the reference's formatted layout; and a
run resumed from pdac.res and massl.NNNN against the uninterrupted run.

Tolerances as in the other parity tests: the step tolerance 1e-9
(relative L-infinity) for fields; the sink of the first boundary call,
from identical inputs, to 1e-13.  The massl file holds six significant
digits (G14.6E3: 0.dddddd, up to 5e-6 relative rounding), so a resumed
run's massl matches to that precision."""
import os

import numpy as np
import pytest

from helpers import STEP_FIELDS, compare_state, fortran_g, rel_linf
from sink_decks import seeded_case

pytestmark = pytest.mark.gpu


def _pair(builder):
    import pyoracle
    from pdac_b200.engine import Engine
    case = seeded_case(builder)
    return case, Engine(case), pyoracle.Oracle(case, order=pyoracle.ORDER_COLORED)


@pytest.mark.parametrize("builder", ["small_2d_sink", "small_3d_sink"])
def test_sink_parity(builder):
    case, eng, ora = _pair(builder)
    eng.boundary(1); ora.boundary(1)
    assert rel_linf(eng.get("sink"), ora.get("sink")) <= 1e-13
    assert rel_linf(eng.get("massl"), ora.get("massl")) <= 1e-13
    eng.close()
    case, eng, ora = _pair(builder)
    fields = STEP_FIELDS + (("vg", "vs") if case.is3d else ())
    fluid = (case.flag & 1) == 1
    for s in range(1, 5):
        assert eng.step(s) == ora.step(s)
        for name in ("sink", "massl"):
            assert rel_linf(eng.get(name), ora.get(name)) <= 1e-9, (s, name)
        errs, bad = compare_state(eng.download(), ora.get_state(), fields, 1e-9, case.nsolid, case.ncell, cells=fluid)
        assert not bad, (s, bad)
    assert np.count_nonzero(eng.get("massl")) > 0
    eng.close()


def _parse_2d(lines, ns):
    return [[float(v) for v in ln.split()] for ln in lines]


@pytest.mark.parametrize("builder", ["small_2d_sink", "small_3d_sink"])
def test_massl_file_layout(builder, tmp_path):
    from pdac_b200.engine import Engine
    case = seeded_case(builder)
    eng = Engine(case)
    for s in (1, 2):
        eng.step(s)
    path = str(tmp_path / "massl.0001")
    eng.write_mass_loss(path)
    ml = eng.get("massl")
    eng.close()
    ns = case.nsolid
    ntr = case.nx * (case.ny if case.is3d else 1)
    lines = open(path).read().split("\n")
    assert lines[-1] == ""
    lines = lines[:-1]
    at = lambda b, q: ml[q * ntr + b]
    if not case.is3d:
        # one line per column: the classes' values and the running total,
        # FORMAT(10(1x,G14.6E3))
        assert len(lines) == ntr
        total = 0.0
        for b, ln in enumerate(lines):
            s = 0.0
            for q in range(ns):
                s = s + at(b, q)
            total = total + s
            want = "".join(" " + fortran_g(v, 14, 6, 3) for v in [at(b, q) for q in range(ns)] + [total])
            assert ln == want
    else:
        # per class: two empty lines, ' MLn=' and the class total (G14.6),
        # an empty line, then the ntr column values ten to a line
        rows = -(-ntr // 10)
        assert len(lines) == ns * (4 + rows)
        for q in range(ns):
            blk = lines[q * (4 + rows):(q + 1) * (4 + rows)]
            total = 0.0
            for b in range(ntr):
                total = total + at(b, q)
            assert blk[0] == "" and blk[1] == "" and blk[3] == ""
            assert blk[2] == f" ML{q + 1}=" + fortran_g(total, 14, 6, 2)
            vals = [at(b, q) for b in range(ntr)]
            for r in range(rows):
                assert blk[4 + r] == "".join(" " + fortran_g(v, 14, 6, 3) for v in vals[10 * r:10 * r + 10])


@pytest.mark.parametrize("builder", ["small_2d_sink", "small_3d_sink"])
def test_resume_with_mass_loss(builder, tmp_path):
    """Steps 1-4 in one run against steps 1-2, pdac.res + massl file,
    steps 3-4 in a new context (2D without vent fluctuations, whose factor
    a restart does not carry)."""
    from pdac_b200.engine import Engine
    kw = {} if "3d" in builder else {"irand": 0}
    case = seeded_case(builder, **kw)
    a = Engine(case)
    for s in (1, 2):
        a.step(s)
    a.write_restart(str(tmp_path / "pdac.res"), 2 * case.deck["dt"], 1)
    a.write_mass_loss(str(tmp_path / "massl.0001"))
    for s in (3, 4):
        a.step(s)
    b = Engine(seeded_case(builder, **kw))
    b.read_mass_loss(str(tmp_path / "massl.0001"))
    b.read_restart(str(tmp_path / "pdac.res"))
    for s in (3, 4):
        b.step(s)
    fields = STEP_FIELDS + (("vg", "vs") if case.is3d else ())
    fluid = (case.flag & 1) == 1
    errs, bad = compare_state(b.download(), a.download(), fields, 1e-9, case.nsolid, case.ncell, cells=fluid)
    assert not bad, bad
    ma, mb = a.get("massl"), b.get("massl")
    assert np.count_nonzero(ma) > 0
    # six significant digits in the 0.dddddd form: rounding up to 5e-6 relative
    np.testing.assert_allclose(mb, ma, rtol=1e-5, atol=0)
    a.close()
    b.close()
