"""The files of the time loop, written and read by the engine in the
reference's formats: pdac.res (tapewr / taperd), output.NNNN (outp) and
pdac.chm (print_mass_residuals), and the prog.f driver that produces them.

Records are parsed here independently (tests/helpers.fortran_records) and
compared with the engine's state: bit-exact for REAL*8 records, exact
single-precision conversion for the REAL*4 output records.  A run resumed
from a restart file is compared with the uninterrupted run at the step
tolerance 1e-9: taperd does not store the gas specific heat or the void
fraction, and cnvert re-derives them (setup.f:359-391), which moves them by
round-off, as in the reference.
"""
import os
import struct

import numpy as np
import pytest

from helpers import STEP_FIELDS, compare_state, fortran_g, fortran_records, rel_linf

pytestmark = pytest.mark.gpu

def _engine(builder, **kw):
    from pdac_b200 import configs
    from pdac_b200.engine import Engine
    from pdac_b200.setup_state import Case
    case = Case(getattr(configs, builder)(**kw))
    return case, Engine(case)


def _expected_restart_arrays(case, st):
    n, ns, ng = case.ncell, case.nsolid, case.ngas
    blk = lambda name, q: st[name][q * n:(q + 1) * n]
    out = [st["p"], st["ug"]] + ([st["vg"]] if case.is3d else []) + [st["wg"], st["sieg"]]
    out += [blk("rlk", q) for q in range(ns)]
    for q in range(ns):
        out += [blk("us", q)] + ([blk("vs", q)] if case.is3d else []) + [blk("ws", q)]
    out += [blk("sies", q) for q in range(ns)]
    out += [blk("ygc", q) for q in range(ng)]
    out += [st["rgp"], st["rog"], st["tg"]]
    out += [blk("ts", q) for q in range(ns)]
    return out


@pytest.mark.parametrize("builder", ["small_2d", "small_3d"])
def test_restart_file_layout(builder, tmp_path):
    case, eng = _engine(builder)
    for s in range(1, 3):
        eng.step(s)
    path = str(tmp_path / "pdac.res")
    eng.write_restart(path, 0.25, 7)
    recs = fortran_records(path)
    t, nx, ny, nz, ns, ng, nfil = struct.unpack("<d6i", recs[0])
    assert (t, nx, ny, nz, ns, ng, nfil) == (0.25, case.nx, case.ny, case.nz, case.nsolid, case.ngas, 7)
    assert list(struct.unpack(f"<{case.ngas}i", recs[1])) == list(case.gas_type)
    want = _expected_restart_arrays(case, eng.download())
    assert len(recs) == 2 + len(want)
    for r, a in zip(recs[2:], want):
        np.testing.assert_array_equal(np.frombuffer(r, dtype="<f8"), a)


@pytest.mark.parametrize("builder", ["small_2d", "small_3d", "small_2d_rk3"])
def test_resume_from_restart(builder, tmp_path):
    """Steps 1-4 in one run against steps 1-2, restart, steps 3-4.  The 2D
    decks run without vent fluctuations (irand = 0): their previous factor
    is not in the restart file and restarts from zero (vent.f:176-178), in
    the reference as here, so with irand = 1 a resumed run differs from the
    uninterrupted one by design."""
    kw = {} if builder == "small_3d" else {"irand": 0}
    case, a = _engine(builder, **kw)
    path = str(tmp_path / "pdac.res")
    for s in (1, 2):
        a.step(s)
    a.write_restart(path, 2 * case.deck["dt"], 3)
    for s in (3, 4):
        a.step(s)
    _, b = _engine(builder, **kw)
    t, nfil = b.read_restart(path)
    assert t == 2 * case.deck["dt"] and nfil == 3
    # cnvert's derived fields right after the read
    st = b.download()
    ns = case.nsolid
    ep = 1.0 - sum(st["rlk"][q * case.ncell:(q + 1) * case.ncell] / case.deck["density"][q] for q in range(ns))
    assert rel_linf(st["ep"], ep) <= 1e-15
    for s in (3, 4):
        b.step(s)
    fluid = (case.flag & 1) == 1
    fields = STEP_FIELDS + (("vg", "vs") if case.is3d else ())
    got, ref = b.download(), a.download()
    errs, bad = compare_state(got, ref, fields, 1e-9, case.nsolid, case.ncell, cells=fluid)
    assert not bad, bad


def test_restart_rejects_other_mesh(tmp_path):
    from pdac_b200.engine import PdacError
    case, a = _engine("small_2d")
    path = str(tmp_path / "pdac.res")
    a.write_restart(path, 0.0, 0)
    _, b = _engine("small_2d", nx=14)
    with pytest.raises(PdacError, match="inconsistent dimension nx"):
        b.read_restart(path)


@pytest.mark.parametrize("builder", ["small_2d", "small_3d"])
def test_output_file_layout(builder, tmp_path):
    case, eng = _engine(builder)
    eng.step(1)
    path = str(tmp_path / "output.0001")
    eng.write_output(path, 0.01)
    recs = fortran_records(path)
    assert np.frombuffer(recs[0], dtype="<f4")[0] == np.float32(0.01)
    st = eng.download()
    n, ns, ng = case.ncell, case.nsolid, case.ngas
    blk = lambda name, q: st[name][q * n:(q + 1) * n]
    want = [st["p"], st["ug"]] + ([st["vg"]] if case.is3d else []) + [st["wg"], st["tg"]]
    want += [blk("xgc", q) for q in range(ng)]
    for q in range(ns):
        want += [blk("rlk", q) * (1.0 / case.deck["density"][q])]
        want += [blk("us", q)] + ([blk("vs", q)] if case.is3d else []) + [blk("ws", q), blk("ts", q)]
    assert len(recs) == 1 + len(want)
    for r, a in zip(recs[1:], want):
        np.testing.assert_array_equal(np.frombuffer(r, dtype="<f4"), a.astype(np.float32))


def _serial_residuals(case, st, nswp, dt):
    """print_mass_residuals in the reference's serial cell order."""
    n, ns, ng = case.ncell, case.nsolid, case.ngas
    nx, ny = case.nx, case.ny
    dx, dz = case.dx, case.dz
    # radial metric of grid.f:306-345 (ones in Cartesian geometry)
    r, rb = np.ones(nx), np.ones(nx)
    if not case.is3d and case.itc == 1:
        xb, x = np.zeros(nx), np.zeros(nx)
        x[0] = -0.5 * dx[0] + xb[0]
        for i in range(1, nx):
            xb[i] = xb[i - 1] + dx[i]
            x[i] = xb[i] - 0.5 * dx[i]
        r, rb = x, xb
    res_g, res_s, res_gc = 0.0, [0.0] * ns, [0.0] * ng
    mag = np.zeros(1 + ns + ng)  # sums of |term|, the scale of each total's round-off
    for c in range(n):
        i, j, k = c % nx, (c // nx) % ny, c // (nx * ny)
        f = int(case.flag[c])
        if f & 1:
            vol = dx[i] * case.dy[j] * dz[k] if case.is3d else r[i] * dx[i] * dz[k]
            res_g += st["rgp"][c] * vol
            mag[0] += abs(st["rgp"][c] * vol)
            for q in range(ns):
                res_s[q] += st["rlk"][q * n + c] * vol
                mag[1 + q] += abs(st["rlk"][q * n + c] * vol)
            for q in range(ng):
                res_gc[q] += st["rgp"][c] * st["ygc"][q * n + c] * vol
                mag[1 + ns + q] += abs(st["rgp"][c] * st["ygc"][q * n + c] * vol)
        elif f in (16, 64):
            if case.is3d:
                sx, sy, sz = dz[k] * case.dy[j], dx[i] * dz[k], case.dy[j] * dx[i]
            else:
                sx, sy, sz = dz[k] * rb[i], 0.0, dx[i] * r[i]
            fl = st["ug"][c] * sx + st["wg"][c] * sz + (st["vg"][c] * sy if case.is3d else 0.0)
            res_g -= st["rgp"][c] * fl * nswp * dt
            mag[0] += abs(st["rgp"][c] * fl * nswp * dt)
            for q in range(ns):
                fs = st["us"][q * n + c] * sx + st["ws"][q * n + c] * sz + (st["vs"][q * n + c] * sy if case.is3d else 0.0)
                res_s[q] -= st["rlk"][q * n + c] * fs * nswp * dt
                mag[1 + q] += abs(st["rlk"][q * n + c] * fs * nswp * dt)
            for q in range(ng):
                res_gc[q] -= st["rgp"][c] * st["ygc"][q * n + c] * fl * nswp * dt
                mag[1 + ns + q] += abs(st["rgp"][c] * st["ygc"][q * n + c] * fl * nswp * dt)
    return np.array([res_g] + res_s + res_gc), mag


@pytest.mark.parametrize("builder", ["small_2d", "small_3d"])
def test_mass_check_line(builder, tmp_path):
    case, eng = _engine(builder)
    dt = case.deck["dt"]
    for s in (1, 2, 3):
        eng.step(s)
    res = eng.mass_residuals(3, dt)
    vals = np.concatenate([[res["res_g"]], res["res_s"], res["res_gc"]])
    # the totals are sums of many terms, some of them cancelling: the
    # device's summation order differs from the reference's serial order by
    # round-off of the terms' magnitude
    ref, mag = _serial_residuals(case, eng.download(), 3, dt)
    assert np.all(np.abs(vals - ref) <= 1e-13 * mag), (vals, ref, mag)
    path = str(tmp_path / "pdac.chm")
    eng.append_mass_check(path, 3, dt)
    eng.append_mass_check(path, 4, dt)
    lines = open(path).read().splitlines()
    assert len(lines) == 2
    allv = list(vals) + [res["mfr"]]
    want = f"{3:8d}" + "".join(fortran_g(v) for v in allv)
    assert lines[0] == want
    assert float(lines[0][8:38]) == pytest.approx(res["res_g"], rel=1e-19)


def test_time_loop_driver_files(tmp_path):
    """files.run on the 2D deck: output.0000 at the first step and every
    nprint steps, pdac.chm every step, pdac.res every ndump steps; a second
    call in restart mode continues from the restart file."""
    from pdac_b200 import configs, files
    from pdac_b200.engine import Engine
    from pdac_b200.setup_state import Case
    d = configs.small_2d()
    dt = d["dt"]
    d.set("control", tpr=2 * dt, tdump=4 * dt, imr=1, tstop=1.0)
    case = Case(d)
    eng = Engine(case)
    t, nfil, sweep = files.run(eng, str(tmp_path), max_steps=5)
    assert sweep == 5 and nfil == 3
    names = sorted(os.listdir(tmp_path))
    assert names == ["output.0000", "output.0001", "output.0002", "pdac.chm", "pdac.res"]
    assert len(open(tmp_path / "pdac.chm").read().splitlines()) == 5
    recs = fortran_records(str(tmp_path / "pdac.res"))
    assert struct.unpack("<d6i", recs[0])[0] == pytest.approx(4 * dt) and struct.unpack("<d6i", recs[0])[6] == 3
    d.set("control", restart_mode="restart")
    eng2 = Engine(Case(d))
    t2, nfil2, sweep2 = files.run(eng2, str(tmp_path), max_steps=2)
    assert sweep2 == 6 and nfil2 == 4


@pytest.mark.parametrize("builder", ["small_2d_mixture", "small_3d_mixture"])
def test_mixture_fields_match_oracle(builder):
    """compute_mixture_fields after every step (prog.f:331): mixture
    density, velocity, temperature and mass fractions against the oracle at
    the step tolerance."""
    import pyoracle
    from pdac_b200 import configs
    from pdac_b200.engine import Engine
    from pdac_b200.setup_state import Case
    case = Case(getattr(configs, builder)())
    eng = Engine(case)
    ora = pyoracle.Oracle(case, order=pyoracle.ORDER_COLORED)
    names = ["rhom", "um", "wm", "tm", "yd"] + (["vm"] if case.is3d else [])
    for s in (1, 2, 3):
        assert eng.step(s) == ora.step(s)
        for name in names:
            assert rel_linf(eng.get(name), ora.get(name)) <= 1e-9, (s, name)
    eng.close()


def _formatted_blocks(text):
    """Split a formatted output file into (time line, [(name, values)])."""
    lines = text.split("\n")
    assert lines[:3] == ["", "", ""] and lines[3].startswith(" @@@ TIME = ")
    blocks, q = [], 4
    while q < len(lines) and lines[q:q + 2] == ["", ""] and q + 3 < len(lines):
        name = lines[q + 2]
        assert lines[q + 3] == ""
        q += 4
        rows = []
        while q < len(lines) and lines[q] != "":
            rows.append(lines[q])
            q += 1
        blocks.append((name, rows))
    assert q == len(lines) - 1 and lines[-1] == ""
    return lines[3], blocks


@pytest.mark.parametrize("builder", ["small_2d_mixture", "small_3d_mixture"])
def test_formatted_output_layout(builder, tmp_path):
    """outp with formatted_output: the time header, then per field its name
    and the values plane by plane, FORMAT(1x,10(1x,G14.6E3)) (io_parallel.f:
    38-50), the mixture fields last."""
    from pdac_b200 import configs
    from pdac_b200.engine import Engine
    from pdac_b200.setup_state import Case
    case = Case(getattr(configs, builder)(formatted=True))
    eng = Engine(case)
    eng.step(1)
    path = str(tmp_path / "output.0001")
    eng.write_output(path, 0.01)
    head, blocks = _formatted_blocks(open(path).read())
    assert head == " @@@ TIME = " + fortran_g(0.01, 11, 4, 2)
    st = eng.download()
    n, ns, ng = case.ncell, case.nsolid, case.ngas
    blk = lambda a, q: a[q * n:(q + 1) * n]
    want = [("P   ", st["p"]), ("UG  ", st["ug"])] + ([("VG  ", st["vg"])] if case.is3d else [])
    want += [("WG  ", st["wg"]), ("TG  ", st["tg"])]
    want += [(f"XGC{g + 1}", blk(st["xgc"], g)) for g in range(ng)]
    for q in range(ns):
        want += [(f"EPS{q + 1}", blk(st["rlk"], q) * (1.0 / case.deck["density"][q])),
                 (f" US{q + 1}", blk(st["us"], q))]
        want += [(f" VS{q + 1}", blk(st["vs"], q))] if case.is3d else []
        want += [(f" WS{q + 1}", blk(st["ws"], q)), (f" TS{q + 1}", blk(st["ts"], q))]
    mix = {k: eng.get(k) for k in ("rhom", "um", "vm", "wm", "tm", "yd") if k != "vm" or case.is3d}
    want += [("RHOM", mix["rhom"]), ("UM  ", mix["um"])] + ([("VM  ", mix["vm"])] if case.is3d else [])
    want += [("WM  ", mix["wm"]), ("TM  ", mix["tm"])]
    want += [(f"YD{q + 1}", blk(mix["yd"], q)) for q in range(ng + ns)]
    assert [b[0] for b in blocks] == [" " + w[0] for w in want]
    ntr = case.nx * (case.ny if case.is3d else 1)
    for (name, rows), (_, vals) in zip(blocks, want):
        expect = []
        for first in range(0, n, ntr):
            plane = [" " + fortran_g(v, 14, 6, 3) for v in vals[first:first + ntr]]
            chunks = ["".join(plane[r:r + 10]) for r in range(0, ntr, 10)]
            chunks[0] = " " + chunks[0]
            expect += chunks
        assert rows == expect, name
    eng.close()


def test_unformatted_output_with_mixture_fields(tmp_path):
    """The unformatted output ends with the mixture fields' REAL*4 records."""
    from pdac_b200 import configs
    from pdac_b200.engine import Engine
    from pdac_b200.setup_state import Case
    case = Case(configs.small_2d_mixture())
    eng = Engine(case)
    eng.step(1)
    path = str(tmp_path / "output.0001")
    eng.write_output(path, 0.01)
    recs = fortran_records(path)
    ns, ng = case.nsolid, case.ngas
    assert len(recs) == 1 + 4 + ng + 4 * ns + 4 + ng + ns
    n = case.ncell
    tail = [eng.get("rhom"), eng.get("um"), eng.get("wm"), eng.get("tm")]
    yd = eng.get("yd")
    tail += [yd[q * n:(q + 1) * n] for q in range(ng + ns)]
    for r, a in zip(recs[-len(tail):], tail):
        np.testing.assert_array_equal(np.frombuffer(r, dtype="<f4"), a.astype(np.float32))
    eng.close()


@pytest.mark.parametrize("formatted", [False, True])
def test_outp_recover_continues_a_run(tmp_path, formatted):
    """restart_mode = 'outp_recover' (setup.f:151-155): files.run writes
    output.0000 .. output.0002; a second run with nfil = 1 starts from the
    fields of output.0001 (outp_recover, cnvert with itd > 2) at that file's
    time, writes output.0002 next, and its steps agree with the oracle's
    from the same recovered state (same sweeps, 1e-9)."""
    import pyoracle
    from pdac_b200 import configs, files
    from pdac_b200.engine import Engine
    from pdac_b200.setup_state import Case
    d = configs.small_2d()
    dt = d["dt"]
    d.set("control", tpr=2 * dt, tdump=100 * dt, tstop=1.0, formatted_output=formatted, formatted_input=formatted)
    eng = Engine(Case(d))
    files.run(eng, str(tmp_path), max_steps=4)
    eng.close()
    d.set("control", restart_mode="outp_recover", nfil=1)
    case = Case(d)
    t_file, st = files.recover_output(case, str(tmp_path / "output.0001"))
    assert t_file == pytest.approx(2 * dt, rel=1e-6)
    eng2 = Engine(case)
    t, nfil, sweep = files.run(eng2, str(tmp_path), max_steps=2)
    assert sweep == 4 and nfil == 3
    # the same recovered state through both, two steps
    eng3 = Engine(case, upload=False)
    eng3.upload(st)
    ora = pyoracle.Oracle(case, order=pyoracle.ORDER_COLORED)
    ora.set_state(st)
    for s in (3, 4):
        assert eng3.step(s) == ora.step(s)
        errs, bad = compare_state(eng3.download(), ora.get_state(), STEP_FIELDS, 1e-9, case.nsolid, case.ncell,
                                  cells=(case.flag & 1) == 1)
        assert not bad, f"step {s}: {bad}"
    eng2.close()
    eng3.close()
