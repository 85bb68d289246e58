"""restart_mode = 'outp_recover': the state rebuilt from an output file
(outp_recover, io_restart.f:341-493, and cnvert with itd > 2, setup.f:
393-440), on the CPU from output files written here in the reference's
two layouts (one REAL*4 record per field after REAL(time, 4); or the
formatted layout of outp with FORMAT(1x,10(1x,G14.6E3)) rows).
"""
import struct

import numpy as np
import pytest

from helpers import fortran_g


def _case(is3d, formatted=False):
    from pdac_b200 import configs
    from pdac_b200.setup_state import Case
    d = configs.small_3d() if is3d else configs.small_2d()
    d.set("control", formatted_input=formatted)
    return Case(d)


def _written_fields(case):
    """The fields outp writes, in order, from the case's initial state with
    its gas velocity and temperature perturbed so every field differs."""
    st = case.state
    n, ns, ng = case.ncell, case.nsolid, case.ngas
    rng = np.random.default_rng(7)
    p = st["p"] * (1.0 + 0.01 * rng.random(n))
    out = [p, st["ug"] + rng.random(n), ] + ([st["vg"] + rng.random(n)] if case.is3d else [])
    out += [st["wg"] + rng.random(n), st["tg"] + 50.0 * rng.random(n)]
    out += [st["xgc"][g * n:(g + 1) * n] for g in range(ng)]
    rl = case.deck["density"]
    for s in range(ns):
        blk = slice(s * n, (s + 1) * n)
        out += [st["rlk"][blk] / rl[s], st["us"][blk] + rng.random(n)]
        out += [st["vs"][blk]] if case.is3d else []
        out += [st["ws"][blk] - rng.random(n), st["ts"][blk] + 10.0 * rng.random(n)]
    return out


def _record(b):
    return struct.pack("<i", len(b)) + b + struct.pack("<i", len(b))


def _write_unformatted(path, time, fields):
    with open(path, "wb") as f:
        f.write(_record(np.float32(time).tobytes()))
        for a in fields:
            f.write(_record(np.asarray(a, dtype="<f4").tobytes()))
        f.write(_record(np.zeros(len(fields[0]), dtype="<f4").tobytes()))  # a mixture field, not read


def _write_formatted(path, time, fields, nplane):
    lines = ["", "", "", " @@@ TIME = " + fortran_g(time, 11, 4, 2)]
    for q, a in enumerate(fields):
        lines += ["", "", f" F{q:03d}", ""]
        for first in range(0, len(a), nplane):
            row = [" " + fortran_g(v, 14, 6, 3) for v in a[first:first + nplane]]
            chunks = ["".join(row[r:r + 10]) for r in range(0, len(row), 10)]
            chunks[0] = " " + chunks[0]
            lines += chunks
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def _check(case, time, st, want_time, fields, tol):
    from pdac_b200.setup_state import GMW, hcapg, mas, thermal_eosg
    n, ns, ng = case.ncell, case.nsolid, case.ngas
    assert time == pytest.approx(want_time, rel=1e-6)
    names = ["p", "ug"] + (["vg"] if case.is3d else []) + ["wg", "tg"]
    got = [st[k] for k in names] + [st["xgc"][g * n:(g + 1) * n] for g in range(ng)]
    rl = case.deck["density"]
    for s in range(ns):
        blk = slice(s * n, (s + 1) * n)
        got += [st["rlk"][blk] / rl[s], st["us"][blk]] + ([st["vs"][blk]] if case.is3d else [])
        got += [st["ws"][blk], st["ts"][blk]]
    for q, (a, b) in enumerate(zip(got, fields)):
        assert np.allclose(a, b, rtol=tol, atol=tol * np.max(np.abs(b))), q
    X = st["xgc"].reshape(ng, n)
    assert np.array_equal(st["ygc"].reshape(ng, n), mas(X, case.gas_type))
    ep = np.ones(n)  # ep = 1, then one class subtracted after the other (setup.f:407-410)
    for s in range(ns):
        ep = ep - st["rlk"][s * n:(s + 1) * n] * (1.0 / rl[s])
    assert np.array_equal(st["ep"], ep)
    rog = thermal_eosg(st["tg"], st["p"], X, case.gas_type)
    assert np.array_equal(st["rog"], rog) and np.array_equal(st["rgp"], rog * ep)
    cp = hcapg(st["tg"], case.deck["icpc"], case.deck["tref"])
    cg = sum(cp[gt - 1] * st["ygc"][g * n:(g + 1) * n] for g, gt in enumerate(case.gas_type))
    assert np.allclose(st["cg"], cg, rtol=1e-15) and np.array_equal(st["sieg"], st["tg"] * st["cg"])


@pytest.mark.parametrize("is3d", [False, True])
def test_recover_unformatted(tmp_path, is3d):
    from pdac_b200 import files
    case = _case(is3d)
    fields = _written_fields(case)
    path = str(tmp_path / "output.0003")
    _write_unformatted(path, 1.25, fields)
    t, st = files.recover_output(case, path)
    # REAL*4 in the file: each value is the nearest single
    f32 = [np.asarray(a, dtype=np.float32).astype(np.float64) for a in fields]
    _check(case, t, st, 1.25, f32, 0.0)


@pytest.mark.parametrize("is3d", [False, True])
def test_recover_formatted(tmp_path, is3d):
    from pdac_b200 import files
    case = _case(is3d, formatted=True)
    fields = _written_fields(case)
    path = str(tmp_path / "output.0003")
    _write_formatted(path, 1.25, fields, case.nx * (case.ny if case.is3d else 1))
    t, st = files.recover_output(case, path)
    # six significant digits in the file: half a unit of the sixth
    _check(case, t, st, 1.25, fields, 5e-6)


def test_mas_inverts_mole():
    from pdac_b200.setup_state import mas, mole
    y = np.array([[0.2, 1.0, 0.0], [0.8, 0.0, 1.0]])
    assert np.allclose(mas(mole(y, [6, 5]), [6, 5]), y, rtol=1e-15, atol=0.0)
