"""The compiled time-loop driver (pdac_b200/host/pdac_run.cpp) without a
GPU: it builds against the engine library, reports its usage and rejects
files that are not case files; the case file holds what the format says."""
import os
import struct
import subprocess

import pytest


def _driver():
    from pdac_b200 import build
    build.build()
    return build.build_host()


def test_driver_builds_and_reports_usage():
    exe = _driver()
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 2 and "usage: pdac_run CASEFILE WORKDIR" in r.stderr


def test_driver_rejects_a_file_that_is_not_a_case(tmp_path):
    exe = _driver()
    bad = tmp_path / "x.bin"
    bad.write_bytes(b"NOTACASE" + b"\0" * 64)
    r = subprocess.run([exe, str(bad), str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 2 and "not a case file" in r.stderr
    trunc = tmp_path / "t.bin"
    trunc.write_bytes(b"PDACCAS1" + b"\0" * 16)
    r = subprocess.run([exe, str(trunc), str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 2 and "truncated" in r.stderr


@pytest.mark.parametrize("builder", ["small_2d", "small_3d"])
def test_case_file_layout(builder, tmp_path):
    from pdac_b200 import casefile, configs
    from pdac_b200.setup_state import Case
    d = getattr(configs, builder)()
    d.set("control", tpr=0.02, tdump=0.04, imr=1)
    case = Case(d)
    path = casefile.write(case, str(tmp_path / "case.bin"))
    raw = open(path, "rb").read()
    n, ns, ng = case.ncell, case.nsolid, case.ngas
    nstate = (10 - (0 if case.is3d else 1)) * n + (6 - (0 if case.is3d else 1)) * ns * n + 2 * ng * n
    size = (8 + casefile.cfg_size() + struct.calcsize(casefile.CONTROL) + 8 * (case.nx + case.nz)
            + (8 * case.ny if case.is3d else 0) + 4 * n + 16 * case.nz + 4 * len(case.vent) + 8 * nstate)
    assert len(raw) == size
    off = 8 + casefile.cfg_size()
    tstop, tpr, tdump, maxs, imr, nfil, restart, isink, mix = struct.unpack_from(casefile.CONTROL, raw, off)
    assert (tpr, tdump, imr, restart) == (0.02, 0.04, 1, 0)
