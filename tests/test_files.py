"""Host-side helpers of the time-loop files: output-file names (lettera,
letter.f:1-21), Fortran NINT (prog.f:84-86) and the test-side parsers of
Fortran records and G editing used by the GPU file tests."""
import struct

import pytest

from helpers import fortran_g, fortran_records


def test_output_names():
    from pdac_b200.files import lettera, output_name
    assert output_name(0) == "output.0000"
    assert output_name(7) == "output.0007"
    assert output_name(123) == "output.0123"
    assert lettera(9999) == "9999"
    # the reference's arithmetic past 9999: the thousands digit runs on in ASCII
    assert lettera(10000) == ":000"


def test_nint_rounds_halves_away_from_zero():
    from pdac_b200.files import nint
    assert nint(2.5) == 3 and nint(-2.5) == -3 and nint(2.4999) == 2 and nint(100.0) == 100


def test_fortran_records_round_trip(tmp_path):
    p = tmp_path / "f.bin"
    body = [b"abc", b"", struct.pack("<3d", 1.0, 2.0, 3.0)]
    with open(p, "wb") as fh:
        for b in body:
            fh.write(struct.pack("<i", len(b)) + b + struct.pack("<i", len(b)))
        # one record written as two subrecords (leading -4 / trailing 4, then 2 / -2)
        fh.write(struct.pack("<i", -4) + b"wxyz" + struct.pack("<i", 4))
        fh.write(struct.pack("<i", 2) + b"12" + struct.pack("<i", -2))
    assert fortran_records(str(p)) == body + [b"wxyz12"]


@pytest.mark.parametrize("x,want", [
    (1234.5, "    1234.5000000000000000     "),
    (0.0, "    0.0000000000000000000     "),
    (1.5e-3, "   0.15000000000000000312E-002"),
    (-3.2e-7, "  -0.32000000000000000670E-006"),
    (1e20, "   0.10000000000000000000E+021"),
])
def test_fortran_g_rules(x, want):
    """G30.20E3: F form with 20 significant digits and 5 trailing blanks
    for 0.1 <= |x| < 1e20, E form otherwise (F2008 10.7.5.2.2)."""
    assert fortran_g(x) == want
