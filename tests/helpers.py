"""Shared helpers of the test suite: field comparison with stated tolerances."""
import numpy as np

# fields compared after a time step and their role
STEP_FIELDS = ("p", "ep", "rog", "rgp", "tg", "sieg", "cg", "ug", "wg",
               "rlk", "ts", "sies", "us", "ws", "ygc", "xgc")


def rel_linf(a, b):
    """max |a - b| / max |b|  (relative L-infinity against the field scale)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.max(np.abs(b)) if b.size else 0.0
    if scale == 0.0:
        return float(np.max(np.abs(a))) if a.size else 0.0
    return float(np.max(np.abs(a - b)) / scale)


def compare_fields(got, ref, names, tol):
    errs = {n: rel_linf(got[n], ref[n]) for n in names}
    bad = {n: e for n, e in errs.items() if not (e <= tol)}
    return errs, bad


def compare_state(got, ref, names, tol, nsolid, ncell, rlk_min=1e-5, cells=None, dilute=("ts", "sies")):
    """Relative L-inf per field; the fields named in `dilute` (by default the
    particle temperature and enthalpy) are compared only where the class is
    present (rlk > rlk_min): where it is absent, invdm (ftem.f:221-226)
    decouples the class below flim and its temperature is not defined by the
    solve."""
    errs = {}
    for n in names:
        a, b = np.asarray(got[n]), np.asarray(ref[n])
        nb = a.size // ncell
        sel = np.ones(a.size, dtype=bool)
        if cells is not None:
            sel &= np.tile(np.asarray(cells, dtype=bool), nb)
        if n in dilute:
            sel &= (np.asarray(ref["rlk"]) > rlk_min) & (np.asarray(got["rlk"]) > rlk_min)
        a, b = a[sel], b[sel]
        errs[n] = rel_linf(a, b)
    bad = {n: e for n, e in errs.items() if not (e <= tol)}
    return errs, bad


def frame_mismatches(got, ref, names, case, tol, rlk_min=1e-5, round_off=1e-9):
    """Boundary-frame (non-fluid) values that differ by more than tol times
    the field's scale, cell by cell, except where the rule of the free
    in/outflow boundaries allows it.

    inoutflow (inoutflow.f:64-99) fills a free in/outflow ghost cell with the
    atmosphere or with the interior values according to the sign of the
    boundary-normal velocity on its face.  Where that velocity is at
    round-off level (within round_off of the velocity field's scale in both
    states; in the workloads it is ~1e-37 m/s against tens of m/s) the two
    implementations may pick different branches, as the reference's own
    choice depends on round-off there.  Such a cell is exempt; every other
    frame value is compared.  Particle temperature and enthalpy are compared
    where the class is present, as in compare_state.

    Returns (mismatches, exempt): lists of (field, class, cell, rel. error)."""
    flag = np.asarray(case.flag)
    n, nx, ny, nz = case.ncell, case.nx, case.ny, case.nz
    frame = (flag & 1) == 0
    i = np.arange(n) % nx + 1
    j = (np.arange(n) // nx) % ny + 1
    k = np.arange(n) // (nx * ny) + 1
    # the boundary face of each frame cell and the velocity normal to it
    faces = [("ug", i == nx, -1), ("ug", i == 1, 0), ("wg", k == nz, -nx * ny), ("wg", k == 1, 0)]
    if case.is3d:
        faces += [("vg", j == ny, -nx), ("vg", j == 1, 0)]
    near_zero = np.zeros(n, dtype=bool)
    free_io = flag == 8  # the only ghost cells whose fill depends on the sign of u_n
    for name, on, shift in faces:
        idx = np.flatnonzero(on & free_io)
        face = idx + shift
        for st in (got, ref):
            u = np.asarray(st[name])
            scale = max(np.max(np.abs(u)), 1e-300)
            near_zero[idx] |= np.abs(u[face]) <= round_off * scale
    bad, exempt = [], []
    for nm in names:
        a, b = np.asarray(got[nm]), np.asarray(ref[nm])
        nb = a.size // n
        scale = max(np.max(np.abs(b)), 1e-300)
        for q in range(nb):
            aa, bb = a[q * n:(q + 1) * n], b[q * n:(q + 1) * n]
            sel = frame.copy()
            if nm in ("ts", "sies"):
                sel &= (np.asarray(ref["rlk"])[q * n:(q + 1) * n] > rlk_min) & \
                       (np.asarray(got["rlk"])[q * n:(q + 1) * n] > rlk_min)
            d = np.abs(aa - bb) / scale
            for c in np.flatnonzero(sel & (d > tol)):
                (exempt if near_zero[c] else bad).append((nm, q, int(c), float(d[c])))
    return bad, exempt


def frame_agreement(got, ref, names, ncell, fluid, tol=1e-9):
    """Fraction of boundary-frame (non-fluid) cell values that agree to tol.

    Ghost cells of free in/outflow boundaries switch between copying the
    interior and the atmosphere on the sign of the boundary-normal velocity
    (inoutflow.f:64-99); where that velocity is at round-off level the two
    implementations may pick differently, as the reference's own result
    depends on round-off there."""
    tot = ok = 0
    for n in names:
        a, b = np.asarray(got[n]), np.asarray(ref[n])
        nb = a.size // ncell
        m = np.tile(~np.asarray(fluid, dtype=bool), nb)
        scale = max(np.max(np.abs(b)), 1e-300)
        d = np.abs(a[m] - b[m]) / scale
        tot += d.size
        ok += int(np.count_nonzero(d <= tol))
    return ok / max(tot, 1)


def fortran_records(path):
    """The records of a Fortran unformatted sequential file, as bytes:
    4-byte little-endian length markers around each record; a negative
    leading marker continues the record in the next subrecord."""
    import struct
    data = open(path, "rb").read()
    out, pos, cur = [], 0, b""
    while pos < len(data):
        (m1,) = struct.unpack_from("<i", data, pos)
        n = abs(m1)
        body = data[pos + 4:pos + 4 + n]
        (m2,) = struct.unpack_from("<i", data, pos + 4 + n)
        assert abs(m2) == n, "record framing"
        pos += 8 + n
        cur += body
        if m1 >= 0:
            out.append(cur)
            cur = b""
    assert cur == b"", "unterminated record"
    return out


def fortran_g(x, w=30, d=20, e=3):
    """Fortran Gw.dEe output of one value (F2008 10.7.5.2.2), written out
    with Python's decimal rounding of the exact binary value."""
    from decimal import Decimal, ROUND_HALF_EVEN
    n = e + 2
    if x == 0.0:
        return f"{x:{w - n}.{d - 1}f}" + " " * n
    dec = Decimal(x)
    ex = dec.adjusted()  # exponent of the leading digit before rounding
    q = dec.scaleb(-ex).quantize(Decimal(1).scaleb(-(d - 1)), rounding=ROUND_HALF_EVEN)
    if abs(q) >= 10:
        ex += 1
    s = ex + 1
    if 0 <= s <= d:
        return f"{x:{w - n}.{d - s}f}" + " " * n
    digits = format(abs(dec).scaleb(-ex).quantize(Decimal(1).scaleb(-(d - 1)), rounding=ROUND_HALF_EVEN), "f").replace(".", "")[:d]
    if abs(q) >= 10:
        digits = "1" + "0" * (d - 1)
    body = ("-" if x < 0 else "") + "0." + digits + "E" + ("-" if s < 0 else "+") + f"{abs(s):0{e}d}"
    return f"{body:>{w}}"
