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


def compare_state(got, ref, names, tol, nsolid, ncell, rlk_min=1e-5, cells=None):
    """Relative L-inf per field; particle temperature/enthalpy (ts, sies) are
    compared only where the class is present (rlk > rlk_min): where it is
    absent, invdm (ftem.f:221-226) decouples the class below flim and its
    temperature is not defined by the solve."""
    errs = {}
    for n in names:
        a, b = np.asarray(got[n]), np.asarray(ref[n])
        nb = a.size // ncell
        sel = np.ones(a.size, dtype=bool)
        if cells is not None:
            sel &= np.tile(np.asarray(cells, dtype=bool), nb)
        if n in ("ts", "sies"):
            sel &= (np.asarray(ref["rlk"]) > rlk_min) & (np.asarray(got["rlk"]) > rlk_min)
        a, b = a[sel], b[sel]
        errs[n] = rel_linf(a, b)
    bad = {n: e for n, e in errs.items() if not (e <= tol)}
    return errs, bad


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
