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


def compare_state(got, ref, names, tol, nsolid, ncell, rlk_min=1e-5):
    """Relative L-inf per field; particle temperature/enthalpy (ts, sies) are
    compared only where the class is present (rlk > rlk_min): where it is
    absent, invdm (ftem.f:221-226) decouples the class below flim and its
    temperature is not defined by the solve."""
    errs = {}
    for n in names:
        a, b = np.asarray(got[n]), np.asarray(ref[n])
        if n in ("ts", "sies"):
            mask = (np.asarray(ref["rlk"]) > rlk_min) & (np.asarray(got["rlk"]) > rlk_min)
            a, b = a[mask], b[mask]
        errs[n] = rel_linf(a, b)
    bad = {n: e for n, e in errs.items() if not (e <= tol)}
    return errs, bad
