"""ctypes driver for the CPU FP64 oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU arms import this
module; the product package never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from pdac_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libpdac_oracle.so")

ORDER_COLORED = 0
ORDER_LEXICOGRAPHIC = 1

_lib = None


def build(force=False):
    """Compile the oracle with its Makefile (g++ only; seconds)."""
    srcs = ("pdac_oracle.cpp", "pdac_oracle3d.inc", "pdac_oracle_rk3.inc", "pdac_oracle_les.inc", "pdac_oracle_ib.inc",
            "../pdac_b200/csrc/fpmath.h", "../pdac_b200/csrc/fpmath_tables.h")
    if force or not os.path.exists(LIB_PATH) or \
            os.path.getmtime(LIB_PATH) < max(os.path.getmtime(os.path.join(HERE, f)) for f in srcs):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        L.pdac_oracle_create.argtypes = [C.POINTER(abi.PdacCfg), C.POINTER(C.c_void_p)]
        L.pdac_oracle_create.restype = C.c_int
        L.pdac_oracle_destroy.argtypes = [C.c_void_p]
        L.pdac_oracle_set_order.argtypes = [C.c_void_p, C.c_int]
        L.pdac_oracle_set_state.argtypes = [C.c_void_p, C.POINTER(abi.PdacStateView)]
        L.pdac_oracle_get_state.argtypes = [C.c_void_p, C.POINTER(abi.PdacStateView)]
        L.pdac_oracle_set_vent_factors.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.c_int]
        L.pdac_oracle_last_nit.argtypes = [C.c_void_p]
        L.pdac_oracle_eos_fail.argtypes = [C.c_void_p]
        L.pdac_oracle_limiter.argtypes = [C.c_int, C.c_double, C.c_double]
        L.pdac_oracle_limiter.restype = C.c_double
        abi.declare(L, "pdac_oracle", C.c_void_p)
        _lib = L
    return _lib


class Oracle:
    """One oracle context over a :class:`pdac_b200.setup_state.Case`."""

    def __init__(self, case, order=ORDER_COLORED):
        self.case = case
        self.L = lib()
        self._cfg = case.cfg()
        self.h = C.c_void_p()
        st = self.L.pdac_oracle_create(C.byref(self._cfg), C.byref(self.h))
        if st != 0:
            raise RuntimeError(f"pdac_oracle_create failed: {abi.STATUS_NAMES.get(st, st)}")
        self.L.pdac_oracle_set_order(self.h, order)
        self.set_state(case.state)

    def __del__(self):
        try:
            if self.h:
                self.L.pdac_oracle_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def set_state(self, state):
        self._in = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in state.items()}
        view = abi.make_state_view(self._in)
        self.L.pdac_oracle_set_state(self.h, C.byref(view))

    def get_state(self):
        out = {k: np.zeros_like(v) for k, v in self.case.state.items()}
        view = abi.make_state_view(out)
        self.L.pdac_oracle_get_state(self.h, C.byref(view))
        return out

    def get(self, name):
        n = C.c_long(0)
        buf = np.zeros(1)
        self.L.pdac_oracle_get_array(self.h, name.encode(), abi.dptr(buf), C.byref(n))
        buf = np.zeros(n.value)
        st = self.L.pdac_oracle_get_array(self.h, name.encode(), abi.dptr(buf), C.byref(n))
        if st != 0:
            raise KeyError(name)
        return buf

    def _chk(self, st, what):
        if st != 0:
            raise RuntimeError(f"oracle {what}: {abi.STATUS_NAMES.get(st, st)}")

    def boundary(self, sweep):
        self._chk(self.L.pdac_oracle_boundary(self.h, sweep), "boundary")

    def fieldn(self):
        self._chk(self.L.pdac_oracle_fieldn(self.h), "fieldn")

    def tilde(self, dt):
        self._chk(self.L.pdac_oracle_tilde(self.h, dt), "tilde")

    def iter(self, dt):
        nit = C.c_int(0)
        self._chk(self.L.pdac_oracle_iter(self.h, dt, C.byref(nit)), "iter")
        return nit.value

    def ygas(self, dt):
        self._chk(self.L.pdac_oracle_ygas(self.h, dt), "ygas")

    def htilde(self, dt):
        self._chk(self.L.pdac_oracle_htilde(self.h, dt), "htilde")

    def ftem(self, dt):
        self._chk(self.L.pdac_oracle_ftem(self.h, dt), "ftem")

    def sgs(self):
        """sgsg and sgss as prog.f:207-208 call them after fieldn."""
        self._chk(self.L.pdac_oracle_sgs(self.h), "sgs")

    def initialize_fieldn(self):
        self._chk(self.L.pdac_oracle_initialize_fieldn(self.h), "initialize_fieldn")

    def explicit_iter(self, dt):
        self._chk(self.L.pdac_oracle_explicit_iter(self.h, dt), "explicit_iter")

    def step(self, sweep):
        nit = C.c_int(0)
        self._chk(self.L.pdac_oracle_step(self.h, sweep, C.byref(nit)), "step")
        return nit.value

    def unconverged_cells(self):
        """Cells of the last iter's last sweep that ran the inner loop."""
        L = self.L
        L.pdac_oracle_unconverged_cells.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_long)]
        L.pdac_oracle_unconverged_cells.restype = C.c_int
        n = C.c_long(0)
        L.pdac_oracle_unconverged_cells(self.h, None, C.byref(n))
        buf = np.zeros(max(n.value, 1), dtype=np.int32)
        self._chk(L.pdac_oracle_unconverged_cells(self.h, buf.ctypes.data_as(C.POINTER(C.c_int)), C.byref(n)),
                  "unconverged_cells")
        return buf[:n.value].copy()

    def mass_totals(self):
        n = 1 + self.case.nsolid + self.case.ngas
        out = np.zeros(n)
        self._chk(self.L.pdac_oracle_mass_totals(self.h, abi.dptr(out), n), "mass_totals")
        return out


def set_threads(n):
    """Threads of the oracle's 3D cell loops in this process; returns the
    count in use (the results are the same bits on any count)."""
    L = lib()
    L.pdac_oracle_set_threads.argtypes = [C.c_int]
    L.pdac_oracle_set_threads.restype = C.c_int
    return L.pdac_oracle_set_threads(int(n))


def limiter(lim_type, erre, beta=0.25):
    return lib().pdac_oracle_limiter(lim_type, erre, beta)
