"""Python binding of the CUDA engine (ctypes over include/pdac_gpu.h).

:class:`Engine` mirrors the reference's time-loop calls (prog.f:143-417):
``boundary``, ``fieldn``, ``tilde``, ``iter``, ``ygas``, ``htilde``,
``ftem`` and the fused ``step``.  There is no CPU fallback: if the CUDA
library is missing or no GPU is visible, construction raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libpdac_b200.so")

_lib = None


class PdacError(RuntimeError):
    def __init__(self, status, where, detail=""):
        self.status = status
        name = abi.STATUS_NAMES.get(status, str(status))
        super().__init__(f"{where}: {name}" + (f" ({detail})" if detail else ""))


def lib():
    """Load libpdac_b200.so (built in-tree by pdac_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"CUDA engine library not built: {LIB_PATH} (run python -m pdac_b200.build)")
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.pdac_gpu_create.argtypes = [C.POINTER(abi.PdacCfg), C.POINTER(P)]
        L.pdac_gpu_create.restype = C.c_int
        L.pdac_gpu_destroy.argtypes = [P]
        L.pdac_gpu_destroy.restype = C.c_int
        L.pdac_gpu_last_error.argtypes = [P]
        L.pdac_gpu_last_error.restype = C.c_char_p
        L.pdac_gpu_upload_state.argtypes = [P, C.POINTER(abi.PdacStateView)]
        L.pdac_gpu_upload_state.restype = C.c_int
        L.pdac_gpu_download_state.argtypes = [P, C.POINTER(abi.PdacStateView)]
        L.pdac_gpu_download_state.restype = C.c_int
        L.pdac_gpu_exchange_state.argtypes = [P, C.POINTER(abi.PdacStateView), C.POINTER(abi.PdacStateView)]
        L.pdac_gpu_exchange_state.restype = C.c_int
        L.pdac_gpu_phase_times.argtypes = [P, C.POINTER(C.c_double)]
        L.pdac_gpu_phase_times.restype = C.c_int
        L.pdac_gpu_set_vent_factors.argtypes = [P, C.POINTER(C.c_double), C.c_int]
        L.pdac_gpu_set_vent_factors.restype = C.c_int
        L.pdac_gpu_stats.argtypes = [P, C.POINTER(C.c_double), C.c_int]
        L.pdac_gpu_stats.restype = C.c_int
        L.pdac_gpu_reset_stats.argtypes = [P, C.c_int]
        L.pdac_gpu_reset_stats.restype = C.c_int
        L.pdac_gpu_mark.argtypes = [P, C.c_int]
        L.pdac_gpu_mark.restype = C.c_int
        L.pdac_gpu_elapsed.argtypes = [P, C.c_int, C.c_int, C.POINTER(C.c_double)]
        L.pdac_gpu_elapsed.restype = C.c_int
        abi.declare(L, "pdac_gpu", P)
        _lib = L
    return _lib


EXPORTED = (
    "pdac_gpu_create", "pdac_gpu_destroy", "pdac_gpu_last_error", "pdac_gpu_upload_state",
    "pdac_gpu_download_state", "pdac_gpu_exchange_state", "pdac_gpu_boundary", "pdac_gpu_fieldn", "pdac_gpu_tilde", "pdac_gpu_iter",
    "pdac_gpu_initialize_fieldn", "pdac_gpu_explicit_iter", "pdac_gpu_sgsg", "pdac_gpu_sgss",
    "pdac_gpu_ygas", "pdac_gpu_htilde", "pdac_gpu_ftem", "pdac_gpu_step", "pdac_gpu_set_vent_factors",
    "pdac_gpu_get_array", "pdac_gpu_mass_totals", "pdac_gpu_phase_times", "pdac_gpu_stats",
    "pdac_gpu_reset_stats", "pdac_gpu_mark", "pdac_gpu_elapsed",
    "pdac_gpu_write_restart", "pdac_gpu_read_restart", "pdac_gpu_write_output", "pdac_gpu_mass_residuals",
    "pdac_gpu_append_mass_check", "pdac_gpu_write_mass_loss", "pdac_gpu_read_mass_loss",
    "pdac_gpu_compute_mixture_fields", "pdac_gpu_batch_create", "pdac_gpu_batch_step", "pdac_gpu_batch_elapsed",
    "pdac_gpu_batch_last_error", "pdac_gpu_batch_destroy", "pdac_gpu_unconverged_cells",
    "pdac_gpu_autotune", "pdac_gpu_set_tuning",
)

# the launch shapes pdac_gpu_autotune / pdac_gpu_set_tuning exchange, in order
TUNING_KEYS = ("tile_shape", "tile_kchunk", "inner_grid", "test_grid", "coop_cells_per_block")


class Engine:
    """One device-resident domain set up from a :class:`~pdac_b200.setup_state.Case`."""

    def __init__(self, case, upload=True):
        self.case = case
        self.L = lib()
        self._cfg = case.cfg()
        self.h = C.c_void_p()
        st = self.L.pdac_gpu_create(C.byref(self._cfg), C.byref(self.h))
        if st != 0:
            raise PdacError(st, "pdac_gpu_create")
        self.sweep = 0
        if upload:
            self.upload(case.state)

    def close(self):
        if getattr(self, "h", None):
            self.L.pdac_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, st, where):
        if st != 0:
            raise PdacError(st, where, (self.L.pdac_gpu_last_error(self.h) or b"").decode())

    # ---- state -----------------------------------------------------------
    def upload(self, state):
        self._up = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in state.items()}
        view = abi.make_state_view(self._up)
        self._chk(self.L.pdac_gpu_upload_state(self.h, C.byref(view)), "upload_state")

    def download(self):
        out = {k: np.zeros_like(v) for k, v in self.case.state.items()}
        view = abi.make_state_view(out)
        self._chk(self.L.pdac_gpu_download_state(self.h, C.byref(view)), "download_state")
        return out

    def get(self, name):
        n = C.c_long(0)
        self.L.pdac_gpu_get_array(self.h, name.encode(), abi.dptr(None), C.byref(n))
        if n.value <= 0:
            raise KeyError(name)
        buf = np.zeros(n.value)
        self._chk(self.L.pdac_gpu_get_array(self.h, name.encode(), abi.dptr(buf), C.byref(n)), f"get_array({name})")
        return buf

    # ---- time-loop calls ---------------------------------------------------
    def boundary(self, sweep):
        self._chk(self.L.pdac_gpu_boundary(self.h, sweep), "boundary")

    def fieldn(self):
        self._chk(self.L.pdac_gpu_fieldn(self.h), "fieldn")

    def sgsg(self):
        """The sub-grid turbulence model after fieldn (prog.f:207)."""
        self._chk(self.L.pdac_gpu_sgsg(self.h), "sgsg")

    def sgss(self):
        """The particle sub-grid stress after fieldn (prog.f:208)."""
        self._chk(self.L.pdac_gpu_sgss(self.h), "sgss")

    def initialize_fieldn(self):
        self._chk(self.L.pdac_gpu_initialize_fieldn(self.h), "initialize_fieldn")

    def explicit_iter(self, dt):
        self._chk(self.L.pdac_gpu_explicit_iter(self.h, dt), "explicit_iter")

    def tilde(self, dt):
        self._chk(self.L.pdac_gpu_tilde(self.h, dt), "tilde")

    def iter(self, dt):
        nit = C.c_int(0)
        self._chk(self.L.pdac_gpu_iter(self.h, dt, C.byref(nit)), "iter")
        return nit.value

    def unconverged_cells(self):
        """Flat indices of the cells the last iter's last sweep did not
        converge (the reference's report at maxout, iter.f:428-447)."""
        L = self.L
        L.pdac_gpu_unconverged_cells.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_long)]
        L.pdac_gpu_unconverged_cells.restype = C.c_int
        n = C.c_long(0)
        L.pdac_gpu_unconverged_cells(self.h, None, C.byref(n))
        buf = np.zeros(max(n.value, 1), dtype=np.int32)
        self._chk(L.pdac_gpu_unconverged_cells(self.h, buf.ctypes.data_as(C.POINTER(C.c_int)), C.byref(n)),
                  "unconverged_cells")
        return buf[:n.value].copy()

    def autotune(self, cache_path=None):
        """Time the tunable launch shapes on the current state and keep the
        fastest (pdac_gpu_autotune); returns them as a dict."""
        L = self.L
        L.pdac_gpu_autotune.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_int), C.c_int]
        L.pdac_gpu_autotune.restype = C.c_int
        out = (C.c_int * len(TUNING_KEYS))()
        path = os.fsencode(cache_path) if cache_path is not None else None
        self._chk(L.pdac_gpu_autotune(self.h, path, out, len(TUNING_KEYS)), "autotune")
        return dict(zip(TUNING_KEYS, list(out)))

    def set_tuning(self, tuning):
        """Install launch shapes (a dict with TUNING_KEYS)."""
        L = self.L
        L.pdac_gpu_set_tuning.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.c_int]
        L.pdac_gpu_set_tuning.restype = C.c_int
        arr = (C.c_int * len(TUNING_KEYS))(*[int(tuning[k]) for k in TUNING_KEYS])
        self._chk(L.pdac_gpu_set_tuning(self.h, arr, len(TUNING_KEYS)), "set_tuning")

    def ygas(self, dt):
        self._chk(self.L.pdac_gpu_ygas(self.h, dt), "ygas")

    def htilde(self, dt):
        self._chk(self.L.pdac_gpu_htilde(self.h, dt), "htilde")

    def ftem(self, dt):
        self._chk(self.L.pdac_gpu_ftem(self.h, dt), "ftem")

    def step(self, sweep=None):
        if sweep is None:
            sweep = self.sweep + 1
        self.sweep = sweep
        nit = C.c_int(0)
        self._chk(self.L.pdac_gpu_step(self.h, sweep, C.byref(nit)), "step")
        return nit.value

    # ---- files of the time loop (pdac.res, output.NNNN, pdac.chm) --------
    def write_restart(self, path, time, nfil):
        """tapewr: the restart file in the reference's record layout."""
        self._chk(self.L.pdac_gpu_write_restart(self.h, os.fsencode(path), float(time), int(nfil)), "write_restart")

    def read_restart(self, path):
        """taperd + cnvert: load a restart file; returns (time, nfil)."""
        t = C.c_double(0)
        nf = C.c_int(0)
        self._chk(self.L.pdac_gpu_read_restart(self.h, os.fsencode(path), C.byref(t), C.byref(nf)), "read_restart")
        return t.value, nf.value

    def write_output(self, path, time):
        """outp (unformatted form) into path, e.g. output_name(nfil)."""
        self._chk(self.L.pdac_gpu_write_output(self.h, os.fsencode(path), float(time)), "write_output")

    def mass_residuals(self, nswp, dt=None):
        """print_mass_residuals values: dict res_g, res_s, res_gc, mfr."""
        n = 2 + self.case.nsolid + self.case.ngas
        out = np.zeros(n)
        dt = self.case.deck["dt"] if dt is None else dt
        self._chk(self.L.pdac_gpu_mass_residuals(self.h, int(nswp), float(dt), abi.dptr(out), n), "mass_residuals")
        ns = self.case.nsolid
        return dict(res_g=out[0], res_s=out[1:1 + ns], res_gc=out[1 + ns:-1], mfr=out[-1])

    def append_mass_check(self, path, nswp, dt=None):
        """Append the pdac.chm line of step nswp to path."""
        dt = self.case.deck["dt"] if dt is None else dt
        self._chk(self.L.pdac_gpu_append_mass_check(self.h, os.fsencode(path), int(nswp), float(dt)), "append_mass_check")

    def compute_mixture_fields(self):
        """compute_mixture_fields (prog.f:331): rhom, um, vm, wm, tm, yd."""
        self._chk(self.L.pdac_gpu_compute_mixture_fields(self.h), "compute_mixture_fields")

    def write_mass_loss(self, path):
        """print_mass_loss: the ground columns' lost mass (massl.NNNN / massl.res)."""
        self._chk(self.L.pdac_gpu_write_mass_loss(self.h, os.fsencode(path)), "write_mass_loss")

    def read_mass_loss(self, path):
        """read_mass_loss: values added back at each column's next sink update."""
        self._chk(self.L.pdac_gpu_read_mass_loss(self.h, os.fsencode(path)), "read_mass_loss")

    def set_vent_factors(self, fact):
        fact = np.ascontiguousarray(fact, dtype=np.float64)
        self._chk(self.L.pdac_gpu_set_vent_factors(self.h, abi.dptr(fact), len(fact)), "set_vent_factors")

    def mass_totals(self):
        n = 1 + self.case.nsolid + self.case.ngas
        out = np.zeros(n)
        self._chk(self.L.pdac_gpu_mass_totals(self.h, abi.dptr(out), n), "mass_totals")
        return out

    def stats(self):
        out = (C.c_double * 13)()
        self._chk(self.L.pdac_gpu_stats(self.h, out, 13), "stats")
        return dict(launches=int(out[0]), sweeps=int(out[1]), corr_launches=int(out[2]), corr_ms=out[3],
                    resid_ms=out[4], inner_ms=out[5], work_cells=int(out[6]), tested_cells=int(out[7]),
                    rk3_ms={"flux": out[8], "stage": out[9], "wave": out[10], "final": out[11]},
                    rk3_calls=int(out[12]))

    def sweep_log(self):
        """Per colour phase since the last profiling reset: array of rows
        (sweep, colour, worklist, tested, resid_ms, inner_ms)."""
        L = self.L
        L.pdac_gpu_sweep_log.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_long)]
        L.pdac_gpu_sweep_log.restype = C.c_int
        n = C.c_long(0)
        L.pdac_gpu_sweep_log(self.h, None, C.byref(n))
        buf = np.zeros(max(n.value, 1))
        self._chk(L.pdac_gpu_sweep_log(self.h, buf.ctypes.data_as(C.POINTER(C.c_double)), C.byref(n)), "sweep_log")
        return buf[:n.value].reshape(-1, 6)

    def reset_stats(self, profile_corrector=False):
        self._chk(self.L.pdac_gpu_reset_stats(self.h, int(profile_corrector)), "reset_stats")

    def mark(self, slot):
        self._chk(self.L.pdac_gpu_mark(self.h, slot), "mark")

    def elapsed(self, a, b):
        ms = C.c_double(0)
        self._chk(self.L.pdac_gpu_elapsed(self.h, a, b, C.byref(ms)), "elapsed")
        return ms.value

    def phase_times(self):
        out = (C.c_double * 7)()
        self._chk(self.L.pdac_gpu_phase_times(self.h, out), "phase_times")
        return dict(zip(("boundary", "fieldn", "tilde", "iter", "ygas", "htilde", "ftem"), list(out)))
