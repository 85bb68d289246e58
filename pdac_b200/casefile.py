"""The case file: a set-up run handed to a compiled host program.

The input side of PDAC (namelists, atmosphere, mesh, vent, initial state:
input.f, setup.f, atmosphere.f, grid.f, vent.f) is restated in Python
(:mod:`pdac_b200.deck`, :mod:`pdac_b200.setup_state`); a compiled time-loop
driver (pdac_b200/host/pdac_run.cpp) takes its result from this file:

    magic      8 bytes  b"PDACCAS1"
    cfg        the bytes of struct pdac_cfg (include/pdac_gpu.h; its pointer
               members are meaningless here and replaced by the reader)
    control    <4d5i: dt-independent &control values of prog.f's loop:
               tstop, tpr, tdump, max_seconds, imr, nfil, restart (0 from
               scratch, 1 restart), isink, compute_mixture
    dx, dy, dz nx, ny, nz doubles (dy absent in 2D)
    flag       ncell int32
    p_atm, t_atm  nz doubles each
    vent_ijk   nvent int32
    state      the fields of struct pdac_state_view in order, ncell (or
               ncell * nsolid, ncell * ngas) doubles each; vg and vs are
               absent in 2D

All values little-endian, as the host writes them.
"""
from __future__ import annotations

import ctypes as C
import struct

import numpy as np

from . import abi

MAGIC = b"PDACCAS1"
CONTROL = "<4d5i"


def write(case, path):
    """Write `case` (a :class:`~pdac_b200.setup_state.Case`) to `path`."""
    d = case.deck
    cfg = case.cfg()
    mode = str(d["restart_mode"]).strip()
    if mode == "outp_recover":
        # the case file carries no start time or output counter
        raise ValueError("restart_mode 'outp_recover' runs through the Python driver (pdac_b200.files.run)")
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(bytes(cfg))
        f.write(struct.pack(CONTROL, float(d["tstop"]), float(d["tpr"]), float(d["tdump"]), float(d["max_seconds"]),
                            int(d["imr"]), int(d["nfil"]), 1 if mode == "restart" else 0, int(d["isink"]),
                            int(bool(d["compute_mixture"]))))
        f.write(np.ascontiguousarray(case.dx, dtype="<f8").tobytes())
        if case.is3d:
            f.write(np.ascontiguousarray(case.dy, dtype="<f8").tobytes())
        f.write(np.ascontiguousarray(case.dz, dtype="<f8").tobytes())
        f.write(np.ascontiguousarray(case.flag, dtype="<i4").tobytes())
        f.write(np.ascontiguousarray(case.p_atm, dtype="<f8").tobytes())
        f.write(np.ascontiguousarray(case.t_atm, dtype="<f8").tobytes())
        f.write(np.array([v["ijk"] for v in case.vent], dtype="<i4").tobytes())
        for name in abi.STATE_FIELDS:
            if name in ("vg", "vs") and not case.is3d:
                continue
            f.write(np.ascontiguousarray(case.state[name], dtype="<f8").tobytes())
    return path


def cfg_size():
    return C.sizeof(abi.PdacCfg)
