"""Ensembles of independent PDAC runs advanced together on one device.

The reference runs one domain per job; an ensemble there is many jobs.  Here
a batch (``pdac_gpu_batch_*`` in include/pdac_gpu.h) steps many engine
contexts at once, each on its own stream, so that small 2D members, which
fill a few percent of a B200 each, run side by side.  A member computes
exactly what it computes alone: in the batch its sweep loop and wavefront
take their multi-launch forms instead of one cooperative launch, with the
same arithmetic, so a member of a batch produces the same bits as the same
deck run alone.

:func:`member_decks` draws the members of the 2D cylindrical ensemble: the
plume of :func:`pdac_b200.configs.plume_2d` (10 m cells, axis vent of radius
50 m injecting water vapour, two particle classes of 50 and 500 um at
2500 kg/m3) with, per member, a grid of U{64..256} x U{96..384} cells, a
vent velocity ~ U[50, 200] m/s, a vent temperature ~ U[900, 1200] K and a
volume fraction per class log-uniform in [1e-3, 5e-2].  Each member's draws
come from its own Philox stream (key = (seed, member)), so a member's deck
does not depend on how many members are drawn or on which rank draws it.

:func:`split` partitions the members over ranks (one GPU each) by the
longest-processing-time rule on cell counts; ranks exchange nothing.

The CUDA runtime maps streams onto CUDA_DEVICE_MAX_CONNECTIONS hardware
queues (8 by default, read when CUDA starts in the process): set it to 32
before CUDA starts so that the members' streams do not share queues.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import configs
from .engine import Engine, PdacError, lib

NX_RANGE = (64, 256)
NZ_RANGE = (96, 384)
W_RANGE = (50.0, 200.0)
T_RANGE = (900.0, 1200.0)
EPS_RANGE = (1.0e-3, 5.0e-2)


def member_params(m, seed=0, nsolid=2):
    """The draws of member m: nx, nz, w_gas, t_gas, ep_solid."""
    g = np.random.Generator(np.random.Philox(key=np.array([seed, m], dtype=np.uint64)))
    nx = int(g.integers(NX_RANGE[0], NX_RANGE[1] + 1))
    nz = int(g.integers(NZ_RANGE[0], NZ_RANGE[1] + 1))
    w = float(g.uniform(*W_RANGE))
    t = float(g.uniform(*T_RANGE))
    lo, hi = math.log(EPS_RANGE[0]), math.log(EPS_RANGE[1])
    eps = tuple(float(math.exp(g.uniform(lo, hi))) for _ in range(nsolid))
    return dict(nx=nx, nz=nz, w_gas=w, t_gas=t, ep_solid=eps)


def member_decks(n=64, seed=0, first=0, builder="plume_2d", **kw):
    """Decks of members first .. first + n - 1 (keyword arguments override
    the drawn values or the builder's other defaults)."""
    out = []
    for m in range(first, first + n):
        p = member_params(m, seed)
        p.update(kw)
        out.append(getattr(configs, builder)(**p))
    return out


def split(cells, nranks):
    """Member indices of each rank: largest member first to the rank with
    the fewest cells so far (ties to the lowest rank)."""
    order = sorted(range(len(cells)), key=lambda i: (-cells[i], i))
    load = [0] * nranks
    parts = [[] for _ in range(nranks)]
    for i in order:
        r = min(range(nranks), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += cells[i]
    return [sorted(p) for p in parts]


class Batch:
    """Many :class:`~pdac_b200.engine.Engine` members stepped together."""

    def __init__(self, engines, nthreads=0):
        self.L = L = lib()
        P = C.c_void_p
        L.pdac_gpu_batch_create.argtypes = [C.POINTER(P), C.c_int, C.c_int, C.POINTER(P)]
        L.pdac_gpu_batch_step.argtypes = [P, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.pdac_gpu_batch_elapsed.argtypes = [P, C.POINTER(C.c_double)]
        L.pdac_gpu_batch_destroy.argtypes = [P]
        L.pdac_gpu_batch_last_error.argtypes = [P]
        L.pdac_gpu_batch_last_error.restype = C.c_char_p
        for f in ("create", "step", "elapsed", "destroy"):
            getattr(L, f"pdac_gpu_batch_{f}").restype = C.c_int
        self.engines = list(engines)
        n = len(self.engines)
        arr = (P * n)(*[e.h for e in self.engines])
        self.h = P()
        st = L.pdac_gpu_batch_create(arr, n, int(nthreads), C.byref(self.h))
        if st != 0:
            raise PdacError(st, "pdac_gpu_batch_create")
        self.sweep = 0
        self.nit = (C.c_int * n)()
        self.status = (C.c_int * n)()

    def step(self, sweep=None):
        """One time step of every member; returns the members' nit.  Raises
        if any member failed (all members were stepped)."""
        if sweep is None:
            sweep = self.sweep + 1
        self.sweep = sweep
        for e in self.engines:
            e.sweep = sweep
        st = self.L.pdac_gpu_batch_step(self.h, sweep, self.nit, self.status)
        if st != 0:
            raise PdacError(st, "batch_step", (self.L.pdac_gpu_batch_last_error(self.h) or b"").decode())
        return list(self.nit)

    def elapsed(self):
        """Device ms of the last batch step."""
        ms = C.c_double(0)
        self.L.pdac_gpu_batch_elapsed(self.h, C.byref(ms))
        return ms.value

    def close(self):
        if getattr(self, "h", None):
            self.L.pdac_gpu_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
