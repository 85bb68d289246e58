"""File names and the time-loop driver of the reference's host program.

``run`` mirrors ``main_prog`` (prog.f:143-417) over an :class:`Engine`:
boundary, the initial dump at the first step, fieldn and the Runge-Kutta
loop (or initialize_fieldn and explicit_iter with time_integration = 1),
then the output dump every ``nprint`` steps (outp, output.NNNN), the
mass-check line every step when ``imr >= 1`` (pdac.chm) and the restart
file every ``ndump`` steps (tapewr, pdac.res), with nprint = NINT(tpr/dt)
and ndump = NINT(tdump/dt) (prog.f:84-85); with the ground sink (isink > 0)
also the columns' lost mass before each output (massl.NNNN, prog.f:355) and
after each restart file (massl.res, prog.f:386).  ``restart_mode =
'restart'`` starts from pdac.res (taperd, setup.f:147-150) and, with the
sink, from massl.NNNN of the namelist's nfil.  The files themselves are
written by the engine's C entry points in the reference's formats.
"""
from __future__ import annotations

import math
import os
import time as _time


def lettera(k):
    """letter.f:1-21: the four characters of the output file counter."""
    ithou = int(k / 1000)
    ihund = int((k - ithou * 1000) / 100)
    iten = int((k - ithou * 1000 - ihund * 100) / 10)
    ione = k - ithou * 1000 - ihund * 100 - iten * 10
    return "".join(chr(v + 48) for v in (ithou, ihund, iten, ione))


def output_name(nfil):
    """outp.f:221: output.NNNN."""
    return "output." + lettera(nfil)


def massl_name(nfil=None):
    """sink.f:141-145: massl.NNNN, or massl.res without a counter."""
    return "massl.res" if nfil is None else "massl." + lettera(nfil)


def nint(x):
    """Fortran NINT: nearest integer, halves away from zero."""
    return int(math.floor(abs(x) + 0.5)) * (1 if x >= 0 else -1)


RESTART_FILE = "pdac.res"   # io_files.f:41
CHECK_FILE = "pdac.chm"     # io_files.f:38


def run(engine, workdir, max_steps=None, log=None):
    """Advance `engine` through the time loop of its deck, writing the
    reference's files into `workdir`; returns (time, nfil, sweep).

    The deck's &control group sets restart_mode ('from_scratch' or
    'restart'), dt, tstop, tpr, tdump, imr, max_seconds; `max_steps`
    bounds the number of steps of this call."""
    case = engine.case
    d = case.deck
    dt = d["dt"]
    mode = str(d["restart_mode"]).strip()
    if mode not in ("from_scratch", "default", "restart", "check_init"):
        raise ValueError(f"restart_mode {mode!r} is not supported by this driver")
    os.makedirs(workdir, exist_ok=True)
    path = lambda name: os.path.join(workdir, name)
    sink = int(d["isink"]) > 0
    if mode == "restart":
        if sink:
            # setup.f:147: read_mass_loss(nfil) with the namelist's nfil
            engine.read_mass_loss(path(massl_name(int(d["nfil"]))))
        t, nfil = engine.read_restart(path(RESTART_FILE))
    else:
        t, nfil = 0.0, 0
    nprint = max(1, nint(d["tpr"] / dt))
    ndump = max(1, nint(d["tdump"] / dt))
    sweep = nint(t / dt)
    if d["update_eosg"]:
        raise ValueError("update_eosg is not built")
    explicit = int(d["time_integration"]) == 1
    rk = int(d["rungekut"])
    w0 = _time.time()
    steps = 0
    while True:
        sweep += 1
        engine.boundary(sweep)
        if sweep == 1:
            engine.write_output(path(output_name(nfil)), t)
            nfil += 1
        if mode == "check_init":
            break
        if explicit:
            engine.initialize_fieldn()
        else:
            engine.fieldn()
        engine.sgsg()
        engine.sgss()
        ifx, ien = bool(d["implicit_fluxes"]), bool(d["implicit_enthalpy"])
        nit = 0
        for r in range(1, rk + 1):
            dtr = dt / (rk + 1 - r)
            if explicit:
                engine.explicit_iter(dtr)
                engine.ygas(dtr)
            else:
                # prog.f:246-292: the implicit modes move tilde (and htilde)
                # into iter's sweeps
                if not ifx:
                    engine.tilde(dtr)
                    if ien:
                        engine.htilde(dtr)
                nit = engine.iter(dtr)
                engine.ygas(dtr)
                if not ien:
                    engine.htilde(dtr)
                    engine.ftem(dtr)
        if d["compute_mixture"]:
            engine.compute_mixture_fields()  # prog.f:331
        t = t + dt
        if log:
            log.write(f"Iteration: {sweep:6d} nit: {0 if explicit else nit:5d}\n")
        if sweep % nprint == 0:
            if sink:
                engine.write_mass_loss(path(massl_name(nfil)))
            engine.write_output(path(output_name(nfil)), t)
            nfil += 1
        if int(d["imr"]) >= 1:
            engine.append_mass_check(path(CHECK_FILE), sweep, dt)
        steps += 1
        stop_now = (_time.time() - w0) > float(d["max_seconds"])
        if sweep % ndump == 0 or stop_now:
            engine.write_restart(path(RESTART_FILE), t, nfil)
            if sink:
                engine.write_mass_loss(path(massl_name()))
        if t + 0.1 * dt >= d["tstop"] or stop_now or (max_steps is not None and steps >= max_steps):
            break
    return t, nfil, sweep
