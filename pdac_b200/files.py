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
sink, from massl.NNNN of the namelist's nfil; ``'outp_recover'`` starts
from the fields of output.NNNN of the namelist's nfil (outp_recover,
io_restart.f:341-493, and the itd > 2 branch of cnvert, setup.f:393-440;
:func:`recover_output`).  The files themselves are written by the engine's
C entry points in the reference's formats.
"""
from __future__ import annotations

import math
import os
import time as _time

import numpy as np


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


def _unformatted_records(raw):
    """The records of a Fortran unformatted sequential file (4-byte length
    markers before and after each record)."""
    out, q = [], 0
    while q < len(raw):
        n = int(np.frombuffer(raw, "<i4", 1, q)[0])
        out.append(raw[q + 4:q + 4 + n])
        if int(np.frombuffer(raw, "<i4", 1, q + 4 + n)[0]) != n:
            raise ValueError("output file: record markers do not match")
        q += n + 8
    return out


def read_output_fields(case, path):
    """The fields outp_recover reads from an output file (io_restart.f:
    341-493): (time, [arrays in file order]) for p, the gas velocity (u, w;
    u, v, w in 3D), tg, xgc per gas and per class eps, the particle velocity
    and ts, each ncell long.  The unformatted form holds REAL(time, 4) and one
    REAL*4 record per field (read_array with sgl, io_parallel.f:166-230);
    the formatted one (&control formatted_input) three lines, the time line
    '(12x, g11.4)', then per field four header lines (FORMAT 122) and the
    values list-directed.  Records after the last of these (the mixture
    fields) are not read."""
    n, ns, ng = case.ncell, case.nsolid, case.ngas
    nvel = 3 if case.is3d else 2
    nfields = 1 + nvel + 1 + ng + ns * (2 + nvel)
    if not case.deck["formatted_input"]:
        with open(path, "rb") as f:
            recs = _unformatted_records(f.read())
        if len(recs) < 1 + nfields:
            raise ValueError(f"{path}: {len(recs)} records, outp_recover needs {1 + nfields}")
        time = float(np.frombuffer(recs[0], "<f4", 1)[0])
        fields = []
        for r in recs[1:1 + nfields]:
            a = np.frombuffer(r, "<f4")
            if a.size != n:
                raise ValueError(f"{path}: a record of {a.size} values, the mesh has {n} cells")
            fields.append(a.astype(np.float64))
        return time, fields
    with open(path) as f:
        lines = f.read().split("\n")
    time = float(lines[3][12:23])
    fields, q = [], 4
    for _ in range(nfields):
        q += 4  # FORMAT(1x,//,6x,/): two empty lines, the name, one empty line
        vals = []
        while len(vals) < n:
            if q >= len(lines):
                raise ValueError(f"{path}: the file ends inside a field")
            vals += [float(t) for t in lines[q].replace(",", " ").split()]
            q += 1
        fields.append(np.array(vals[:n], dtype=np.float64))
    return time, fields


def recover_output(case, path):
    """outp_recover (io_restart.f:341-493) followed by cnvert with itd > 2
    (setup.f:393-440): the state of `case` rebuilt from the fields of an
    output file.  Returns (time, state).  Read: p, gas velocity, tg, xgc, and
    per class rlk = eps rl, particle velocity, ts; every other gas and
    particle field is derived per cell: ygc from xgc (mas), rog from the
    thermal equation of state, ep = 1 - sum rlk / rl, rgp = rog ep, cg from
    the specific heats at tg, sieg = (tg - tzero) cg + hzerog and sies =
    (ts - tzero) ck + hzeros with tzero = hzerog = hzeros = 0 and ck the
    class's constant specific heat (hcaps)."""
    from .setup_state import hcapg, mas, thermal_eosg
    d = case.deck
    n, ns, ng = case.ncell, case.nsolid, case.ngas
    time, f = read_output_fields(case, path)
    st = {k: np.array(v, dtype=np.float64, copy=True) for k, v in case.state.items()}
    it = iter(f)
    st["p"][:] = next(it)
    st["ug"][:] = next(it)
    if case.is3d:
        st["vg"][:] = next(it)
    st["wg"][:] = next(it)
    st["tg"][:] = next(it)
    X = np.stack([next(it) for _ in range(ng)])
    rl = np.array(d["density"][:ns], dtype=np.float64)
    for s in range(ns):
        blk = slice(s * n, (s + 1) * n)
        st["rlk"][blk] = next(it) * rl[s]
        st["us"][blk] = next(it)
        if case.is3d:
            st["vs"][blk] = next(it)
        st["ws"][blk] = next(it)
        st["ts"][blk] = next(it)
    st["xgc"][:] = X.reshape(-1)
    Y = mas(X, case.gas_type)
    st["ygc"][:] = Y.reshape(-1)
    st["rog"][:] = thermal_eosg(st["tg"], st["p"], X, case.gas_type)
    ep = np.ones(n)
    for s in range(ns):
        ep = ep - st["rlk"][s * n:(s + 1) * n] * (1.0 / rl[s])
    st["ep"][:] = ep
    st["rgp"][:] = st["rog"] * st["ep"]
    cp = hcapg(st["tg"], d["icpc"], d["tref"])
    hc = np.zeros(n)
    for ig, gt in enumerate(case.gas_type):
        hc = hc + cp[gt - 1] * Y[ig]
    st["cg"][:] = hc
    st["sieg"][:] = (st["tg"] - 0.0) * st["cg"] + 0.0
    cps = np.array(d["specific_heat"][:ns], dtype=np.float64)
    for s in range(ns):
        blk = slice(s * n, (s + 1) * n)
        st["sies"][blk] = (st["ts"][blk] - 0.0) * cps[s] + 0.0
    return time, st


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
    if mode not in ("from_scratch", "default", "restart", "check_init", "outp_recover"):
        raise ValueError(f"restart_mode {mode!r} is not supported by this driver")
    os.makedirs(workdir, exist_ok=True)
    path = lambda name: os.path.join(workdir, name)
    sink = int(d["isink"]) > 0
    if mode == "restart":
        if sink:
            # setup.f:147: read_mass_loss(nfil) with the namelist's nfil
            engine.read_mass_loss(path(massl_name(int(d["nfil"]))))
        t, nfil = engine.read_restart(path(RESTART_FILE))
    elif mode == "outp_recover":
        # setup.f:151-155: read_mass_loss(nfil), outp_recover(nfil) (which
        # advances nfil), cnvert
        nfil = int(d["nfil"])
        if sink:
            engine.read_mass_loss(path(massl_name(nfil)))
        t, state = recover_output(case, path(output_name(nfil)))
        engine.upload(state)
        nfil += 1
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
