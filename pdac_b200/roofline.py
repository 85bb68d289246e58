"""Algorithmic byte counts of the time step, per cell.

Compulsory HBM traffic model: every array a pass needs is read once and
every array it produces is written once, FP64 (8 B).  Symbols: S = 1 + ns
phases, d dimensions, G gas species, N_app = d * S(S+1)/2 interphase terms.

  corrector sweep (iter.f:204-410), per fluid cell:
    R_sweep = 8 + G + 2 ns + 2 d S + N_app     (p, ep, rog, rgp, rgpn, tg,
              conv, abeta, xgc, rlk/rlkn, face velocities, tilde momenta,
              interphase terms)
    W_sweep = 4 + ns + d S                      (p, ep, rog, rgp, rlk,
              face velocities)
  whole step (semi-implicit path, rungekut = 1):
    B_step = 8 [ fixed + nit (R_sweep + W_sweep) ]

  A colour phase of the corrector runs as three kernels:
    collect: the active-set bitmask (ncell / 8 bytes) and 4 bytes per
      candidate written;
    residual test, per candidate: mass-flux faces (2d), rgp, rgpn, conv; a
      converged cell also reads its particle mass-flux faces (2d ns), rlkn,
      sink (2 ns) and rog, and writes rlk (ns), ep and rgp:
        converged    8 [(2d + 3) + (2d + 2) ns + 1 + ns + 2] + 4
        unconverged  8 (2d + 3) + 4 + 4 (worklist entry)
    inner loop, per unconverged cell: 8 (R_sweep + W_sweep) + 4

  explicit SSP-RK3 solver (explicit_solver.f), per fluid cell and kernel
  group of one explicit_iter, neq = (2 + d) S rows:
    flux pass (x3): reads density, enthalpy and temperature of every phase,
      d S velocities, ep, kapg (4 S + d S + 2); writes d S mass, d d S
      momentum and d S enthalpy face fluxes
    stage kernel (x2): reads the 2 d S + d d S + d ns fluxes it
      differentiates, d S viscous terms, p, ep, rgp, rlk (3 + ns), the
      n-level rgp, rlk, sies and d S velocities (1 + 2 ns + d S), k1 in the
      second stage (neq - 1); writes neq - 1 rows, the parked rgp, rlk, ep
      and d gas velocities (2 + ns + d), d ns particle velocities, sies,
      ts (2 ns) and rog
    wavefront (x2): reads d enthalpy fluxes, d + d gas velocities (own and
      lower face), p and its 2 d neighbours, ep, pn, rgpn, siegn, tg, rog,
      2 G mass and mole fractions, the parked 2 + ns + d values, k1 in the
      second stage; writes its row, sieg, tg, cg, p and commits 2 + ns + d
    final (rhs3, coefficients, solve): reads the stage-3 inputs of the stage
      kernel plus gas enthalpy and k1, k2 (2 neq); writes rhs3 (neq); the
      coefficients read d S velocities, rlk, rgp, ep, rog, tg, cg, G mole
      fractions and write rgp, rlk, mug, kapg, ns hv, N_app; the solve
      reads rhs3, N_app (own and upper neighbours), rgp, rlk, hv, cg, tg,
      ts, G mass and mole fractions, and writes the d S velocities, sieg,
      sies, tg, ts, cg, ep, rog, p
"""
from __future__ import annotations


def sweep_doubles(ns, ng, d=2):
    S = 1 + ns
    n_app = d * S * (S + 1) // 2
    r = 8 + ng + 2 * ns + 2 * d * S + n_app
    w = 4 + ns + d * S
    return r, w


def step_fixed_doubles(ns, ng, d=2):
    """Doubles per cell of the non-iterative passes of one step."""
    S = 1 + ns
    n_state = 6 + d + ns * (3 + d) + 2 * ng
    n_old = 4 + 2 * ns + ng + d * S
    n_app = d * S * (S + 1) // 2
    # boundary + fieldn, tilde (+fluxes), predictor/betas, ygas, htilde, ftem
    return (n_state + n_old + 2) + (n_state + d * S + n_app) + (d * S + n_app + 5 + d * S + 2) \
        + (2 * ng + d + 2) + (2 * S + d * S + 2) + (2 * S + n_state)


def corrector_bytes_per_cell_sweep(ns, ng, d=2):
    r, w = sweep_doubles(ns, ng, d)
    return 8 * (r + w)


def step_bytes_per_cell(ns, ng, nit, d=2):
    r, w = sweep_doubles(ns, ng, d)
    return 8 * (step_fixed_doubles(ns, ng, d) + nit * (r + w))


def resid_bytes(ns, d, converged, unconverged, ncell=0, phases=0):
    """Algorithmic bytes of the collect + residual-test launches of `phases`
    colour phases that tested the given cells."""
    conv = 8 * ((2 * d + 3) + (2 * d + 2) * ns + 1 + ns + 2) + 4
    unconv = 8 * (2 * d + 3) + 8
    return conv * converged + unconv * unconverged + phases * (ncell // 8)


def inner_bytes(ns, ng, d, unconverged):
    """Algorithmic bytes of inner-loop launches over the given worklist cells."""
    r, w = sweep_doubles(ns, ng, d)
    return (8 * (r + w) + 4) * unconverged


def rk3_group_doubles(ns, ng, d):
    """Doubles per fluid cell moved by each kernel group of one explicit_iter
    (all repetitions of the group included)."""
    S = 1 + ns
    neq = (2 + d) * S
    n_app = d * S * (S + 1) // 2
    flux = 3 * ((4 * S + d * S + 2) + (d * S + d * d * S + d * S))
    stage_r = (2 * d * S + d * d * S + d * ns) + d * S + (3 + ns) + (1 + 2 * ns + d * S)
    stage_w = (neq - 1) + (2 + ns + d) + d * ns + 2 * ns + 1
    stage = 2 * (stage_r + stage_w) + (neq - 1)
    wave_r = d + 2 * d + (1 + 2 * d) + 6 + 2 * ng + (2 + ns + d)
    wave_w = 1 + 4 + (2 + ns + d)
    wave = 2 * (wave_r + wave_w) + 1
    final = (stage_r + d + 2 * neq + neq) \
        + (d * S + ns + 1 + 1 + 1 + 1 + 1 + ng + 2 + ns + 2 + ns + n_app) \
        + (neq + n_app + 1 + ns + ns + 1 + 1 + ns + 2 * ng + d * S + 1 + ns + 1 + ns + 1 + 1 + 1 + 1)
    return {"flux": flux, "stage": stage, "wave": wave, "final": final}


def rk3_group_bytes(ns, ng, d, fluid_cells):
    """Algorithmic bytes of each kernel group of one explicit_iter."""
    return {k: 8 * v * fluid_cells for k, v in rk3_group_doubles(ns, ng, d).items()}
