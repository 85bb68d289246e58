"""The per-cell frame comparison of the parity tests (helpers.frame_mismatches)
flags every differing boundary-frame value except where a free in/outflow
face carries a boundary-normal velocity at round-off level.  Mistakes are
planted in a copy of the oracle's own state, on the CPU."""
import numpy as np

import pyoracle
from helpers import STEP_FIELDS, frame_mismatches
from pdac_b200 import configs
from pdac_b200.setup_state import Case


def _state():
    case = Case(configs.plume_2d(nx=32, nz=48))
    o = pyoracle.Oracle(case)
    o.step(1)
    o.step(2)
    return case, o.get_state()


def test_identical_states_have_no_mismatch():
    case, st = _state()
    bad, exempt = frame_mismatches(st, st, STEP_FIELDS, case, 1e-12)
    assert bad == [] and exempt == []


def test_a_planted_frame_error_is_flagged():
    """Wall ghost cells (normal velocity exactly zero) and free in/outflow
    cells with a resolved normal velocity are never exempt."""
    case, st = _state()
    nx = case.nx
    k = case.nz // 2
    wall = nx * (k - 1)                  # axis (slip wall) ghost cell, i = 1
    top = (nx // 2 - 1) + nx * (case.nz - 1)   # top free in/outflow ghost cell
    assert case.flag[wall] == 2 and case.flag[top] == 8
    got = {kk: np.array(v, copy=True) for kk, v in st.items()}
    got["tg"][wall] *= 1.0 + 1e-6
    got["wg"][top - nx] = 5.0            # a resolved normal velocity on the top face
    ref = {kk: np.array(v, copy=True) for kk, v in st.items()}
    ref["wg"][top - nx] = 5.0
    got["p"][top] *= 1.0 + 1e-6
    bad, exempt = frame_mismatches(got, ref, STEP_FIELDS, case, 1e-9)
    assert sorted((b[0], b[2]) for b in bad) == sorted([("tg", wall), ("p", top)])
    assert exempt == []


def test_a_round_off_normal_velocity_exempts_its_ghost_cell():
    case, st = _state()
    nx = case.nx
    k = case.nz // 2
    c = (nx - 1) + nx * (k - 1)         # east ghost cell
    face = c - 1                         # its boundary face (stored at i = nx - 1)
    got = {kk: np.array(v, copy=True) for kk, v in st.items()}
    ref = {kk: np.array(v, copy=True) for kk, v in st.items()}
    got["ug"][face] = 3.0e-37
    ref["ug"][face] = -3.0e-37
    got["tg"][c] = ref["tg"][c] * (1.0 + 1e-7)
    bad, exempt = frame_mismatches(got, ref, STEP_FIELDS, case, 1e-9)
    assert bad == []
    assert ("tg", c) in [(e[0], e[2]) for e in exempt]
