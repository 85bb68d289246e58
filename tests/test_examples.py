"""The reference's own input decks (its examples/ directory, read in place
from the directory PDAC_REFERENCE_EXAMPLES names; skipped when it is not
set or does not exist): every run deck
parses with the reference's namelist and card syntax (list-directed
records, quoted card names, r*v repeats), the decks whose options are built
set up, the others are rejected naming the option, and the shock-tube deck
(densities given in place of temperatures, density_specified) runs through
the oracle with its gas mass growing by exactly its inflow."""
import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXAMPLES = os.environ.get("PDAC_REFERENCE_EXAMPLES", "")
pytestmark = pytest.mark.skipif(not EXAMPLES or not os.path.isdir(EXAMPLES),
                                reason="set PDAC_REFERENCE_EXAMPLES to the reference's examples directory")

RUN_DECKS = ["dam_break_1", "jet_Ladenburg", "jet_Lewis", "jet_NASA", "jet_Sommerfeld", "shock_tube_1"]


def _deck(name):
    from pdac_b200.deck import Deck
    return Deck.parse(open(os.path.join(EXAMPLES, name + ".dat")).read())


@pytest.mark.parametrize("name", RUN_DECKS)
def test_example_deck_parses(name):
    d = _deck(name)
    assert d["nx"] > 0 and d["nz"] > 0 and len(d.blocks) >= 1
    for b in d.blocks:
        assert 1 <= b["xlo"] <= b["xhi"] <= d["nx"] and 1 <= b["zlo"] <= b["zhi"] <= d["nz"]


def test_example_decks_set_up_or_name_what_is_missing():
    from pdac_b200.setup_state import Case
    outcome = {}
    for name in RUN_DECKS:
        d = _deck(name)
        try:
            Case(d)
            outcome[name] = "ok"
        except ValueError as e:
            outcome[name] = str(e)
    assert outcome["shock_tube_1"] == "ok" and outcome["jet_Ladenburg"] == "ok" and outcome["jet_Lewis"] == "ok"
    assert outcome["dam_break_1"] == "ok"  # generated mesh (grigen = 1)
    assert "ctu" in outcome["jet_NASA"] and "ctu" in outcome["jet_Sommerfeld"]


def test_shock_tube_runs_in_the_oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from pdac_b200.setup_state import Case
    case = Case(_deck("shock_tube_1"))
    o = pyoracle.Oracle(case, order=pyoracle.ORDER_COLORED)
    m0 = o.mass_totals()
    steps = 10
    for s in range(1, steps + 1):
        o.step(s)
    st = o.get_state()
    assert all(np.all(np.isfinite(v)) for v in st.values())
    # the tube's only opening is the fixed-flow cell under its first column:
    # the gas mass grows by that cell's donor flux through the face above it
    c = int(np.flatnonzero(case.flag == 16)[0])
    i = c % case.nx
    inflow = steps * st["rgp"][c] * st["wg"][c] * case.dx[i] * case.deck["dt"]
    m1 = o.mass_totals()
    # each cell's continuity residual is only driven below delg * rgp
    # (1e-8 of its gas mass), so the growth matches to that accuracy
    np.testing.assert_allclose(m1[0] - m0[0], inflow, rtol=1e-5)
    ns = case.nsolid
    np.testing.assert_allclose(m1[1:1 + ns], m0[1:1 + ns], rtol=1e-12)  # no particles enter
    np.testing.assert_allclose(m1[1 + ns:].sum() - m0[1 + ns:].sum(), inflow, rtol=1e-5)  # the one gas species
