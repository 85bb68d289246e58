"""The CUDA engine against the committed colored-order oracle fixtures
(tests/golden/oracle_small.json): equal outer-sweep counts and probe values
at fluid cells within 1e-9 of each field's scale; particle temperature and
enthalpy probes only where that class is present (rlk > 1e-5)."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "oracle_small.json")))
TOL = 1e-9


@pytest.mark.parametrize("deck", ["small_2d", "small_3d", "small_2d_rk3", "small_3d_rk3", "small_2d_les", "small_3d_les",
                                  "small_2d_rk3_les"])
def test_engine_matches_colored_fixture(deck):
    """The explicit-solver decks (no corrector, no sweep order) have one
    fixture, stored under the lexicographic key."""
    from pdac_b200 import configs
    from pdac_b200.engine import Engine
    from pdac_b200.setup_state import Case
    from golden.make_golden import summarize
    ref = GOLDEN.get(f"{deck}/colored") or GOLDEN[f"{deck}/lexicographic"]
    case = Case(getattr(configs, deck)())
    eng = Engine(case)
    cells = ref["probe_cells"]
    for st in ref["steps"]:
        nit = eng.step(st["step"])
        assert nit == st["nit"], f"step {st['step']}: {nit} vs {st['nit']}"
        got = summarize(eng.download(), cells, case.ncell)
        rlk_probe = np.asarray(st["fields"]["rlk"]["probe"])
        for f, want in st["fields"].items():
            g, w = np.asarray(got[f]["probe"]), np.asarray(want["probe"])
            sel = np.ones(w.size, dtype=bool)
            if f in ("ts", "sies"):
                sel = rlk_probe > 1e-5
            scale = max(want["max_abs"], 1e-300)
            assert np.all(np.abs(g[sel] - w[sel]) <= TOL * scale), (st["step"], f, g[sel], w[sel])
    eng.close()
