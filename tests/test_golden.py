"""The oracle reproduces its committed regression fixtures
(tests/golden/oracle_small.json, made by tests/golden/make_golden.py):
outer-sweep counts exactly, per-field summaries and probe values to 1e-12
relative to each field's scale."""
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "oracle_small.json")))
TOL = 1e-12


@pytest.mark.parametrize("key", sorted(GOLDEN))
def test_oracle_matches_fixture(key):
    import pyoracle
    from pdac_b200 import configs
    from golden.make_golden import summarize
    deck, order = key.split("/")
    ref = GOLDEN[key]
    from pdac_b200.setup_state import Case
    case = Case(getattr(configs, deck)())
    o = pyoracle.Oracle(case, order=pyoracle.ORDER_COLORED if order == "colored" else pyoracle.ORDER_LEXICOGRAPHIC)
    for st in ref["steps"]:
        nit = o.step(st["step"])
        assert nit == st["nit"]
        got = summarize(o.get_state(), ref["probe_cells"], case.ncell)
        for f, want in st["fields"].items():
            scale = max(want["max_abs"], 1e-300)
            assert abs(got[f]["sum"] - want["sum"]) <= TOL * max(want["abs_sum"], 1e-300), (st["step"], f)
            np.testing.assert_allclose(got[f]["probe"], want["probe"], rtol=0, atol=TOL * scale, err_msg=f)
