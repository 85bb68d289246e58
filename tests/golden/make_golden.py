"""Generate the oracle regression fixtures in this directory.

    python tests/golden/make_golden.py

Runs the CPU oracle on the small 2D and 3D plume decks for three time steps
in both sweep orders (lexicographic = the reference's order, colored = the
CUDA engine's order), and on the same decks with the explicit SSP-RK3
solver (time_integration = 1, which has no sweep order) and with the
sub-grid turbulence model (iturb = 1, iss = 1), and records, after every step, the outer-sweep count
and per-field summaries (sum, sum of |x|, max |x|) plus the values at a few
fixed fluid cells.  The fixtures pin the oracle against unintended change;
the GPU parity tests also compare the engine with the colored fixture.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

FIELDS = ("p", "ep", "rog", "rgp", "tg", "sieg", "cg", "ug", "vg", "wg",
          "rlk", "ts", "sies", "us", "vs", "ws", "ygc", "xgc")
STEPS = 3


def probe_cells(case, count=6):
    fluid = np.flatnonzero(case.flag & 1)
    idx = np.linspace(0, fluid.size - 1, count).astype(int)
    return [int(c) for c in fluid[idx]]


def summarize(state, cells, ncell):
    out = {}
    for f in FIELDS:
        a = np.asarray(state[f], dtype=np.float64)
        nb = a.size // ncell
        out[f] = {"sum": float(a.sum()), "abs_sum": float(np.abs(a).sum()), "max_abs": float(np.abs(a).max()),
                  "probe": [float(a[b * ncell + c]) for b in range(nb) for c in cells]}
    return out


def run(builder_name, order):
    import pyoracle
    from pdac_b200 import configs
    from pdac_b200.setup_state import Case
    case = Case(getattr(configs, builder_name)())
    o = pyoracle.Oracle(case, order=order)
    cells = probe_cells(case)
    steps = []
    for s in range(1, STEPS + 1):
        nit = o.step(s)
        steps.append({"step": s, "nit": int(nit), "fields": summarize(o.get_state(), cells, case.ncell)})
    return {"deck": builder_name, "ncell": case.ncell, "probe_cells": cells, "steps": steps}


def main():
    import pyoracle
    pyoracle.build()
    data = {}
    for deck in ("small_2d", "small_3d"):
        for name, order in (("lexicographic", pyoracle.ORDER_LEXICOGRAPHIC), ("colored", pyoracle.ORDER_COLORED)):
            data[f"{deck}/{name}"] = run(deck, order)
    # the explicit solver has no corrector, so its single fixture serves both orders
    for deck in ("small_2d_rk3", "small_3d_rk3", "small_2d_rk3_les"):
        data[f"{deck}/lexicographic"] = run(deck, pyoracle.ORDER_LEXICOGRAPHIC)
    # the sub-grid turbulence model (iturb = 1, iss = 1)
    for deck in ("small_2d_les", "small_3d_les"):
        for name, order in (("lexicographic", pyoracle.ORDER_LEXICOGRAPHIC), ("colored", pyoracle.ORDER_COLORED)):
            data[f"{deck}/{name}"] = run(deck, order)
    path = os.path.join(HERE, "oracle_small.json")
    with open(path, "w") as fh:
        json.dump(data, fh, indent=1)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
