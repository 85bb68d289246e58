"""The ground sink of the oracle (sink.f:46-121, the checker of the CUDA
sink) against its definition, computed here independently: after one
boundary call every fluid cell above a wall inside the ring rprox < r <
rdist takes out rlk min(0, ws) / dz, every other cell nothing, and each
ground column's massl is the sum of its cells' sink dx dz dt (dx dy dz dt
in 3D)."""
import os
import sys

import numpy as np
import pytest

from sink_decks import seeded_case

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def _centres(d):
    xb, x = 0.0, [-0.5 * d[0]]
    for v in d[1:]:
        xb = xb + v
        x.append(xb - 0.5 * v)
    return x


@pytest.mark.parametrize("builder", ["small_2d_sink", "small_3d_sink"])
def test_oracle_sink_after_one_boundary_call(builder):
    import pyoracle
    case = seeded_case(builder)
    o = pyoracle.Oracle(case, order=pyoracle.ORDER_COLORED)
    before = o.get_state()
    o.boundary(1)
    sink, massl = o.get("sink"), o.get("massl")
    d = case.deck
    n, ns, nx = case.ncell, case.nsolid, case.nx
    ny = case.ny if case.is3d else 1
    x = _centres(list(case.dx))
    y = _centres(list(case.dy)) if case.is3d else [0.0]
    ntr = nx * ny
    want_sink = np.zeros(n * ns)
    want_massl = np.zeros(ntr * ns)
    flag = case.flag
    for c in range(n):
        i, j, k = c % nx, (c // nx) % ny, c // (nx * ny)
        if k == 0 or flag[c] not in (1, 5, 129) or flag[c - nx * ny] not in (2, 4, 512, 1024):
            continue
        r2 = (x[i] - d["center_x"]) ** 2 + (y[j] - d["center_y"]) ** 2
        for q in range(ns):
            s = 0.0
            if d["rprox"] ** 2 < r2 < d["rdist"] ** 2:
                s = before["rlk"][q * n + c] * min(0.0, before["ws"][q * n + c]) / case.dz[k]
            want_sink[q * n + c] = s
            vol = case.dx[i] * case.dz[k] * (case.dy[j] if case.is3d else 1.0)
            want_massl[q * ntr + i + nx * j] += s * vol * d["dt"]
    assert np.count_nonzero(want_sink) > 0
    np.testing.assert_allclose(sink, want_sink, rtol=1e-13, atol=0)
    np.testing.assert_allclose(massl, want_massl, rtol=1e-12, atol=0)


def test_sink_options_reach_the_configuration():
    from pdac_b200 import configs
    from pdac_b200.setup_state import Case
    cfg = Case(configs.small_3d_sink()).cfg()
    assert (cfg.isink, cfg.rprox, cfg.rdist, cfg.center_x, cfg.center_y) == (1, 20.0, 70.0, 100.0, 80.0)
