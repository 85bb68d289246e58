"""Ensembles through pdac_gpu_batch_*: members of different grids, decks and
time integrations stepped together on one device give the same bits as the
same decks stepped alone, and the batch reports every member's outcome."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _members():
    from pdac_b200 import configs
    return [
        configs.small_2d(nx=12, nz=16),
        configs.small_2d(nx=14, nz=19, w_gas=150.0, t_gas=950.0, ep_solid=(0.002, 0.03)),
        configs.small_2d(nx=9, nz=23, w_gas=60.0, t_gas=1180.0, ep_solid=(0.04, 0.001)),
        configs.small_3d(),
        configs.small_2d_rk3(nx=13, nz=17),
    ]


def _run_alone(deck, steps):
    from pdac_b200.engine import Engine
    from pdac_b200.setup_state import Case
    e = Engine(Case(deck))
    nits = [e.step(s) for s in range(1, steps + 1)]
    out = e.download()
    e.close()
    return nits, out


@pytest.mark.parametrize("nthreads", [0, 2])
def test_batch_matches_members_run_alone(nthreads):
    from pdac_b200.engine import Engine
    from pdac_b200.ensemble import Batch
    from pdac_b200.setup_state import Case
    decks = _members()
    steps = 3
    engines = [Engine(Case(d)) for d in decks]
    b = Batch(engines, nthreads=nthreads)
    got_nit = [b.step(s) for s in range(1, steps + 1)]
    assert b.elapsed() > 0.0
    got = [e.download() for e in engines]
    b.close()
    for e in engines:
        e.close()
    for m, d in enumerate(decks):
        nits, ref = _run_alone(d, steps)
        assert [row[m] for row in got_nit] == nits, m
        for name, v in ref.items():
            np.testing.assert_array_equal(got[m][name], v, err_msg=f"member {m} field {name}")


def test_batch_graph_rebuilt_after_new_launch_shapes():
    """The semi-implicit members run as one graph built at the first batch
    step; a member's new launch shapes (pdac_gpu_set_tuning between batch
    steps) rebuild it, and the results stay those of the decks run alone."""
    from pdac_b200 import configs
    from pdac_b200.engine import Engine
    from pdac_b200.ensemble import Batch
    from pdac_b200.setup_state import Case
    decks = [configs.plume_3d(nx=40, ny=21, nz=30, vent_cells=4), configs.small_2d(nx=14, nz=19)]
    steps = 4
    engines = [Engine(Case(d)) for d in decks]
    b = Batch(engines)
    got_nit = []
    for s in range(1, steps + 1):
        if s == 3:
            engines[0].set_tuning(dict(tile_shape=2, tile_kchunk=7, inner_grid=148 * 4, test_grid=148 * 2,
                                       coop_cells_per_block=1024))
        got_nit.append(b.step(s))
    got = [e.download() for e in engines]
    b.close()
    for e in engines:
        e.close()
    for m, d in enumerate(decks):
        nits, ref = _run_alone(d, steps)
        assert [row[m] for row in got_nit] == nits, m
        for name, v in ref.items():
            np.testing.assert_array_equal(got[m][name], v, err_msg=f"member {m} field {name}")


def test_batch_rejects_a_member_given_twice():
    from pdac_b200 import configs
    from pdac_b200.engine import Engine, PdacError
    from pdac_b200.ensemble import Batch
    from pdac_b200.setup_state import Case
    e = Engine(Case(configs.small_2d()))
    with pytest.raises(PdacError):
        Batch([e, e])
    e.close()


def test_drawn_members_step_in_a_batch():
    """Members of the 2D ensemble's distribution (grids scaled down) run and
    conserve what a closed step conserves: finite fields, positive density."""
    from pdac_b200.engine import Engine
    from pdac_b200.ensemble import Batch, member_decks, member_params
    from pdac_b200.setup_state import Case
    decks = []
    for m in range(6):
        p = member_params(m)
        decks += member_decks(1, first=m, nx=max(8, p["nx"] // 8), nz=max(12, p["nz"] // 8))
    engines = [Engine(Case(d)) for d in decks]
    b = Batch(engines)
    for s in range(1, 3):
        nit = b.step(s)
        assert all(n >= 1 for n in nit)
    for e in engines:
        st = e.download()
        assert all(np.all(np.isfinite(v)) for v in st.values())
        assert np.all(st["rog"] > 0.0)
    b.close()
    for e in engines:
        e.close()


def test_drawn_members_match_the_oracle():
    """Two members of the 2D ensemble as drawn (grid, vent velocity and
    temperature, class volume fractions), stepped in a batch, against the
    oracle run on each member's deck: same outer sweeps, fields to 1e-9
    (relative L-infinity over the fluid cells) after every step."""
    import pyoracle
    from helpers import STEP_FIELDS, compare_state
    from pdac_b200.engine import Engine
    from pdac_b200.ensemble import Batch, member_decks, split
    from pdac_b200.setup_state import Case
    decks = member_decks(64)
    cells = [d["nx"] * d["nz"] for d in decks]
    pick = [min(range(64), key=lambda m: cells[m]), sorted(range(64), key=lambda m: cells[m])[32]]
    cases = [Case(decks[m]) for m in pick]
    engines = [Engine(c) for c in cases]
    oracles = [pyoracle.Oracle(c, order=pyoracle.ORDER_COLORED) for c in cases]
    b = Batch(engines)
    for s in range(1, 6):
        nit = b.step(s)
        for q, (c, e, o) in enumerate(zip(cases, engines, oracles)):
            assert nit[q] == o.step(s), f"member {pick[q]} step {s}"
            fluid = (c.flag & 1) == 1
            errs, bad = compare_state(e.download(), o.get_state(), STEP_FIELDS, 1e-9, c.nsolid, c.ncell, cells=fluid)
            assert not bad, f"member {pick[q]} step {s}: {bad}"
    b.close()
    for e in engines:
        e.close()
