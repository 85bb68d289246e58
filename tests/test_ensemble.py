"""Host logic of the ensemble (no GPU): the members' draws, the split of
members over ranks, and a two-rank gloo run in which each rank advances its
members with the oracle and the gathered results equal one process's."""
import math
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_member_draws_lie_in_their_ranges_and_are_reproducible():
    from pdac_b200 import ensemble as E
    ps = [E.member_params(m) for m in range(64)]
    for p in ps:
        assert E.NX_RANGE[0] <= p["nx"] <= E.NX_RANGE[1]
        assert E.NZ_RANGE[0] <= p["nz"] <= E.NZ_RANGE[1]
        assert E.W_RANGE[0] <= p["w_gas"] <= E.W_RANGE[1]
        assert E.T_RANGE[0] <= p["t_gas"] <= E.T_RANGE[1]
        assert len(p["ep_solid"]) == 2
        assert all(E.EPS_RANGE[0] <= e <= E.EPS_RANGE[1] for e in p["ep_solid"])
    assert ps == [E.member_params(m) for m in range(64)]
    # a member's draws do not depend on which members are drawn with it
    assert E.member_decks(1, first=17)[0]["nx"] == ps[17]["nx"]
    # the grids are uneven
    assert len({(p["nx"], p["nz"]) for p in ps}) == 64
    # log-uniform volume fractions: the median sits near the geometric mean
    med = np.median([e for p in ps for e in p["ep_solid"]])
    assert abs(math.log(med) - 0.5 * (math.log(1e-3) + math.log(5e-2))) < 0.6


@pytest.mark.parametrize("nranks", [1, 2, 3, 8])
def test_split_partitions_and_balances(nranks):
    from pdac_b200 import ensemble as E
    cells = [E.member_params(m)["nx"] * E.member_params(m)["nz"] for m in range(64)]
    parts = E.split(cells, nranks)
    assert sorted(i for p in parts for i in p) == list(range(64))
    loads = [sum(cells[i] for i in p) for p in parts]
    # longest-processing-time bound: no rank exceeds another by more than the largest member
    assert max(loads) - min(loads) <= max(cells)


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from pdac_b200 import ensemble as E
    from pdac_b200.setup_state import Case
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    decks = [E.member_decks(1, first=m, nx=8 + m, nz=12 + 2 * m)[0] for m in range(5)]
    cells = [d["nx"] * d["nz"] for d in decks]
    mine = E.split(cells, world)[rank]
    res = {}
    for m in mine:
        o = pyoracle.Oracle(Case(decks[m]), order=0)
        nits = [o.step(s) for s in (1, 2)]
        res[m] = (nits, o.mass_totals().tolist())
    gathered = [None] * world
    dist.all_gather_object(gathered, res)
    if rank == 0:
        merged = {}
        for g in gathered:
            merged.update(g)
        out.put(merged)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_advance_disjoint_members():
    import multiprocessing as mp
    import socket
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from pdac_b200 import ensemble as E
    from pdac_b200.setup_state import Case
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    merged = q.get(timeout=300)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(merged) == list(range(5))
    for m in range(5):
        o = pyoracle.Oracle(Case(E.member_decks(1, first=m, nx=8 + m, nz=12 + 2 * m)[0]), order=0)
        nits = [o.step(s) for s in (1, 2)]
        assert merged[m] == (nits, o.mass_totals().tolist())
