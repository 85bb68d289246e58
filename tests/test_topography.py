"""Host-side topography and immersed-boundary set-up (no GPU).

Known answers for the interpolations (arrfil.f), the DEM file round trip,
the flags the topography gives the mesh (topo.f set_flags and
export_topography), the forcing points and face factors of the immersed
boundaries (immb.f, ghost.f:2888-3345), and a few oracle steps on every
topography deck.
"""
import numpy as np
import pytest

from pdac_b200 import configs, topography
from pdac_b200.deck import Deck
from pdac_b200.setup_state import Case


def test_nint_rounds_half_away_from_zero():
    assert list(topography.nint([0.5, 1.5, 2.5, -0.5, -1.5, 2.4999])) == [1, 2, 3, -1, -2, 2]


def test_interp_1d_known_answers():
    x1 = np.array([0.0, 10.0, 20.0])
    f1 = np.array([0.0, 5.0, 25.0])
    f2, t = topography.interp_1d(x1, f1, np.array([-3.0, 0.0, 4.0, 10.0, 15.0, 20.0]))
    # left of the profile: its first value (t = 1); then linear by segment
    assert list(t) == [1, 1, 2, 2, 3, 3]
    np.testing.assert_array_equal(f2, [0.0, 0.0, 2.0, 5.0, 15.0, 25.0])
    with pytest.raises(ValueError):
        topography.interp_1d(x1, f1, np.array([21.0]))


def test_interp_2d_is_exact_on_bilinear_fields():
    x1 = np.linspace(0.0, 100.0, 11)
    y1 = np.linspace(0.0, 50.0, 6)
    X, Y = np.meshgrid(x1, y1, indexing="ij")
    f1 = 3.0 + 0.5 * X - 0.25 * Y + 0.01 * X * Y
    x2 = np.array([0.0, 3.0, 47.5, 100.0])
    y2 = np.array([0.0, 12.5, 50.0])
    f2, tx, ty = topography.interp_2d(x1, y1, f1, x2, y2)
    X2, Y2 = np.meshgrid(x2, y2, indexing="ij")
    np.testing.assert_allclose(f2, 3.0 + 0.5 * X2 - 0.25 * Y2 + 0.01 * X2 * Y2, rtol=1e-13)


def test_mean_filter_keeps_a_constant_surface():
    x = np.arange(0.0, 200.0, 10.0)
    y = np.arange(0.0, 150.0, 10.0)
    f = np.full((x.size, y.size), 42.0)
    np.testing.assert_allclose(topography.mean_filter_2d(x, y, f, 30.0), 42.0, rtol=1e-14)


def test_dem_file_round_trip(tmp_path):
    z = np.arange(12, dtype=float).reshape(4, 3) * 1.5
    p = tmp_path / "d.asc"
    topography.write_dem_ascii(str(p), 100.0, 200.0, 5.0, z)
    xd, yd, zd = topography.read_dem_ascii(str(p))
    np.testing.assert_array_equal(xd, [100.0, 105.0, 110.0, 115.0])
    np.testing.assert_array_equal(yd, [200.0, 205.0, 210.0])
    np.testing.assert_array_equal(zd, z)


def test_staircase_flags_2d(tmp_path):
    case = Case(configs.small_2d_topo(tmp_path, immb=0))
    topo = case.topography
    f = case.flag3[:, 0, :]
    for i in range(1, case.nx - 1):
        q = int(topo.ord[i])
        # cells up to ord are no-slip walls (set_flags) unless they are vent cells
        assert all(f[k, i] in (4, 64) for k in range(q)), i
        # the rows just above are boundary-layer cells or stay fluid
        assert f[q, i] in (5, 64, 1)
    assert np.count_nonzero(f == 4) > 2 * case.nx  # the hill adds walls above the ground row


def test_immersed_boundary_set_up(tmp_path):
    for builder in ("small_2d_topo", "small_3d_topo"):
        case = Case(getattr(configs, builder)(tmp_path, immb=1))
        ib = case.ib
        f = case.flag
        ibc = np.flatnonzero((f == 257) | (f == 512) | (f == 1024))
        assert ibc.size > 0
        forced = (ib.num[0][ibc] != 0) | (ib.num[1][ibc] != 0) | (ib.num[2][ibc] != 0)
        assert forced.all()  # bdry.f:111-113 stops on an unforced one
        # the numbering covers every forcing point of each axis once
        for a, lst in enumerate((ib.fptx, ib.fpty, ib.fptz)):
            nums = ib.num[a][ib.num[a] != 0]
            assert len(np.unique(nums)) == nums.size
            assert nums.size <= len(lst)
        # the face factors: bits of the six faces, ivf = 1 / vf for open cells
        fluid = (f & 1) == 1
        assert np.all((ib.faces >= 0) & (ib.faces <= 63))
        sel = fluid & (ib.vf > 0)
        if ib.stopped_at < 0:
            np.testing.assert_allclose(ib.ivf[sel], 1.0 / ib.vf[sel], rtol=0)
        assert np.any(ib.faces[fluid] != 63)  # some faces are closed by the topography


def test_deck_checks():
    d = configs.plume_2d()
    d.set("topography", itp=2)
    assert any("itp" in b for b in d.check())
    d = configs.small_2d_rk3()
    d.set("topography", itp=1)
    d.set("boundaries", immb=1)
    assert any("explicit solver" in b for b in d.check())
    d = configs.plume_2d()
    d.set("topography", itp=1)
    assert not d.check()


@pytest.mark.parametrize("builder,immb", [("small_2d_topo", 0), ("small_2d_topo", 1), ("small_3d_topo", 1)])
def test_oracle_steps_on_topography(tmp_path, builder, immb):
    import pyoracle
    case = Case(getattr(configs, builder)(tmp_path, immb=immb))
    ora = pyoracle.Oracle(case)
    for s in range(1, 6):
        ora.step(s)
    st = ora.get_state()
    assert all(np.all(np.isfinite(v)) for v in st.values())
