"""Input deck reader: namelist defaults, parsing and the MESH/FIXED_FLOWS cards."""
import numpy as np
import pytest

from pdac_b200 import configs
from pdac_b200.deck import Deck, f32
from pdac_b200.setup_state import Case, FLUID, SLIP, NOSLIP, FREE_IO, VENT


def test_single_precision_defaults():
    d = Deck()
    assert d["omega"] == float(np.float32(1.1)) != 1.1
    assert d["maxout"] == 500 and d["inmax"] == 8 and d["delg"] == 1e-8
    assert d["alpha"] == 1.0 and d["pmodel"] == 2 and d["icpc"] == 2


def test_round_trip_text():
    d = configs.plume_2d(nx=10, nz=12)
    d.set("mesh", iuni=0)
    d.delta_x = np.full(10, 10.0)
    d.delta_z = np.full(12, 12.5)
    d.blocks = [dict(typ=5, xlo=2, xhi=3, ylo=0, yhi=0, zlo=1, zhi=1, ug=0.0, vg=0.0, wg=50.0, p=1.01e5,
                     ep=0.99, tg=900.0, solids=[dict(u=0.0, v=0.0, w=50.0, eps=0.005, t=900.0)] * 2,
                     ygc=[0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0])]
    d2 = Deck.parse(d.to_text())
    for g in d.nml:
        for k, v in d.nml[g].items():
            assert d2.nml[g][k] == v, (g, k)
    np.testing.assert_array_equal(d2.delta_z, d.delta_z)
    assert d2.blocks[0]["typ"] == 5 and d2.blocks[0]["wg"] == 50.0


HAND_DECK = """
 &control
   run_name = 'tube', job_type = '2D', dt = 0.005D0, tstop = 1.0
 /
 &model
   iturb = 0, ngas = 1
 /
 &mesh
   nx = 8, nz = 10, itc = 0, iuni = 1, dx0 = 5.0, dz0 = 5.0
 /
 &boundaries
   west = 3, east = 3, bottom = 3, top = 3
 /
 &topography
 /
 &inlet
 /
 &dome
 /
 &atmosphere
   stratification = .FALSE.
 /
 &particles
   nsolid = 1, diameter = 200, density = 2500.
 /
 &numeric
   muscl = 1, maxout = 300
 /
MESH
FIXED_FLOWS
0
"""


def test_parse_hand_written_deck_and_set_up_a_closed_box():
    d = Deck.parse(HAND_DECK)
    assert d["dt"] == 0.005 and d["nx"] == 8 and d["diameter"][0] == 200.0
    case = Case(d)
    f = case.flag.reshape(case.nz, case.nx)
    assert (f[0, 1:-1] == NOSLIP).all() and (f[-1, 1:-1] == NOSLIP).all()
    assert (f[:, 0] == NOSLIP).all()
    # export_topography (topo.f:1114-1181): the three rows above the no-slip
    # ground are boundary-layer cells
    assert (f[1:4, 1:-1] == 5).all() and (f[4:-1, 1:-1] == FLUID).all()
    assert case.gas_type == [6]


def test_plume_vent_and_flags():
    case = Case(configs.plume_2d())
    f = case.flag.reshape(case.nz, case.nx)
    assert (f[:, 0] == SLIP).all()                    # axis
    assert (f[1:, -1] == FREE_IO).all() and (f[-1, 1:-1] == FREE_IO).all()
    vent_i = [v["i"] for v in case.vent]
    assert vent_i == [2, 3, 4, 5, 6]                   # r in [0, 50] m with 10 m cells
    assert all(f[0, i - 1] == VENT for i in vent_i)
    # boundary-layer rows (topo.f:1114-1181): three above the no-slip ground,
    # two above the vent, whose columns hold no no-slip cell and keep the
    # starting row 0
    assert (f[1:4, 6:-1] == 5).all() and (f[4:-1, 6:-1] == FLUID).all()
    assert (f[1:3, 1:6] == 5).all() and (f[3:-1, 1:6] == FLUID).all()
    assert case.gas_type == [5, 6]                     # H2O, Air (gas_check order)
    st = case.state
    c = case.vent[0]["ijk"]
    assert st["tg"][c] == 1100.0 and st["wg"][c] == 100.0 and st["ygc"][c] == 1.0


def test_unsupported_options_are_rejected():
    d = configs.plume_2d()
    d.set("model", iturb=3)
    with pytest.raises(ValueError, match="iturb"):
        Case(d)
    d = configs.plume_3d(nx=8, ny=8, nz=8)
    d.set("model", iturb=1, modturbo=3)
    with pytest.raises(ValueError, match="modturbo"):
        Case(d)


def test_sub_grid_model_reaches_the_configuration():
    d = configs.plume_2d()
    d.set("model", iturb=1, iss=1, cmut=0.2)
    cfg = Case(d).cfg()
    assert (cfg.iturb, cfg.modturbo, cfg.iss, cfg.cmut) == (1, 1, 1, 0.2)
    d = configs.plume_3d(nx=8, ny=8, nz=8)
    d.set("model", iturb=1, modturbo=2)
    assert Case(d).cfg().modturbo == 2


def test_ground_roughness_reaches_the_configuration():
    d = configs.plume_2d()
    d.set("model", iturb=2)
    d.set("topography", zrough=0.5)
    case = Case(d)
    cfg = case.cfg()
    assert cfg.iturb == 2 and cfg.zrough == 0.5
    # flat ground: the top of the no-slip bottom row under every column
    assert [cfg.topo_c[i] for i in range(case.nx)] == [case.zb[0]] * case.nx


def test_explicit_solver_selection():
    """time_integration = 1 selects the explicit SSP-RK3 solver; it needs
    pmodel 1 or 2 (compute_rhs, explicit_solver.f:632-642) and reaches the
    C configuration struct."""
    d = configs.plume_2d_rk3()
    case = Case(d)
    assert case.cfg().time_integration == 1
    d.set("model", pmodel=0)
    with pytest.raises(ValueError, match="pmodel"):
        Case(d)
    d = configs.plume_2d()
    d.set("numeric", time_integration=2)
    with pytest.raises(ValueError, match="time_integration"):
        Case(d)
    assert Case(configs.plume_2d()).cfg().time_integration == 0


def test_implicit_flux_modes_reach_the_configuration():
    d = configs.small_2d_implicit(fluxes=True, enthalpy=False)
    cfg = Case(d).cfg()
    assert (cfg.implicit_fluxes, cfg.implicit_enthalpy) == (1, 0)
    d = configs.small_2d_implicit()
    d.set("numeric", alpha=0.5)
    with pytest.raises(ValueError, match="implicit_fluxes"):
        Case(d)


def test_inner_loop_variants():
    assert Case(configs.small_2d_opt()).cfg().optimization == 2
    assert Case(configs.small_2d_opt(optimization=3)).cfg().optimization == 3  # runs as 2 in 2D
    d = configs.small_3d(diameters=(30.0, 250.0), ep_solid=(0.005, 0.01))
    d.set("numeric", optimization=3)
    with pytest.raises(ValueError, match="optimization=3"):
        Case(d)


def test_generated_mesh():
    """generate_grid (grid.f:485-786): a band of n0 cells of the minimum
    size at the relative position alpha, sizes growing at one rate to the
    maximum, the domain filled to the mesh's 1e-4 rounding."""
    from pdac_b200.setup_state import generate_grid
    dz = generate_grid(110, 1000.0, 0.0, 5.0, 40.0, 81, 1.2)
    assert len(dz) == 110 and np.all(dz[:81] == 5.0) and dz.max() == 40.0
    assert np.all(np.diff(dz) >= -1e-9)  # growing away from the band at the bottom
    assert abs(dz.sum() - 1000.0) < 0.5
    assert np.allclose(dz * 1e4, np.round(dz * 1e4), rtol=0, atol=1e-6)
    dx = generate_grid(200, 4000.0, 0.5, 10.0, 40.0, 40, 1.2)
    c = np.argmin(dx)
    assert dx.min() == 10.0 and np.count_nonzero(dx == 10.0) == 40 and abs(dx.sum() - 4000.0) < 1.0
    assert np.all(generate_grid(10, 100.0, 0.5, 10.0, 10.0, 1, 1.2) == 10.0)
