"""The mixed-precision mode (PDAC_PREC_MIXED) against the FP64 form of the
same run on the GPU.

In the mixed mode the flux passes (momentum, mass, scalar and enthalpy face
fluxes: flux_u/v/w.f, flux_m.f, flux_sc.f, hotc.f; 2D and 3D, both time
integrations) compute in FP32 from
the FP64 state and store their fluxes in FP64; everything else, including
the conservative updates and the pressure correction, stays in FP64.  The
fields stay within 1e-5 relative L-inf of the FP64 run (measured: a few
1e-7 over tens of steps, not growing), the phase masses within 1e-8 and the
species masses within 1e-6 relative (a face flux is shared by its two cells,
so only the flows through the open boundaries differ: their FP32 fluxes
carry ~1e-7 relative error, and over tens of steps the mass that crossed
the boundary of the small 2D deck moves the gas mass by 2e-9).  The fields must also differ from the
FP64 run: that shows the FP32 kernels ran."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-5
PHASE_MASS_TOL = 1e-8
SPECIES_MASS_TOL = 1e-6
FIELDS = ("p", "ep", "rlk", "ug", "vg", "wg", "us", "vs", "ws", "tg", "ts", "ygc")


def _rel_linf(a, b):
    scale = float(np.max(np.abs(b)))
    diff = float(np.max(np.abs(a - b)))
    return diff / scale if scale > 0 else diff  # an all-zero field (vg, vs in 2D)


@pytest.mark.parametrize("builder,kw,steps", [
    ("small_2d", {}, 20),
    ("small_2d_rk3", {}, 30),
    ("plume_2d", {"nx": 64, "nz": 96}, 20),
    ("small_3d", {}, 12),
    ("small_3d_rk3", {}, 30),
    ("plume_3d", {"nx": 32, "ny": 32, "nz": 24}, 10),
    ("plume_3d_rk3", {"nx": 32, "ny": 32, "nz": 24}, 30),
])
def test_mixed_matches_fp64(builder, kw, steps):
    from pdac_b200 import abi, configs
    from pdac_b200.engine import Engine
    from pdac_b200.setup_state import Case
    e64 = Engine(Case(getattr(configs, builder)(**kw)))
    emx = Engine(Case(getattr(configs, builder)(**kw), precision=abi.PREC_MIXED))
    for s in range(1, steps + 1):
        e64.step(s)
        emx.step(s)
    a, b = emx.download(), e64.download()
    errs = {k: _rel_linf(a[k], b[k]) for k in FIELDS if k in b}
    assert max(errs.values()) <= FIELD_TOL, errs
    assert errs["ug"] > 0 and errs["wg"] > 0, "the mixed run equals the FP64 run: its FP32 kernels did not run"
    ma, mb = emx.mass_totals(), e64.mass_totals()
    nph = 1 + e64.case.nsolid
    np.testing.assert_allclose(ma[:nph], mb[:nph], rtol=PHASE_MASS_TOL, atol=0)
    np.testing.assert_allclose(ma[nph:], mb[nph:], rtol=SPECIES_MASS_TOL, atol=0)
    e64.close()
    emx.close()


def test_mixed_ensemble_members_in_a_batch():
    """Mixed-precision members of the 2D ensemble's distribution stepped in a
    batch (one graph) give the bits of the same mixed decks stepped alone,
    and stay within the field tolerance of their FP64 runs."""
    from pdac_b200 import abi
    from pdac_b200.engine import Engine
    from pdac_b200.ensemble import Batch, member_decks, member_params
    from pdac_b200.setup_state import Case
    decks = []
    for m in range(3):
        p = member_params(m)
        decks += member_decks(1, first=m, nx=max(16, p["nx"] // 4), nz=max(24, p["nz"] // 4))
    steps = 6
    engines = [Engine(Case(d, precision=abi.PREC_MIXED)) for d in decks]
    b = Batch(engines)
    got_nit = [b.step(s) for s in range(1, steps + 1)]
    got = [e.download() for e in engines]
    b.close()
    for e in engines:
        e.close()
    for m, d in enumerate(decks):
        alone = Engine(Case(d, precision=abi.PREC_MIXED))
        e64 = Engine(Case(d))
        nits = [alone.step(s) for s in range(1, steps + 1)]
        for s in range(1, steps + 1):
            e64.step(s)
        ref, r64 = alone.download(), e64.download()
        alone.close()
        e64.close()
        assert [row[m] for row in got_nit] == nits, m
        for name, v in ref.items():
            np.testing.assert_array_equal(got[m][name], v, err_msg=f"member {m} field {name}")
        errs = {k: _rel_linf(ref[k], r64[k]) for k in FIELDS if k in r64}
        assert max(errs.values()) <= FIELD_TOL, (m, errs)
