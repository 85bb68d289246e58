"""The mixed-precision mode (PDAC_PREC_MIXED) against the FP64 form of the
same run on the GPU.

In the mixed mode the 3D flux passes (momentum, mass, scalar and enthalpy
face fluxes: flux_u/v/w.f, flux_m.f, flux_sc.f, hotc.f) compute in FP32 from
the FP64 state and store their fluxes in FP64; everything else, including
the conservative updates and the pressure correction, stays in FP64.  The
fields stay within 1e-5 relative L-inf of the FP64 run (measured: a few
1e-7 over tens of steps, not growing), the phase masses within 1e-9 and the
species masses within 1e-6 relative (a face flux is shared by its two cells,
so only the boundary flows differ).  The fields must also differ from the
FP64 run: that shows the FP32 kernels ran."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-5
PHASE_MASS_TOL = 1e-9
SPECIES_MASS_TOL = 1e-6
FIELDS = ("p", "ep", "rlk", "ug", "vg", "wg", "us", "vs", "ws", "tg", "ts", "ygc")


def _rel_linf(a, b):
    scale = float(np.max(np.abs(b)))
    return float(np.max(np.abs(a - b))) / scale


@pytest.mark.parametrize("builder,kw,steps", [
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
    errs = {k: _rel_linf(a[k], b[k]) for k in FIELDS}
    assert max(errs.values()) <= FIELD_TOL, errs
    assert errs["ug"] > 0 and errs["wg"] > 0, "the mixed run equals the FP64 run: its FP32 kernels did not run"
    ma, mb = emx.mass_totals(), e64.mass_totals()
    nph = 1 + e64.case.nsolid
    np.testing.assert_allclose(ma[:nph], mb[:nph], rtol=PHASE_MASS_TOL, atol=0)
    np.testing.assert_allclose(ma[nph:], mb[nph:], rtol=SPECIES_MASS_TOL, atol=0)
    e64.close()
    emx.close()
