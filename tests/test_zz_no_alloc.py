"""pdac_gpu_iter_static against pdac_gpu_iter, both through the C ABI.

The static-scratch variant runs the same kernels on the same inputs; only
the placement of the corrector's scratch differs, so two engines set up
from the same deck must agree after each of two consecutive time steps
(tolerance 1e-12 relative L-infinity, same outer-sweep counts).
"""
import ctypes as C

import pytest

from helpers import STEP_FIELDS, compare_state

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _bind(lib):
    lib.pdac_gpu_iter_static.argtypes = [C.c_void_p, C.c_double, C.POINTER(C.c_int)]
    lib.pdac_gpu_iter_static.restype = C.c_int


def _step(eng, sweep, static):
    L = eng.L
    dt = eng.case.deck["dt"]
    eng.boundary(sweep)
    eng.fieldn()
    eng.tilde(dt)
    nit = C.c_int(0)
    fn = L.pdac_gpu_iter_static if static else L.pdac_gpu_iter
    st = fn(eng.h, dt, C.byref(nit))
    assert st == 0, (L.pdac_gpu_last_error(eng.h) or b"").decode()
    eng.ygas(dt)
    eng.htilde(dt)
    eng.ftem(dt)
    return nit.value


@pytest.mark.parametrize("which", ["2d", "3d"])
def test_static_scratch_iter_matches_iter(which):
    from pdac_b200 import configs
    from pdac_b200.engine import Engine
    from pdac_b200.setup_state import Case
    case = Case(configs.small_2d() if which == "2d" else configs.small_3d())
    ref, new = Engine(case), Engine(case)
    _bind(new.L)
    fields = STEP_FIELDS + (("vg", "vs") if case.is3d else ())
    for sweep in (1, 2):
        n_ref = _step(ref, sweep, static=False)
        n_new = _step(new, sweep, static=True)
        assert n_new == n_ref, f"step {sweep}: outer sweeps {n_new} vs {n_ref}"
        errs, bad = compare_state(new.download(), ref.download(), fields, TOL, case.nsolid, case.ncell)
        assert not bad, f"step {sweep}: {bad}"
    ref.close()
    new.close()


def _scratch_bytes(nx, ny, nz):
    """The static variant's scratch for a mesh (the header's formula)."""
    wl = 4 * ((nx + 2) // 3) * ny * nz
    wl = (wl + 255) // 256 * 256
    return 256 + 2 * wl + 4 * ((nx * ny * nz + 31) // 32)


def test_static_scratch_near_its_bound():
    """A 2D plume of 1600 x 1850 cells (2.96 M) needs 98.6 % of the 8 MiB
    array: one step through pdac_gpu_iter_static equals one through
    pdac_gpu_iter."""
    from pdac_b200 import configs
    from pdac_b200.engine import Engine
    from pdac_b200.setup_state import Case
    nx, nz = 1600, 1850
    need = _scratch_bytes(nx, 1, nz)
    assert 0.98 * 8 * 1024 * 1024 < need <= 8 * 1024 * 1024
    case = Case(configs.plume_2d(nx=nx, nz=nz))
    ref, new = Engine(case), Engine(case)
    _bind(new.L)
    n_ref = _step(ref, 1, static=False)
    n_new = _step(new, 1, static=True)
    assert n_new == n_ref
    errs, bad = compare_state(new.download(), ref.download(), STEP_FIELDS, TOL, case.nsolid, case.ncell)
    assert not bad, bad
    ref.close()
    new.close()


def test_static_scratch_rejects_a_mesh_that_does_not_fit():
    from pdac_b200 import configs
    from pdac_b200.engine import Engine
    from pdac_b200.setup_state import Case
    case = Case(configs.plume_2d(nx=2000, nz=1900))
    eng = Engine(case)
    _bind(eng.L)
    nit = C.c_int(-1)
    st = eng.L.pdac_gpu_iter_static(eng.h, case.deck["dt"], C.byref(nit))
    msg = (eng.L.pdac_gpu_last_error(eng.h) or b"").decode()
    assert st == 6  # PDAC_ERR_ARG
    assert "static scratch" in msg and "limit" in msg
    assert nit.value == -1
    eng.close()
