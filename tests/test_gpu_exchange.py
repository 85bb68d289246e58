"""pdac_gpu_exchange_state: the download of one step's result and the upload
of the next step's inputs in one call, the two copy directions overlapped.

Checked against the separate calls it stands for: with out and in the same
view (the host hands back what it read) the downloaded fields are those of
pdac_gpu_download_state and the next steps give the bits of a context that
was never exchanged; with two views the device ends with in's fields while
out receives the old ones; a NaN in in is refused as an upload refuses it.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(is3d):
    from pdac_b200 import configs
    from pdac_b200.setup_state import Case
    return Case(configs.small_3d() if is3d else configs.small_2d())


def _engines(is3d):
    from pdac_b200.engine import Engine
    return Engine(_case(is3d)), Engine(_case(is3d))


def _pinned_like(state):
    return {k: np.array(v, dtype=np.float64, copy=True) for k, v in state.items()}


@pytest.mark.parametrize("is3d", [False, True])
def test_exchange_with_one_view_equals_download_then_upload(is3d):
    from pdac_b200 import abi
    eng, ref = _engines(is3d)
    L = eng.L
    host = _pinned_like(eng.case.state)
    view = abi.make_state_view(host)
    for s in (1, 2):
        eng.step(s)
        ref.step(s)
    assert L.pdac_gpu_exchange_state(eng.h, C.byref(view), C.byref(view)) == 0
    want = ref.download()
    for k, v in want.items():
        assert np.array_equal(host[k], v), k
    for s in (3, 4):
        n1, n2 = eng.step(s), ref.step(s)
        assert n1 == n2
    a, b = eng.download(), ref.download()
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    eng.close()
    ref.close()


def test_exchange_with_two_views_swaps_the_state():
    from pdac_b200 import abi
    eng, ref = _engines(False)
    L = eng.L
    eng.step(1)
    ref.step(1)
    ref.step(2)
    nxt = ref.download()  # the state after step 2 of the other context
    out = {k: np.zeros_like(v) for k, v in eng.case.state.items()}
    vin, vout = abi.make_state_view(nxt), abi.make_state_view(out)
    want_out = eng.download()
    assert L.pdac_gpu_exchange_state(eng.h, C.byref(vout), C.byref(vin)) == 0
    for k in want_out:
        assert np.array_equal(out[k], want_out[k]), k
    got = eng.download()
    for k in nxt:
        assert np.array_equal(got[k], nxt[k]), k
    eng.close()
    ref.close()


def test_exchange_refuses_a_nan_in_the_upload():
    from pdac_b200 import abi
    eng, other = _engines(False)
    other.close()
    L = eng.L
    eng.step(1)
    bad = _pinned_like(eng.case.state)
    bad["tg"][len(bad["tg"]) // 2] = np.nan
    out = {k: np.zeros_like(v) for k, v in eng.case.state.items()}
    st = L.pdac_gpu_exchange_state(eng.h, C.byref(abi.make_state_view(out)), C.byref(abi.make_state_view(bad)))
    assert st == abi.PDAC_ERR_NONFINITE
    assert b"tg" in (L.pdac_gpu_last_error(eng.h) or b"")
    eng.close()
