"""The launch-shape autotuner (pdac_gpu_autotune / pdac_gpu_set_tuning):
shapes change only the speed, never a result, and tuning leaves the state
the caller sees as it was.

* Every form of the 3D momentum-flux pass (per-thread gathers, four tile
  shapes, several march chunks) gives the same bits as the default form.
* A run that tunes after its second step agrees bit for bit with one that
  does not, in 3D (flux tile, corrector grids) and in 2D (cells per block of
  the one-launch sweep loop); the chosen shapes land in the cache file and a
  second context with the same key installs them without timing.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(deck_builder, steps, tune_after=None, tuning=None, cache=None, **kw):
    from pdac_b200.engine import Engine
    from pdac_b200.setup_state import Case
    e = Engine(Case(deck_builder(**kw)))
    if tuning is not None:
        e.set_tuning(tuning)
    nits, chosen = [], None
    for s in range(1, steps + 1):
        nits.append(e.step(s))
        if tune_after == s:
            chosen = e.autotune(cache)
    out = e.download()
    e.close()
    return nits, out, chosen


def _same(a, b):
    assert a[0] == b[0], (a[0], b[0])
    for k in a[1]:
        np.testing.assert_array_equal(a[1][k], b[1][k], err_msg=k)


def test_every_tile_shape_gives_the_same_bits():
    from pdac_b200 import configs
    kw = dict(nx=40, ny=21, nz=30, vent_cells=4)
    ref = _run(configs.plume_3d, 3, **kw)
    for shape in range(5):
        for kchunk in (1, 7, 30):
            t = dict(tile_shape=shape, tile_kchunk=kchunk, inner_grid=148 * 16, test_grid=148 * 8,
                     coop_cells_per_block=1024)
            _same(_run(configs.plume_3d, 3, tuning=t, **kw), ref)


@pytest.mark.parametrize("which", ["3d", "2d"])
def test_tuning_changes_no_result(which, tmp_path):
    from pdac_b200 import configs
    if which == "3d":
        builder, kw = configs.plume_3d, dict(nx=48, ny=40, nz=36, vent_cells=4)
    else:
        builder, kw = configs.plume_2d, dict(nx=64, nz=96)
    cache = str(tmp_path / "tune.txt")
    ref = _run(builder, 5, **kw)
    tuned = _run(builder, 5, tune_after=2, cache=cache, **kw)
    _same(tuned, ref)
    lines = open(cache).read().splitlines()
    assert len(lines) == 1 and " | " in lines[0]
    again = _run(builder, 5, tune_after=2, cache=cache, **kw)
    assert again[2] == tuned[2]
    assert len(open(cache).read().splitlines()) == 1  # found, not tuned again
    _same(again, ref)


def test_set_tuning_rejects_bad_values():
    from pdac_b200 import configs
    from pdac_b200.engine import Engine, PdacError
    from pdac_b200.setup_state import Case
    e = Engine(Case(configs.small_3d()))
    with pytest.raises(PdacError):
        e.set_tuning(dict(tile_shape=9, tile_kchunk=8, inner_grid=64, test_grid=32, coop_cells_per_block=1024))
    e.close()
