"""The compiled time-loop driver (pdac_run, prog.f:143-417 over the C ABI)
against the Python one (pdac_b200.files.run) on the GPU: the same case
produces the same files, byte for byte (both call the same engine entry
points in prog.f's order), from scratch and when restarted from their own
pdac.res, for the semi-implicit path with the ground sink, the mixture
fields and text output, and for the explicit solver."""
import filecmp
import os
import subprocess

import pytest

from sink_decks import seeded_case

pytestmark = pytest.mark.gpu


def _python_run(case, workdir, steps):
    from pdac_b200 import files
    from pdac_b200.engine import Engine
    eng = Engine(case)
    out = files.run(eng, workdir, max_steps=steps)
    eng.close()
    return out


def _compiled_run(case, workdir, steps):
    from pdac_b200 import build, casefile
    exe = build.build_host()
    os.makedirs(workdir, exist_ok=True)
    path = casefile.write(case, os.path.join(workdir, "..", os.path.basename(workdir) + ".case"))
    r = subprocess.run([exe, path, workdir, str(steps)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return r.stdout


def _same_files(a, b):
    names = sorted(os.listdir(a))
    assert names == sorted(os.listdir(b))
    for name in names:
        assert filecmp.cmp(os.path.join(a, name), os.path.join(b, name), shallow=False), name
    return names


def _edit(dt, restart=False, formatted=False):
    # a restart reads massl.NNNN of the namelist's nfil (setup.f:147): the
    # last one written before pdac.res, at step 4, is massl.0002
    def edit(d):
        d.set("control", tpr=2 * dt, tdump=2 * dt, imr=1, tstop=1.0, formatted_output=formatted,
              restart_mode="restart" if restart else "from_scratch", nfil=2 if restart else 0)
        d.set("model", compute_mixture=True)
    return edit


@pytest.mark.parametrize("builder,formatted", [("small_2d_sink", True), ("small_3d_sink", False),
                                               ("small_2d_rk3", False)])
def test_compiled_driver_writes_the_python_drivers_files(builder, formatted, tmp_path):
    from pdac_b200 import configs
    dt = getattr(configs, builder)()["dt"]
    kw = {"irand": 0} if "2d" in builder else {}
    a, b = str(tmp_path / "py"), str(tmp_path / "cc")
    _python_run(seeded_case(builder, edit=_edit(dt, formatted=formatted), **kw), a, 5)
    out = _compiled_run(seeded_case(builder, edit=_edit(dt, formatted=formatted), **kw), b, 5)
    assert "Iteration:      5" in out
    names = _same_files(a, b)
    assert "pdac.res" in names and "pdac.chm" in names and "output.0002" in names
    if "sink" in builder:
        assert "massl.0001" in names and "massl.res" in names
    # restart both from their own pdac.res (and massl file) for two more steps
    _python_run(seeded_case(builder, edit=_edit(dt, restart=True, formatted=formatted), **kw), a, 2)
    _compiled_run(seeded_case(builder, edit=_edit(dt, restart=True, formatted=formatted), **kw), b, 2)
    _same_files(a, b)
