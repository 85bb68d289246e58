"""The C-ABI library loads without a GPU and exports every declared symbol."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pdac_gpu.h")


def declared_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"\b(pdac_gpu_\w+)\s*\(", txt)))


def test_header_declares_the_time_loop_calls():
    syms = declared_symbols()
    for name in ("boundary", "fieldn", "tilde", "iter", "ygas", "htilde", "ftem", "step",
                 "create", "destroy", "upload_state", "download_state"):
        assert f"pdac_gpu_{name}" in syms


def test_library_exports_all_declared_symbols():
    from pdac_b200 import build, engine
    build.build()
    lib = C.CDLL(engine.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    assert set(engine.EXPORTED) <= set(declared_symbols())


def test_struct_layout_matches_header():
    """ctypes mirror sizes equal the C sizes (checked with the host compiler)."""
    import subprocess
    import tempfile
    from pdac_b200 import abi
    src = ('#include "pdac_gpu.h"\n#include <stdio.h>\n#include <stddef.h>\n'
           'int main(){printf("%zu %zu %zu %zu\\n", sizeof(pdac_cfg), sizeof(pdac_state_view),'
           ' offsetof(pdac_cfg, precision), offsetof(pdac_cfg, vent_ijk));return 0;}\n')
    with tempfile.TemporaryDirectory() as d:
        cfile = os.path.join(d, "t.c")
        open(cfile, "w").write(src)
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), cfile, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    assert int(out[0]) == C.sizeof(abi.PdacCfg)
    assert int(out[1]) == C.sizeof(abi.PdacStateView)
    assert int(out[2]) == abi.PdacCfg.precision.offset
    assert int(out[3]) == abi.PdacCfg.vent_ijk.offset


def test_create_rejects_bad_config_without_touching_the_gpu():
    from pdac_b200 import abi, engine
    L = engine.lib()
    cfg = abi.PdacCfg()
    cfg.job_type = 2
    cfg.nx = 2  # too small
    h = C.c_void_p()
    assert L.pdac_gpu_create(C.byref(cfg), C.byref(h)) == abi.PDAC_ERR_CONFIG


def test_unknown_precision_is_rejected_without_touching_the_gpu():
    from pdac_b200 import abi, configs, engine
    from pdac_b200.setup_state import Case
    L = engine.lib()
    case = Case(configs.small_2d(), precision=abi.PREC_MIXED)
    cfg = case.cfg()
    h = C.c_void_p()
    cfg.precision = 7
    assert L.pdac_gpu_create(C.byref(cfg), C.byref(h)) == abi.PDAC_ERR_CONFIG


@pytest.mark.parametrize("nx", [9, 10, 11])
def test_colour_phase_fits_the_worklist_bound(nx):
    """A colour phase of the corrector ((i + j + k) mod 3, 1-based) holds at
    most ceil(nx / 3) * ny * nz cells: the per-colour worklists of
    pdac_gpu_iter and the static scratch of pdac_gpu_iter_static are sized
    by that bound."""
    import numpy as np
    ny, nz = 7, 8
    i, j, k = np.meshgrid(np.arange(1, nx + 1), np.arange(1, ny + 1), np.arange(1, nz + 1), indexing="ij")
    col = (i + j + k) % 3
    most = max(int(np.count_nonzero(col == c)) for c in range(3))
    assert most <= (nx + 2) // 3 * ny * nz
