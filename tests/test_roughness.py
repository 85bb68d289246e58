"""The sub-grid model's mixing length with ground roughness (iturb = 2,
turbo.f:72-108, roughness.f:12-36) in the oracle, against a restatement
written here from the reference loop: for every cell in flat-index order,
ls = cmut delta (delta = sqrt(dz dx) in 2D, (dz dy dx)^(1/3) in 3D); a cell
whose centre is zsgs = z(k) - topo_c(i[, j]) > 0 above the ground takes
lm = sqrt(1 / (1 / ls^2 + 1 / lb^2)) with lb = 0.4 (zsgs + zrough), any
other cell keeps the previous cell's lm; smag = lm^2, times the anisotropy
factor in 3D.  Decks: the 2D hill profile with and without immersed
boundaries (whose interpolated profile replaces the staircase level) and
the 3D hills DEM with immersed boundaries.
"""
import math

import numpy as np
import pytest


def _deck(tmp_path, builder, immb, zrough):
    from pdac_b200 import configs
    d = getattr(configs, builder)(tmp_path, immb=immb)
    d.set("model", iturb=2, modturbo=1, iss=0)
    d.set("topography", zrough=zrough)
    return d


def _anis(dx, dy, dz):
    # turbo.f:670-700
    dmax = max(dx, dy, dz)
    la1, la2, la3 = math.log(dx / dmax), math.log(dy / dmax), math.log(dz / dmax)
    fla = la1 * la1 + la2 * la2 + la3 * la3 - la1 * la2 + la1 * la3 - la2 * la3
    return math.cosh(math.sqrt(4.0 / 27.0 * fla))


def _smag(case):
    cfg = case.cfg()
    nx, ny, nz = case.nx, case.ny, case.nz
    dx, dy, dz = case.dx, case.dy, case.dz
    topo = np.array([cfg.topo_c[q] for q in range(nx * (ny if case.is3d else 1))])
    out = np.zeros(case.ncell)
    lm = 0.0
    for c in range(case.ncell):
        i, j, k = c % nx, (c // nx) % ny, c // (nx * ny)
        if case.is3d:
            delt = (dz[k] * dy[j] * dx[i]) ** (1.0 / 3.0)
            zsgs = case.z[k] - topo[j * nx + i]
        else:
            delt = math.sqrt(dz[k] * dx[i])
            zsgs = case.z[k] - topo[i]
        ls = cfg.cmut * delt
        if zsgs > 0.0:
            lb = 0.4 * (zsgs + cfg.zrough)
            lm = math.sqrt(1.0 / (1.0 / ls ** 2 + 1.0 / lb ** 2))
        out[c] = lm * lm
        if case.is3d:
            out[c] *= _anis(dx[i], dy[j], dz[k])
    return out


@pytest.mark.parametrize("builder,immb", [("small_2d_topo", 0), ("small_2d_topo", 1), ("small_3d_topo", 1)])
def test_oracle_mixing_length_with_roughness(tmp_path, builder, immb):
    import pyoracle
    from pdac_b200.setup_state import Case
    case = Case(_deck(tmp_path, builder, immb, zrough=2.0))
    ora = pyoracle.Oracle(case)
    got, want = ora.get("smag"), _smag(case)
    fluid = (case.flag & 1) == 1
    # the fluid cells (the only ones the model reads) to round-off of pow and
    # the order of the operations in the restatement; above the ground the
    # roughness length shortens the Smagorinsky one
    assert np.allclose(got[fluid], want[fluid], rtol=1e-13, atol=0.0)
    iturb1 = _deck(tmp_path, builder, immb, zrough=2.0)
    iturb1.set("model", iturb=1)
    ls2 = pyoracle.Oracle(Case(iturb1)).get("smag")
    assert np.all(got[fluid] < ls2[fluid])
