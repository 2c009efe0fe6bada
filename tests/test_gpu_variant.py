"""The 2014 variant (trunk/lomacte/src/cross.f: spectral T, d(rho) from a
transform round trip of T and Delta T, Dirichlet psi, cumulative-trapezoid
rho v00) on the GPU against the FP64 oracle's restatement of it.

Bars (FP64): 1 RK3 step <= 1e-10 relative L2 per field, 20 steps <= 1e-9
with the momentum thickness equal to 1e-9; in the CFL mode the Deltat
sequence is identical.
"""
import numpy as np
import pytest

from loma_phd_b200 import Lomacte, LomacteError
from tests.helpers import FIELDS, case, oracle_for, rel_l2

pytestmark = pytest.mark.gpu


def _pair(p, y, st, n, hist=False):
    g = Lomacte(p, y)
    assert g.y_family == "mode" and g.launches_per_step == 43
    g.load_state(st)
    o = oracle_for(p, y, st)
    hg, ho = [], []
    for _ in range(n):
        g.step(1)
        o.step(1)
        if hist:
            hg.append(g.diag())
            ho.append(o.diag())
    sg, so = g.get_state(), o.get_state()
    g.close()
    return sg, so, hg, ho


@pytest.mark.parametrize("grid", [(24, 24, 33), (32, 32, 65)])
def test_variant_one_step(gpu, grid):
    p, y, st = case(*grid, variant=1)
    sg, so, _, _ = _pair(p, y, st, 1)
    for k in FIELDS:
        assert rel_l2(sg[k], so[k]) < 1e-10, (k, rel_l2(sg[k], so[k]))
    for k in ("u00", "v00"):
        assert rel_l2(sg[k], so[k]) < 1e-10, (k, rel_l2(sg[k], so[k]))


def test_variant_twenty_steps(gpu):
    p, y, st = case(32, 32, 65, variant=1)
    sg, so, hg, ho = _pair(p, y, st, 20, hist=True)
    for k in FIELDS:
        assert rel_l2(sg[k], so[k]) < 1e-9, (k, rel_l2(sg[k], so[k]))
    a = np.array([h["dm"] for h in hg])
    b = np.array([h["dm"] for h in ho])
    assert np.abs(a - b).max() < 1e-9
    for key in ("trapz", "massu", "time"):
        assert abs(hg[-1][key] - ho[-1][key]) <= 1e-9 * max(1.0, abs(ho[-1][key])), key


def test_variant_cfl_mode(gpu):
    p, y, st = case(24, 24, 33, variant=1, dt_mode=0, dt=1e-4, ncfl=2)
    sg, so, hg, ho = _pair(p, y, st, 5, hist=True)
    assert [h["Deltat"] for h in hg] == [h["Deltat"] for h in ho]
    for k in FIELDS:
        assert rel_l2(sg[k], so[k]) < 1e-9, k


def test_variant_is_fp64_only(gpu):
    p, y, st = case(24, 24, 33, variant=1, precision=1)
    with pytest.raises(LomacteError):
        Lomacte(p, y)
