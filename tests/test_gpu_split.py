"""The slab decomposition of the transform stage on one device
(lmc_step_split; change.f:1-211): each block's z transforms over its kx
planes, its x stage over its (z, y) lines, and the plane <-> line exchanges
as device copies between the blocks' buffers.  Every transform and every
point of the x stage computes exactly what the whole-domain step computes,
so the split step must match it (through the C ABI):
  * relative L2 <= 1e-12 per field (and for Z), FP64 and mixed form 1, with
    2 and 3 blocks (uneven blocks of pointers_calc), the reference CFL mode
    (the same Deltat), and with mu = T^0.7 and the passive scalar.
"""
import numpy as np
import pytest

from loma_phd_b200 import Lomacte
from tests.helpers import FIELDS, case, mixing_scalar, rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _run(p, y, st, n, nblocks=0, Z=None):
    g = Lomacte(p, y)
    g.load_state(st)
    if Z is not None:
        g.load_scalar(Z)
    if nblocks:
        g.step_split(nblocks, n)
    else:
        g.step(n)
    out = g.get_state(), (g.get_scalar() if Z is not None else None), g.diag()
    g.close()
    return out


def _check(a, b, za=None, zb=None):
    e = {k: rel_l2(a[k], b[k]) for k in FIELDS}
    e["u00"] = rel_l2(a["u00"], b["u00"])
    for k in ("v00", "w00"):
        e[k] = np.linalg.norm(a[k] - b[k]) / np.linalg.norm(b["u00"])
    if zb is not None:
        e["Z"] = rel_l2(za, zb)
    assert max(e.values()) <= TOL, e


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("nblocks", [2, 3])
def test_split_matches_whole_domain(gpu, prec, nblocks):
    p, y, st = case(96, 96, 33, precision=prec)
    a, _, da = _run(p, y, st, 3, nblocks)
    b, _, db = _run(p, y, st, 3)
    _check(a, b)
    assert abs(da["dm"] - db["dm"]) <= TOL * abs(db["dm"])


def test_split_cfl_mode_same_deltat(gpu):
    p, y, st = case(128, 128, 65, dt_mode=0, dt=1e-4)
    p.ncfl = 1
    a, _, da = _run(p, y, st, 3, 2)
    b, _, db = _run(p, y, st, 3)
    _check(a, b)
    assert da["Deltat"] == db["Deltat"] and da["Deltat_next"] == db["Deltat_next"]


@pytest.mark.parametrize("prec", [0, 1])
def test_split_with_viscosity_and_scalar(gpu, prec):
    p, y, st = case(96, 96, 33, precision=prec, visc=1, sigma=0.7, scalar=1)
    Z = mixing_scalar(p, y)
    a, za, _ = _run(p, y, st, 2, 3, Z)
    b, zb, _ = _run(p, y, st, 2, 0, Z)
    _check(a, b, za, zb)
