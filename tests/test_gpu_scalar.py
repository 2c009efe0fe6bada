"""Passive scalar Z on the device (lmc_params.scalar = 1) against the
oracle's restatement (Z advanced exactly as the lomacte3 substep advances
T; no lomacte code carries a scalar), through the C ABI.

Bars: FP64, 1 RK3 step <= 1e-10 relative L2 per field and for Z, 20 steps
<= 1e-9; the manufactured invariant (Re*Sc = Pe and Z = (T - T_bot) /
(T_top - T_bot) at the start) holds on the device to 1e-12 after 20 steps;
mixed form, 1 step against the FP64 oracle <= 1e-6 for Z.
"""
import numpy as np
import pytest

from loma_phd_b200 import Lomacte, LomacteError, ICParams, make_ic
from tests.helpers import FIELDS, case, oracle_for, rel_l2

pytestmark = pytest.mark.gpu

PR = float(np.float32(0.7))  # Pe = Re*0.7f (main.f:569)


def _affine(st):
    T = st["scal"]
    tb, tt = T[0, 0, 0].real, T[0, 0, -1].real
    a, b = -tb / (tt - tb), 1.0 / (tt - tb)
    Z = b * T.copy()
    Z[0, 0, :] += a
    return Z, a, b


def _scalar_ic(p, y, st):
    """affine in T plus fluctuations of their own (a solenoidal field of
    another seed, zero at the walls as the boundary condition wants)"""
    Z, _, _ = _affine(st)
    other = make_ic(p, y, ICParams(seed=11))["psi"]
    f = 0.05 * other / max(np.abs(other).max(), 1e-300)
    f[:, :, 0] = 0.0
    f[:, :, -1] = 0.0
    f[0, 0, :] = 0.0
    return Z + f


def _pair(p, y, st, Z, n, sc):
    g = Lomacte(p, y)
    g.load_state(st)
    g.load_scalar(Z)
    o = oracle_for(p, y, st)
    o.set_scalar(Z, sc)
    g.step(n)
    o.step(n)
    out = (g.get_state(), g.get_scalar(), o.get_state(), o.get_scalar())
    g.close()
    return out


@pytest.mark.parametrize("sc", [PR, 1.0])
def test_scalar_one_step_fp64(gpu, sc):
    p, y, st = case(24, 24, 33, scalar=1, schmidt=sc)
    Z = _scalar_ic(p, y, st)
    sg, zg, so, zo = _pair(p, y, st, Z, 1, sc)
    for k in FIELDS:
        assert rel_l2(sg[k], so[k]) < 1e-10, (k, rel_l2(sg[k], so[k]))
    assert rel_l2(zg, zo) < 1e-10, rel_l2(zg, zo)


def test_scalar_twenty_steps_fp64(gpu):
    p, y, st = case(32, 32, 65, scalar=1, schmidt=1.0)
    Z = _scalar_ic(p, y, st)
    sg, zg, so, zo = _pair(p, y, st, Z, 20, 1.0)
    for k in FIELDS:
        assert rel_l2(sg[k], so[k]) < 1e-9, k
    assert rel_l2(zg, zo) < 1e-9, rel_l2(zg, zo)
    assert rel_l2(zg, Z) > 1e-6  # Z moved


def test_scalar_follows_temperature_on_device(gpu):
    p, y, st = case(32, 32, 65, scalar=1, schmidt=PR)
    Z, a, b = _affine(st)
    g = Lomacte(p, y)
    g.load_state(st)
    g.load_scalar(Z)
    g.step(20)
    s, z = g.get_state(), g.get_scalar()
    g.close()
    pred = b * s["scal"]
    pred[0, 0, :] += a
    assert np.abs(s["scal"] - st["scal"]).max() > 1e-5
    assert np.abs(z - pred).max() < 1e-12 * np.abs(pred).max()


def test_scalar_mixed_one_step(gpu):
    p, y, st = case(32, 32, 65, scalar=1, schmidt=1.0, precision=1)
    Z = _scalar_ic(p, y, st)
    g = Lomacte(p, y)
    g.load_state(st)
    g.load_scalar(Z)
    g.step(1)
    zg = g.get_scalar()
    g.close()
    p64, _, _ = case(32, 32, 65)
    o = oracle_for(p64, y, st)
    o.set_scalar(Z, 1.0)
    o.step(1)
    assert rel_l2(zg, o.get_scalar()) < 1e-6


def test_scalar_rejects(gpu):
    p, y, st = case(24, 24, 33)
    g = Lomacte(p, y)
    with pytest.raises(LomacteError):
        g.load_scalar(st["scal"])  # created without the scalar
    g.close()
    pv, yv, _ = case(24, 24, 33, variant=1, scalar=1)
    with pytest.raises(LomacteError):
        Lomacte(pv, yv)
