"""Variable viscosity mu = k = rho D = T^sigma on the device
(lmc_params.visc = 1) against the oracle's restatement, through the C ABI.

Bars: sigma = 0 with the extension on equals the constant-viscosity path
to 1e-12 after 3 steps; FP64 with sigma = 0.7, 1 RK3 step <= 1e-10
relative L2 per field, 20 steps <= 1e-9 (with the passive scalar, Z
included), the reference's CFL mode (Deltat from the maxima, diffusive
limit with T_max^(1+sigma)) <= 1e-10 after 3 steps, a 2-D run <= 1e-10;
mixed forms, 1 step against the FP64 oracle <= 1e-6 (form 2) and <= 3e-6
(form 1) per field.
"""
import numpy as np
import pytest

from loma_phd_b200 import ICParams, Lomacte, make_ic
from tests.helpers import FIELDS, case, oracle_for, rel_l2

pytestmark = pytest.mark.gpu

PR = float(np.float32(0.7))  # Pe = Re*0.7f (main.f:569)
SIG = 0.7


def _dev(p, y, st, n, Z=None):
    g = Lomacte(p, y)
    g.load_state(st)
    if Z is not None:
        g.load_scalar(Z)
    g.step(n)
    out = g.get_state(), (g.get_scalar() if Z is not None else None), g.diag()
    g.close()
    return out


def _orc(p, y, st, n, sigma, Z=None, sc=None):
    o = oracle_for(p, y, st)
    if Z is not None:
        o.set_scalar(Z, sc)
    o.set_viscosity(sigma)
    o.step(n)
    return o.get_state(), (o.get_scalar() if Z is not None else None), o.diag()


def _check(sg, so, bar):
    for k in FIELDS:
        assert rel_l2(sg[k], so[k]) < bar, (k, rel_l2(sg[k], so[k]))
    for k in ("u00", "w00"):
        assert rel_l2(sg[k], so[k]) < bar, (k, rel_l2(sg[k], so[k]))


def test_visc_sigma_zero_is_constant_viscosity(gpu):
    p, y, st = case(24, 24, 33, visc=1, sigma=0.0)
    a, _, _ = _dev(p, y, st, 3)
    p0, _, _ = case(24, 24, 33)
    b, _, _ = _dev(p0, y, st, 3)
    for k in FIELDS:
        assert rel_l2(a[k], b[k]) < 1e-12, (k, rel_l2(a[k], b[k]))


def test_visc_one_step_fp64(gpu):
    p, y, st = case(24, 24, 33, visc=1, sigma=SIG)
    sg, _, _ = _dev(p, y, st, 1)
    so, _, _ = _orc(p, y, st, 1, SIG)
    _check(sg, so, 1e-10)


def test_visc_twenty_steps_fp64_with_scalar(gpu):
    p, y, st = case(32, 32, 65, visc=1, sigma=SIG, scalar=1, schmidt=1.0)
    other = make_ic(p, y, ICParams(seed=11))["psi"]
    Z = st["scal"] / np.abs(st["scal"]).max() + 0.05 * other / np.abs(other).max()
    Z[:, :, 0] = 0.0
    Z[:, :, -1] = 0.0
    Z[0, 0, 0], Z[0, 0, -1] = 0.0, 1.0
    sg, zg, _ = _dev(p, y, st, 20, Z)
    so, zo, _ = _orc(p, y, st, 20, SIG, Z, 1.0)
    _check(sg, so, 1e-9)
    assert rel_l2(zg, zo) < 1e-9, rel_l2(zg, zo)
    # the viscosity changed the run
    o = oracle_for(p, y, st)
    o.set_scalar(Z, 1.0)
    o.step(20)
    assert rel_l2(so["vor"], o.get_state()["vor"]) > 1e-4


def test_visc_cfl_mode(gpu):
    p, y, st = case(24, 24, 33, visc=1, sigma=SIG, dt_mode=0, dt=1e-4)
    p.ncfl = 1
    sg, _, dg = _dev(p, y, st, 3)
    so, _, do = _orc(p, y, st, 3, SIG)
    _check(sg, so, 1e-10)
    assert abs(dg["Deltat"] - do["Deltat"]) <= 1e-12 * do["Deltat"], (dg["Deltat"], do["Deltat"])


def test_visc_two_dimensional(gpu):
    p, y, st = case(64, 1, 65, visc=1, sigma=SIG)
    sg, _, _ = _dev(p, y, st, 2)
    so, _, _ = _orc(p, y, st, 2, SIG)
    _check(sg, so, 1e-10)


@pytest.mark.parametrize("prec,bar", [(1, 3e-6), (2, 1e-6)])
def test_visc_mixed_one_step(gpu, prec, bar):
    p, y, st = case(32, 32, 65, visc=1, sigma=SIG, precision=prec)
    sg, _, _ = _dev(p, y, st, 1)
    so, _, _ = _orc(p, y, st, 1, SIG)
    for k in FIELDS:
        assert rel_l2(sg[k], so[k]) < bar, (k, rel_l2(sg[k], so[k]))


def test_visc_launches_and_footprint(gpu):
    from loma_phd_b200.lomacte import footprint
    p, y, st = case(24, 24, 33, visc=1, sigma=SIG)
    g = Lomacte(p, y)
    assert g.launches_per_step == 3 * (11 + 1 + 2)
    g.close()
    p0, _, _ = case(24, 24, 33)
    assert footprint(p) > footprint(p0)
