"""Passive scalar Z on the CPU: the oracle's extension (no lomacte code
carries a scalar; it is advanced exactly as the substep advances T).

Manufactured invariant: with Re*Sc equal to the Peclet number of T and Z
started as an affine function of T (Z = (T - T_bot)/(T_top - T_bot)), the
equations of T and Z coincide up to that map, so Z stays that function of
T at every step, to round-off, while T itself changes.  With another
Schmidt number the two separate.
"""
import numpy as np

from tests.helpers import case, oracle_for


def _affine(st):
    T = st["scal"]
    tb, tt = T[0, 0, 0].real, T[0, 0, -1].real
    a, b = -tb / (tt - tb), 1.0 / (tt - tb)
    Z = b * T.copy()
    Z[0, 0, :] += a
    return Z, a, b


def _run(sc_factor, n=5):
    p, y, st = case(24, 24, 33)
    o = oracle_for(p, y, st, nthreads=4)
    Z, a, b = _affine(st)
    pe = p.Re * float(np.float32(0.7))  # Pe = Re*0.7f (main.f:569)
    o.set_scalar(Z, sc_factor * pe / p.Re)
    o.step(n)
    s = o.get_state()
    pred = b * s["scal"]
    pred[0, 0, :] += a
    return o.get_scalar(), pred, s, st


def test_scalar_follows_temperature():
    z, pred, s, st = _run(1.0)
    assert np.abs(s["scal"] - st["scal"]).max() > 1e-5  # T moved
    assert np.abs(z - pred).max() < 1e-13 * np.abs(pred).max()


def test_scalar_uses_its_schmidt_number():
    z, pred, _, _ = _run(0.5)
    assert np.abs(z - pred).max() > 1e-8
