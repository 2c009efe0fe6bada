"""Physical-field export on the device (lmc_physical_f64) against the
oracle's restatement from the same state, through the C ABI.

Bars (those of the FP64 step parity): every quantity (u, v, w, T,
omega_x, omega_y, omega_z, Z) on the chosen planes <= 1e-10 relative L2
and <= 1e-9 relative max difference, FP64 and mixed cases (the export is
FP64 in every form), with the scalar, in a 2-D run and with the
variable viscosity; the state is bit for bit the same before and after,
and the next step is unchanged by an export in between.
"""
import numpy as np
import pytest

from loma_phd_b200 import Lomacte
from tests.helpers import FIELDS, case, oracle_for, rel_l2

pytestmark = pytest.mark.gpu


def _compare(g, p, y, planes, Z=None):
    s = g.get_state()
    o = oracle_for(p, y, s)
    if Z is not None:
        o.set_scalar(g.get_scalar(), 1.0)
    ref = o.physical(planes)
    dev = g.physical(planes)
    names = list(dev)
    assert ref.shape[1] == len(names)
    for q, k in enumerate(names):
        r = ref[:, q]
        assert rel_l2(dev[k], r) < 1e-10, (k, rel_l2(dev[k], r))
        e = np.abs(dev[k] - r).max() / max(np.abs(r).max(), 1e-300)
        assert e < 1e-9, (k, e)
    return dev


@pytest.mark.parametrize("prec", [0, 1])
def test_export_matches_oracle(gpu, prec):
    p, y, st = case(32, 32, 65, precision=prec)
    g = Lomacte(p, y)
    g.load_state(st)
    g.step(3)
    before = g.get_state()
    dev = _compare(g, p, y, [1, 9, 33, 64])
    after = g.get_state()
    for k in FIELDS + ("u00", "v00", "w00"):
        assert np.array_equal(before[k], after[k]), k
    assert np.abs(dev["omega_z"]).max() > 0.1
    g.close()


def test_export_does_not_change_the_run(gpu):
    p, y, st = case(24, 24, 33)
    runs = []
    for export in (False, True):
        g = Lomacte(p, y)
        g.load_state(st)
        g.step(2)
        if export:
            g.physical(list(range(1, p.my + 1)))
        g.step(2)
        runs.append(g.get_state())
        g.close()
    for k in FIELDS:
        assert np.array_equal(runs[0][k], runs[1][k]), k


def test_export_with_scalar_and_viscosity(gpu):
    p, y, st = case(24, 24, 33, scalar=1, schmidt=1.0, visc=1, sigma=0.7)
    T = st["scal"]
    tb, tt = T[0, 0, 0].real, T[0, 0, -1].real
    Z = T / (tt - tb)
    Z[0, 0, :] -= tb / (tt - tb)
    g = Lomacte(p, y)
    g.load_state(st)
    g.load_scalar(Z)
    g.step(2)
    dev = _compare(g, p, y, [1, 17, 33], Z=True)
    assert "Z" in dev
    g.close()


def test_export_two_dimensional(gpu):
    p, y, st = case(64, 1, 65)
    g = Lomacte(p, y)
    g.load_state(st)
    g.step(2)
    dev = _compare(g, p, y, [5, 33])
    assert dev["u"].shape == (2, 3, p.mgalx)
    g.close()
