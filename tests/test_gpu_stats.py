"""Statistics and spectra on the device (addstats1/addstats2 and the phys2
sums, trunk/lomacte3/src/cross.f:1981-2290, 1583-1607) against the FP64
oracle's restatement, through the C ABI.

Bars: FP64, both y families: every profile, spectrum and energy within
1e-10 of the oracle relative to the largest magnitude of its own profile
(floor 1e-8); mixed forms (precision 1 and 2): 1e-5, where the means of
w, rho w and the streamwise vorticity (zero up to noise in these cases,
|w00| ~ 1e-6) are measured against 1e-4 of the largest mean of their
triple (um, rum, w3m).  Accumulating steps leave
the trajectory unchanged (state identical bit for bit to plain steps), two
runs give identical statistics, clear_spectra zeroes only the spectra.
"""
import numpy as np
import pytest

from loma_phd_b200 import Lomacte, LomacteError
from loma_phd_b200.stats import NSTAT
from tests.helpers import FIELDS, case, oracle_for

pytestmark = pytest.mark.gpu

PLANES = [5, 17, 29]


def _err(a, b, floor=None):
    """max |a-b| over each profile (or spectrum field) relative to the
    profile's largest magnitude, at least floor (default 1e-8)"""
    a = np.asarray(a).reshape(a.shape[0], -1) if a.ndim > 1 else np.asarray(a)[:, None]
    b = np.asarray(b).reshape(a.shape)
    den = np.abs(b).max(axis=1)
    den = np.maximum(den, 1e-8 if floor is None else floor)
    return (np.abs(a - b).max(axis=1) / den).max()


def _mean_floor(prof):
    """1e-4 of the largest mean of each triple of 00 means (velocities,
    momenta, vorticities) for the three members of the triple"""
    fl = np.full(prof.shape[0], 1e-8)
    for first in (0, 3, 7):  # (um vm wm), (rum rvm rwm), (w1m w2m w3m)
        fl[first:first + 3] = max(1e-8, 1e-4 * np.abs(prof[first:first + 3]).max())
    return fl


def _device(p, y, st, planes, sigma, nplain, nstat):
    g = Lomacte(p, y)
    g.load_state(st)
    g.stats_reset(planes, sigma)
    g.step(nplain)
    g.stats_step(nstat)
    d = g.stats_read()
    s = g.get_state()
    fam = g.y_family
    g.close()
    return d, s, fam


def _oracle(p, y, st, planes, sigma, nplain, nstat):
    o = oracle_for(p, y, st)
    o.stats_reset(planes, sigma)
    o.step(nplain)
    o.stats_step(nstat)
    return o.stats_read()


def _check(d, ref, tol, mixed=False):
    prof, spec, uner, na, nsp = ref
    assert (d.nacum, d.nacumsp) == (na, nsp)
    fl = _mean_floor(prof) if mixed else None
    assert _err(d.prof, prof, fl) < tol, _err(d.prof, prof, fl)
    # spectra per (field): [nkx,12,nsp,nk] -> rows of field
    sd = np.moveaxis(d.spec, 1, 0).reshape(12, -1)
    so = np.moveaxis(spec, 1, 0).reshape(12, -1)
    assert _err(sd, so) < tol, _err(sd, so)
    assert np.abs(d.uner - uner).max() <= tol * max(np.abs(uner).max(), 1e-8)


@pytest.mark.parametrize("family", ["warp", "mode"])
@pytest.mark.parametrize("sigma", [0.0, 0.7])
def test_stats_fp64_vs_oracle(gpu, monkeypatch, family, sigma):
    monkeypatch.setenv("LMC_YPATH", family)
    p, y, st = case(24, 24, 33)
    d, _, fam = _device(p, y, st, PLANES, sigma, 1, 2)
    assert fam == family
    _check(d, _oracle(p, y, st, PLANES, sigma, 1, 2), 1e-10)


def test_stats_fp64_larger_grid(gpu):
    p, y, st = case(48, 48, 65)
    planes = [9, 33, 57, 33]
    d, _, _ = _device(p, y, st, planes, 0.0, 0, 3)
    _check(d, _oracle(p, y, st, planes, 0.0, 0, 3), 1e-10)


@pytest.mark.parametrize("prec", [1, 2])
def test_stats_mixed_vs_oracle(gpu, prec):
    p, y, st = case(32, 32, 65, precision=prec)
    d, _, _ = _device(p, y, st, PLANES, 0.0, 2, 2)
    p64, _, _ = case(32, 32, 65)
    _check(d, _oracle(p64, y, st, PLANES, 0.0, 2, 2), 1e-5, mixed=True)


def test_stats_steps_leave_the_trajectory(gpu):
    p, y, st = case(32, 32, 65)
    g = Lomacte(p, y)
    g.load_state(st)
    g.step(4)
    ref = g.get_state()
    g.load_state(st)
    g.stats_reset(PLANES)
    g.step(1)
    g.stats_step(2)
    g.step(1)
    s = g.get_state()
    g.close()
    for k in FIELDS + ("u00", "v00", "w00"):
        np.testing.assert_array_equal(s[k], ref[k], err_msg=k)


def test_stats_reproducible_and_clear(gpu):
    p, y, st = case(32, 32, 65)
    a, _, _ = _device(p, y, st, PLANES, 0.0, 1, 2)
    b, _, _ = _device(p, y, st, PLANES, 0.0, 1, 2)
    np.testing.assert_array_equal(a.prof, b.prof)
    np.testing.assert_array_equal(a.spec, b.spec)
    g = Lomacte(p, y)
    g.load_state(st)
    g.stats_reset(PLANES)
    g.stats_step(1)
    d1 = g.stats_read(clear_spectra=True)
    d2 = g.stats_read()
    assert d1.spec.any() and not d2.spec.any()
    assert (d2.nacum, d2.nacumsp) == (1, 0)
    np.testing.assert_array_equal(d1.prof, d2.prof)
    g.stats_step(1)
    d3 = g.stats_read()
    assert (d3.nacum, d3.nacumsp) == (2, 1) and d3.spec.any()
    g.stats_reset([1, 2])  # fewer planes: the buffers are reused
    d4 = g.stats_read()
    assert not d4.prof.any() and d4.spec.shape[2] == 2 and (d4.nacum, d4.nacumsp) == (0, 0)
    g.close()


def test_stats_rejects(gpu):
    p, y, st = case(24, 24, 33)
    g = Lomacte(p, y)
    with pytest.raises(LomacteError):
        g.stats_step(1)  # no reset yet
    with pytest.raises(LomacteError):
        g.stats_reset([0])  # rows are 1-based
    with pytest.raises(LomacteError):
        g.stats_reset([p.my + 1])
    g.close()
    pv, yv, _ = case(24, 24, 33, variant=1)
    gv = Lomacte(pv, yv)
    with pytest.raises(LomacteError):
        gv.stats_reset([17])
    gv.close()
    assert NSTAT == 33
