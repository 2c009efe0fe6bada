"""Statistics without a GPU: the oracle's restatement of addstats1/addstats2
and the phys2 sums (trunk/lomacte3/src/cross.f:1981-2290, 1583-1607)
checked by identities the reference's definitions imply, and the .sta /
.spe writers (escru.f:276-484) by round trips.

Identities (the reference has no golden statistics to pin against):
  * Parseval: Tp(j) (sum over modes of the weighted |T|^2, addstats1) equals
    num(j) / (mgalx mgalz) with sigma = 1 (the plane sum of T^2 in phys2),
    since both see the same T of the substep;
  * mum(j) = mgalx mgalz for sigma = 0, num(j) = mgalx mgalz Tm(j) for
    sigma = 0 (the plane mean of T is its 00 mode);
  * spectra summed over |kz| at a plane equal the profile of the same
    quantity at that row (up = sum_k sp_u, Tp = sum_k sp_T, ...);
  * uner_q = sum_j hy_j (profile increment of the step);
  * nacum and nacumsp count the accumulating steps; clear_spectra zeroes
    the spectra and nacumsp only.
"""
import numpy as np
import pytest

from loma_phd_b200 import files
from loma_phd_b200.stats import (ENERGY_NAMES, FAC_FROM, NSTAT, SPEC_FIELDS, STAT_NAMES, StatsData, enerdis,
                                 energies, fac32)
from tests.helpers import case, oracle_for

S = {n: i for i, n in enumerate(STAT_NAMES)}


@pytest.fixture(scope="module")
def run():
    p, y, st = case(24, 24, 33)
    o = oracle_for(p, y, st, nthreads=4)
    planes = [5, 17, 29]
    o.stats_reset(planes, sigma=1.0)
    o.step(1)
    o.stats_step(2)
    prof, spec, uner, na, nsp = o.stats_read()
    return p, y, o, planes, prof, spec, uner, na, nsp


def test_counts_and_shapes(run):
    p, y, o, planes, prof, spec, uner, na, nsp = run
    assert (na, nsp) == (2, 2)
    assert prof.shape == (NSTAT, p.my)
    assert spec.shape == (p.nplanes, 12, len(planes), (p.mz - 1) // 2 + 1)
    assert np.all(np.isfinite(prof)) and np.all(np.isfinite(spec))


def test_parseval_T(run):
    p, y, o, planes, prof, spec, uner, na, nsp = run
    N = p.mgalx * p.mgalz
    np.testing.assert_allclose(prof[S["Tp"]], prof[S["num"]] / N, rtol=1e-12, atol=0)
    np.testing.assert_allclose(prof[S["mum"]] / N, prof[S["Tm"]], rtol=1e-12, atol=0)
    # 1/T sums: positive, between 1/max T and 1/min T per point
    assert np.all(prof[S["rhom"]] > 0)


def test_spectra_sum_to_profiles(run):
    p, y, o, planes, prof, spec, uner, na, nsp = run
    for iy, j1 in enumerate(planes):
        j = j1 - 1
        for fld, name in (("u", "up"), ("v", "vp"), ("w", "wp"), ("uv_re", "uvr"), ("o1", "w1p"),
                          ("o2", "w2p"), ("o3", "w3p"), ("T", "Tp")):
            s = spec[:, SPEC_FIELDS.index(fld), iy, :].sum()
            assert s == pytest.approx(prof[S[name], j], rel=1e-12, abs=1e-300), (fld, j1)


def test_energies_of_last_step(run):
    p, y, o, planes, prof, spec, uner, na, nsp = run
    hy = np.zeros(p.my)
    ym = np.asarray(y)
    hy[1:-1] = (ym[2:] - ym[:-2]) / 2
    hy[0] = (ym[1] - ym[0]) / 2
    hy[-1] = (ym[-1] - ym[-2]) / 2
    # one more accumulating step: uner is that step's increment, weighted
    before = o.stats_read()[0]
    o.stats_step(1)
    after, _, un, na, nsp = o.stats_read()
    for q, name in enumerate(ENERGY_NAMES):
        inc = after[S[name]] - before[S[name]]
        assert un[q] == pytest.approx(np.sum(inc * hy), rel=1e-10, abs=1e-14), name
    assert na == 3 and nsp == 3
    assert np.all(energies(un) >= 0)


def test_clear_spectra_and_reset():
    p, y, st = case(24, 24, 33)
    o = oracle_for(p, y, st, nthreads=4)
    o.stats_reset([17])
    o.stats_step(1)
    prof, spec, _, na, nsp = o.stats_read(clear_spectra=True)
    assert spec.any() and (na, nsp) == (1, 1)
    prof2, spec2, _, na2, nsp2 = o.stats_read()
    assert not spec2.any() and (na2, nsp2) == (1, 0)
    np.testing.assert_array_equal(prof, prof2)
    N = p.mgalx * p.mgalz
    np.testing.assert_allclose(prof[S["mum"]], N, rtol=1e-15)
    np.testing.assert_allclose(prof[S["num"]] / N, prof[S["Tm"]], rtol=1e-12)
    o.stats_reset([17])
    prof3, spec3, _, na3, nsp3 = o.stats_read()
    assert not prof3.any() and not spec3.any() and (na3, nsp3) == (0, 0)
    # plain steps accumulate nothing
    o.step(1)
    assert not o.stats_read()[0].any()


def _fake(p, planes, seed=3):
    rng = np.random.default_rng(seed)
    prof = rng.standard_normal((NSTAT, p.my))
    spec = np.abs(rng.standard_normal((p.nplanes, 12, len(planes), (p.mz - 1) // 2 + 1)))
    return StatsData(prof=prof, spec=spec, uner=rng.random(9), nacum=7, nacumsp=5, planes=list(planes))


def test_sta_round_trip(tmp_path):
    p, y, _ = case(24, 24, 33)
    fmap = np.linspace(1.0, 2.0, p.my)
    d = _fake(p, [17])
    path = str(tmp_path / "run_001.sta")
    files.write_sta(path, d, y, fmap, time=1.5, Re=160.0, alp=0.5, bet=0.25, mgalx=p.mgalx, mgalz=p.mgalz)
    r = files.read_sta(path)
    assert (r["my"], r["nacum"]) == (p.my, 7)
    assert r["time"] == pytest.approx(1.5) and r["Re"] == pytest.approx(160.0)
    np.testing.assert_array_equal(r["y"], y)
    np.testing.assert_array_equal(r["fmap"], fmap)
    fac = fac32(p.mgalx, p.mgalz)
    np.testing.assert_array_equal(r["prof"][:FAC_FROM], d.prof[:FAC_FROM])
    np.testing.assert_array_equal(r["prof"][FAC_FROM:], d.prof[FAC_FROM:] * fac)
    # record layout: 4-byte markers, 28-byte header, 33 real*8 per row
    raw = open(path, "rb").read()
    assert len(raw) == (8 + 28) + (8 + 16 * p.my) + (8 + 33 * 8 * p.my)
    assert fac == float(np.float32(1.0 / (p.mgalx * p.mgalz)))


def test_spe_round_trip(tmp_path):
    p, y, _ = case(24, 24, 33)
    fmap = np.linspace(1.0, 2.0, p.my)
    planes = [5, 17, 29]
    d = _fake(p, planes)
    path = str(tmp_path / "run_001.spe")
    files.write_spe(path, d, y, fmap, time=2.0, Re=160.0, alp=0.5, bet=0.25, mx=2 * p.nplanes, mz=p.mz)
    r = files.read_spe(path)
    assert (r["mx"], r["my"], r["mz"], r["nacumsp"]) == (2 * p.nplanes, p.my, p.mz, 5)
    np.testing.assert_array_equal(r["planes"], planes)
    np.testing.assert_array_equal(r["spec"], d.spec.astype(np.float32))
    nk = (p.mz - 1) // 2 + 1
    raw = open(path, "rb").read()
    assert len(raw) == (8 + 36) + (8 + 4 * 3 + 16 * p.my) + p.nplanes * (8 + 4 * 12 * 3 * nk)


def test_enerdis():
    d = StatsData(prof=np.zeros((NSTAT, 4)), spec=np.zeros((1, 12, 1, 1)), uner=np.zeros(9), nacum=2, nacumsp=2,
                  planes=[1])
    d.prof[S["ep"]] = [1.0, 2.0, 3.0, 4.0]
    assert enerdis(d, [1.0, 1.0, 0.5, 0.5]) == pytest.approx((1 + 2 + 1.5 + 2) / 2)
