"""GPU parity of the sm_100a substep against the FP64 CPU oracle, through
the C ABI (liblomacte_b200.so).

Bars (FP64 plain path vs FP64 oracle on the same seeded initial condition):
  * single y-operators: relative error <= 1e-12 per mode set
  * 1 RK3 step: relative L2 <= 1e-10 per field
  * 100 RK3 steps: relative L2 <= 1e-8 per field, and the momentum-thickness
    and mass histories equal to 1e-8
"""
import numpy as np
import pytest

from loma_phd_b200 import Lomacte
from tests.helpers import FIELDS, case, oracle_for, rel_l2

pytestmark = pytest.mark.gpu

STEP1_TOL = 1e-10
STEP100_TOL = 1e-8
OP_TOL = 1e-12


def _torch():
    import torch
    return torch


def _kvals(p):
    nkx, mz = p.nplanes, p.mz
    kx = p.alp * np.arange(nkx)
    kzi = np.array([k if k <= (mz - 1) // 2 else k - mz for k in range(mz)])
    kz = p.bet * kzi
    return kx, kz


@pytest.mark.parametrize("ny", [33, 65, 129])
def test_y_operators_match_oracle(gpu, ny):
    torch = _torch()
    p, y, st = case(nx=16, nz=16, ny=ny)
    g = Lomacte(p, y)
    o = oracle_for(p, y, st, nthreads=4)
    rng = np.random.default_rng(7)
    shp = p.shape
    f = (rng.standard_normal(shp) + 1j * rng.standard_normal(shp)) * np.exp(-(y / 6.0) ** 2)
    fin = torch.from_numpy(f.view(np.float64).copy()).cuda()
    out = torch.zeros_like(fin)
    out2 = torch.zeros_like(fin)
    kx, kz = _kvals(p)
    nkx, mz = p.nplanes, p.mz
    for op in (1, 2, 3, 4):
        out.zero_(); out2.zero_()
        g.op_y(op, fin, out, out2 if op == 3 else None)
        torch.cuda.synchronize()
        a = out.cpu().numpy().view(np.complex128).reshape(shp)
        a2 = out2.cpu().numpy().view(np.complex128).reshape(shp)
        ref = np.zeros(shp, dtype=np.complex128)
        ref2 = np.zeros(shp, dtype=np.complex128)
        for i in range(nkx):
            for k in range(mz):
                u = f[i, k]
                k2 = kx[i] ** 2 + kz[k] ** 2
                if op == 1:
                    ref[i, k] = o.deryr(u.real) + 1j * o.deryr(u.imag)
                elif op == 2:
                    ref[i, k] = o.deryyr(u.real) + 1j * o.deryyr(u.imag)
                elif op == 3:
                    ref[i, k], ref2[i, k] = o.lapvdvhom(u, k2)
                else:
                    ref[i, k], _ = o.solvepsi(u, k2)
        e = rel_l2(a, ref)
        assert e < OP_TOL, (op, e)
        if op == 3:
            assert rel_l2(a2, ref2) < OP_TOL
    g.close()


def _run_pair(p, y, st, nsteps, hist=False):
    g = Lomacte(p, y)
    g.load_state(st)
    o = oracle_for(p, y, st)
    hg, ho = [], []
    for _ in range(nsteps):
        g.step(1)
        o.step(1)
        if hist:
            hg.append(g.diag())
            ho.append(o.diag())
    sg = g.get_state()
    so = o.get_state()
    dg, do = g.diag(), o.diag()
    g.close()
    return sg, so, dg, do, hg, ho


@pytest.mark.parametrize("grid", [(24, 24, 33), (32, 32, 65)])
def test_one_step_matches_oracle(gpu, grid):
    p, y, st = case(*grid)
    sg, so, dg, do, _, _ = _run_pair(p, y, st, 1)
    for k in FIELDS:
        e = rel_l2(sg[k], so[k])
        assert e < STEP1_TOL, (k, e)
    for k in ("u00", "v00", "w00"):
        assert rel_l2(sg[k], so[k]) < STEP1_TOL, k
    for k in ("dm", "dw", "masst", "massu", "trapz"):
        assert abs(dg[k] - do[k]) <= STEP1_TOL * max(1.0, abs(do[k])), (k, dg[k], do[k])


@pytest.mark.parametrize("ncfl", [1, 2])
@pytest.mark.parametrize("family", ["warp", "mode"])
def test_cfl_mode_matches_oracle(gpu, monkeypatch, ncfl, family):
    monkeypatch.setenv("LMC_YPATH", family)
    p, y, st = case(24, 24, 33, dt_mode=0, dt=1e-4, ncfl=ncfl)
    sg, so, dg, do, hg, ho = _run_pair(p, y, st, 5, hist=True)
    for a, b in zip(hg, ho):
        assert a["Deltat"] == b["Deltat"]
    for k in FIELDS:
        assert rel_l2(sg[k], so[k]) < STEP1_TOL * 10, k


def test_hundred_steps_match_oracle(gpu):
    # the small mixing-layer case: 64^2 Fourier modes x 129, s = 4, dt = 0.01
    p, y, st = case(64, 64, 129)
    sg, so, dg, do, hg, ho = _run_pair(p, y, st, 100, hist=True)
    for k in FIELDS:
        e = rel_l2(sg[k], so[k])
        assert e < STEP100_TOL, (k, e)
    for key in ("dm", "massu", "massv", "masst"):
        a = np.array([h[key] for h in hg])
        b = np.array([h[key] for h in ho])
        assert np.abs(a - b).max() <= STEP100_TOL * max(1.0, np.abs(b).max()), key
