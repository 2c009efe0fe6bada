"""The mode-parallel y kernels (one thread per (kx,kz) mode, lmc_ytpm.cuh)
against the FP64 oracle and against the warp-per-mode kernels, through the
C ABI.  LMC_YPATH=mode forces the family on grids the automatic choice
would give to the warp kernels.

Bars: single y operators <= 1e-12; 1 RK3 step <= 1e-10 per field (FP64)
and <= 1e-6 (mixed form) against the oracle; 100 steps equal to the warp
family to 1e-10 per field with identical Deltat and momentum thickness to
1e-10.
"""
import numpy as np
import pytest

from loma_phd_b200 import Lomacte
from tests.helpers import FIELDS, case, oracle_for, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture
def mode_family(monkeypatch):
    monkeypatch.setenv("LMC_YPATH", "mode")


def _kvals(p):
    kx = p.alp * np.arange(p.nplanes)
    kz = p.bet * np.array([k if k <= (p.mz - 1) // 2 else k - p.mz for k in range(p.mz)])
    return kx, kz


@pytest.mark.parametrize("ny", [33, 65, 129])
def test_mode_family_operators(gpu, mode_family, ny):
    import torch
    p, y, st = case(nx=16, nz=16, ny=ny)
    g = Lomacte(p, y)
    assert g.y_family == "mode"
    o = oracle_for(p, y, st, nthreads=4)
    rng = np.random.default_rng(11)
    shp = p.shape
    f = (rng.standard_normal(shp) + 1j * rng.standard_normal(shp)) * np.exp(-(y / 6.0) ** 2)
    fin = torch.from_numpy(f.view(np.float64).copy()).cuda()
    out, out2 = torch.zeros_like(fin), torch.zeros_like(fin)
    kx, kz = _kvals(p)
    for op in (1, 2, 3, 4):
        out.zero_()
        out2.zero_()
        g.op_y(op, fin, out, out2 if op == 3 else None)
        torch.cuda.synchronize()
        a = out.cpu().numpy().view(np.complex128).reshape(shp)
        a2 = out2.cpu().numpy().view(np.complex128).reshape(shp)
        ref = np.zeros(shp, dtype=np.complex128)
        ref2 = np.zeros(shp, dtype=np.complex128)
        for i in range(p.nplanes):
            for k in range(p.mz):
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
        assert rel_l2(a, ref) < 1e-12, op
        if op == 3:
            assert rel_l2(a2, ref2) < 1e-12
    g.close()


@pytest.mark.parametrize("prec,grid,tol", [(0, (24, 24, 33), 1e-10), (0, (32, 32, 65), 1e-10),
                                           (1, (32, 32, 65), 1e-6), (2, (32, 32, 65), 1e-6)])
def test_mode_family_one_step(gpu, mode_family, prec, grid, tol):
    p, y, st = case(*grid, precision=prec)
    g = Lomacte(p, y)
    assert g.y_family == "mode"
    g.load_state(st)
    g.step(1)
    sg = g.get_state()
    g.close()
    p64, _, _ = case(*grid)
    o = oracle_for(p64, y, st)
    o.step(1)
    so = o.get_state()
    for k in FIELDS:
        assert rel_l2(sg[k], so[k]) < tol, (k, rel_l2(sg[k], so[k]))
    for k in ("u00", "v00"):
        assert rel_l2(sg[k], so[k]) < tol, k


def test_mode_family_matches_warp_family(gpu, monkeypatch):
    p, y, st = case(64, 64, 129)
    runs = {}
    for fam in ("warp", "mode"):
        monkeypatch.setenv("LMC_YPATH", fam)
        g = Lomacte(p, y)
        assert g.y_family == fam
        g.load_state(st)
        hist = []
        for _ in range(100):
            g.step(1)
            hist.append(g.diag())
        runs[fam] = (g.get_state(), hist)
        g.close()
    (sw, hw), (sm, hm) = runs["warp"], runs["mode"]
    for k in FIELDS:
        assert rel_l2(sm[k], sw[k]) < 1e-10, k
    assert [h["Deltat"] for h in hw] == [h["Deltat"] for h in hm]
    assert max(abs(a["dm"] - b["dm"]) for a, b in zip(hw, hm)) < 1e-10


def test_automatic_family_choice(gpu, monkeypatch):
    monkeypatch.delenv("LMC_YPATH", raising=False)
    small = Lomacte(*case(32, 32, 33)[:2])
    big = Lomacte(*case(192, 192, 33)[:2])  # 96 x 191 = 18336 modes
    assert small.y_family == "warp" and big.y_family == "mode"
    assert big.launches_per_step == 36 and small.launches_per_step == 33
    small.close()
    big.close()
