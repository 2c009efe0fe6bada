"""Mixed-precision forms against the FP64 references, through the C ABI.

precision=1: FP32 transform buffers and FP32 FFT arithmetic; FP64 state,
RK3 accumulators, y solves, 00 modes and pointwise EOS math.
precision=2: the same with FP64 FFT arithmetic (FP32 storage only).

Bars:
  * 1 RK3 step against the FP64 oracle: relative L2 <= 1e-6 per field, and
    measurably different from the FP64 path (the FP32 storage is used)
  * 1000 RK3 steps (s = 4, dt = 0.01) against the FP64 GPU path: relative
    L2 <= 1e-5 per field and the momentum-thickness history to 1e-6, at
    64^2 x 129 for precision=1 and 128^2 x 129 for precision=2.  The FP64
    GPU path stands in for the FP64 oracle here: it matches the oracle to
    1e-8 after 100 steps (test_gpu_parity.py), and 1000 oracle steps at
    these sizes take many minutes.
"""
import numpy as np
import pytest

from loma_phd_b200 import Lomacte
from tests.helpers import FIELDS, case, oracle_for, rel_l2

pytestmark = pytest.mark.gpu

STEP1_TOL = 1e-6
STEP1000_TOL = 1e-5
DM_TOL = 1e-6


def err00(a, b, k):
    """Error of a 00 profile; v00 and w00 are measured against the size of
    u00 (w00 is zero up to round-off in these cases)."""
    den = max(np.linalg.norm(b[k]), np.linalg.norm(b["u00"]))
    return np.linalg.norm(np.asarray(a[k]) - np.asarray(b[k])) / den


def _run(p, y, st, nsteps, hist_every=0):
    g = Lomacte(p, y)
    g.load_state(st)
    hist = []
    for n in range(nsteps):
        g.step(1)
        if hist_every and (n + 1) % hist_every == 0:
            hist.append(g.diag())
    s = g.get_state()
    d = g.diag()
    g.close()
    return s, d, hist


@pytest.mark.parametrize("prec,grid", [(1, (24, 24, 33)), (1, (32, 32, 65)), (2, (32, 32, 65))])
def test_mixed_one_step_vs_oracle(gpu, prec, grid):
    p, y, st = case(*grid, precision=prec)
    sm, dm, _ = _run(p, y, st, 1)
    p64, _, _ = case(*grid)
    s64, _, _ = _run(p64, y, st, 1)
    o = oracle_for(p64, y, st)
    o.step(1)
    so = o.get_state()
    for k in FIELDS:
        e = rel_l2(sm[k], so[k])
        assert e < STEP1_TOL, (k, e)
    for k in ("u00", "v00", "w00"):
        assert err00(sm, so, k) < STEP1_TOL, k
    # the mixed form really computes its transforms in FP32
    assert max(rel_l2(sm[k], s64[k]) for k in FIELDS) > 1e-12


@pytest.mark.parametrize("prec,grid", [(1, (64, 64, 129)), (2, (128, 128, 129))])
def test_mixed_thousand_steps_vs_fp64(gpu, prec, grid):
    p, y, st = case(*grid, precision=prec)
    sm, dm, hm = _run(p, y, st, 1000, hist_every=50)
    p64, _, _ = case(*grid)
    s64, d64, h64 = _run(p64, y, st, 1000, hist_every=50)
    errs = {k: rel_l2(sm[k], s64[k]) for k in FIELDS}
    errs.update({k: err00(sm, s64, k) for k in ("u00", "v00", "w00")})
    for k, e in errs.items():
        assert e < STEP1000_TOL, (k, e, errs)
    a = np.array([h["dm"] for h in hm])
    b = np.array([h["dm"] for h in h64])
    assert np.abs(a - b).max() <= DM_TOL * np.abs(b).max(), (a, b)
    assert np.isfinite(dm["dm"]) and dm["time"] == pytest.approx(d64["time"])


def test_fft64_stage_mask(gpu, monkeypatch):
    """LMC_FFT64 gives chosen transform stages of the mixed form FP64
    butterflies: with the x stage and the direct z transforms in FP64 the
    result is closer to the FP64 path than the plain mixed form."""
    p, y, st = case(64, 64, 129, precision=1)
    p64, _, _ = case(64, 64, 129)
    s64, _, _ = _run(p64, y, st, 20)
    errs = {}
    for mask in ("0", "6"):
        monkeypatch.setenv("LMC_FFT64", mask)
        sm, _, _ = _run(p, y, st, 20)
        errs[mask] = rel_l2(sm["phi"], s64["phi"])
    assert errs["6"] < 0.5 * errs["0"], errs
