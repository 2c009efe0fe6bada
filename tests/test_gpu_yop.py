"""The compact y operators as dense GEMMs on the tensor cores
(lmc_op_y_dense) against the FP64 oracle, and the autotuner that times them
against the banded solves (lmc_yop_tune), through the C ABI.

Bars: FP64 GEMM d/dy <= 1e-12 and d2/dy2 <= 1e-11 relative (the dense
d2/dy2 rows cancel terms of about 3e3 times the result, so FP64 round-off
is amplified); 3xTF32 d/dy <= 1e-5, d2/dy2 <= 1e-3 (the same cancellation
on FP32-level operands)."""
import numpy as np
import pytest

from loma_phd_b200 import Lomacte
from tests.helpers import case, oracle_for, rel_l2

pytestmark = pytest.mark.gpu
BARS = {(1, 1): 1e-12, (2, 1): 1e-11, (1, 2): 1e-5, (2, 2): 1e-3}


@pytest.mark.parametrize("ny", [65, 129])
def test_dense_operators_match_oracle(gpu, ny):
    import torch
    p, y, st = case(nx=16, nz=16, ny=ny)
    g = Lomacte(p, y)
    o = oracle_for(p, y, st, nthreads=2)
    rng = np.random.default_rng(ny)
    shp = p.shape
    f = (rng.standard_normal(shp) + 1j * rng.standard_normal(shp)) * np.exp(-(y / 6.0) ** 2)
    fin = torch.from_numpy(f.view(np.float64).copy()).cuda()
    fo = f.reshape(-1, p.my)
    refs = {1: np.array([o.deryr(u.real) + 1j * o.deryr(u.imag) for u in fo]),
            2: np.array([o.deryyr(u.real) + 1j * o.deryyr(u.imag) for u in fo])}
    errs = {}
    for op in (1, 2):
        for method in (1, 2):
            out = torch.empty_like(fin)
            torch.cuda.synchronize()
            g.op_y_dense(op, method, fin, out)
            got = out.cpu().numpy().view(np.complex128).reshape(-1, p.my)
            errs[(op, method)] = rel_l2(got, refs[op])
    g.close()
    for k, e in errs.items():
        assert e < BARS[k], (k, e, errs)


@pytest.mark.parametrize("prec", [0, 1])
def test_autotuner_reports_and_chooses(gpu, prec):
    p, y, st = case(64, 64, 129, precision=prec)
    g = Lomacte(p, y)
    g.load_state(st)
    g.step(1)
    for op in (1, 2):
        r = g.yop_tune(op)
        assert all(v > 0 for v in r["ms"].values()), r
        assert r["rel_err_vs_banded"]["dense_fp64"] < BARS[(op, 1)]
        assert r["choice"] in ("banded", "dense_fp64", "dense_3xtf32")
        if prec == 0:  # 3xTF32 is outside the FP64 path's budget
            assert r["choice"] != "dense_3xtf32"
        if r["choice"] != "banded":
            assert r["ms"][r["choice"]] < r["ms"]["banded"]
    # the step still runs after the tuner used the staging buffers
    g.step(1)
    assert np.isfinite(g.diag()["dm"])
    g.close()
