"""Why the y-derivatives stay banded FP64 solves and are not applied as a
dense operator on the tensor cores.

The compact schemes d/dy (deryr2, cfdiff.f:518-601) and d2/dy2 (deryyr2,
cfdiff.f:735-797) are mode-independent, so each is one dense my x my
matrix D = P^-1 Q, and applying it to every mode at once is a GEMM
[my x my] x [my x 2 nmode] that tcgen05 could run in split precision
(3xTF32: hi*hi + hi*lo + lo*hi, FP32 accumulation).  This test builds D from
the oracle's banded operators and measures, on the seeded initial condition
at 64^2 x 257, the error of that split-precision product against the FP64
product: about 1e-6 for d/dy but 1e-5 .. 1e-4 for d2/dy2 (the rows of the
dense d2/dy2 operator sum to ~3e3 in magnitude against O(1) results, so
round-off of the inputs alone is amplified by that much).  The mixed form's
budget is <= 1e-5 per field after 1000 steps, so the y-operators stay
banded solves in FP64 on the FP32-stored fields; the banded form also moves
fewer bytes (no my x my operator reads) than the GEMM would.
"""
import numpy as np
import pytest

from tests.helpers import case, oracle_for


def _tf32(x):
    """round FP32 values to TF32 (10 explicit mantissa bits, nearest)"""
    b = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    return (((b + 0x1000) & 0xFFFFE000).astype(np.uint32)).view(np.float32)


def _mm3(A, X):
    A = A.astype(np.float32)
    X = X.astype(np.float32)
    ah, xh = _tf32(A), _tf32(X)
    al, xl = _tf32(A - ah), _tf32(X - xh)
    f = lambda a, b: (a.astype(np.float64) @ b.astype(np.float64)).astype(np.float32)
    return (f(ah, xh) + f(ah, xl) + f(al, xh)).astype(np.float64)


@pytest.fixture(scope="module")
def ops():
    p, y, st = case(64, 64, 257)
    o = oracle_for(p, y, st, nthreads=4)
    my = p.my
    D1 = np.zeros((my, my))
    D2 = np.zeros((my, my))
    for k in range(my):
        e = np.zeros(my)
        e[k] = 1.0
        D1[:, k] = o.deryr(e)
        D2[:, k] = o.deryyr(e)
    fields = {}
    for name in ("vor", "phi", "psi"):
        F = st[name].reshape(-1, my).T[:, 1:]  # [my][modes], the 00 mode excluded
        F = np.concatenate([F.real, F.imag], axis=1)
        fields[name] = F[:, np.abs(F).max(axis=0) > 0]
    return D1, D2, fields


def _rel(D, F):
    ref = D @ F
    return np.linalg.norm(_mm3(D, F) - ref) / np.linalg.norm(ref)


def test_first_derivative_split_precision_error(ops):
    D1, _, fields = ops
    errs = {k: _rel(D1, F) for k, F in fields.items()}
    assert all(1e-8 < e < 1e-5 for e in errs.values()), errs


def test_second_derivative_split_precision_exceeds_budget(ops):
    _, D2, fields = ops
    errs = {k: _rel(D2, F) for k, F in fields.items()}
    assert max(errs.values()) > 1e-5, errs
    assert np.abs(D2).sum(axis=1).max() > 1e3
