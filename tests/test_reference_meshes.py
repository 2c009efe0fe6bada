"""The y operators on the reference's own meshes.

trunk/initloma3 reads its y mesh from a file (list-directed y(1..my),
main.f:726-727) and builds the compact-scheme matrices on it (derivadas,
main.f:753); the three meshes here are copies of files it ships
(tests/golden/make_golden.py): a symmetric s = 8 mesh, the Pantano-case
mesh and an 801-point mesh whose last point stops short of symmetry.  On
each, the library's host-side metrics are compared with the oracle's, and
the oracle's operators meet the known answers of test_oracle_ops.py:
exactness on low-degree polynomials, the compact-scheme systems of
Lapvdvhom and solvepsi solved to round-off with their wall conditions
(laps.f:319-764), and inty8 inverting d/dy.
"""
import os

import numpy as np
import pytest

from loma_phd_b200 import y_metrics
from oracle.oracle import Oracle
from tests.test_oracle_ops import _band

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MESHES = ("meshs8Ly173", "pantanoBmy387", "LOMAmy801")


@pytest.fixture(scope="module", params=MESHES)
def mesh(request):
    y = np.loadtxt(os.path.join(GOLDEN, f"mesh_{request.param}.txt")).ravel()
    return y, Oracle(6, 3, y, 160.0, 0.25, 0.25, nthreads=1)


def test_mesh_files_are_increasing(mesh):
    y, _ = mesh
    assert len(y) in (387, 453, 801)
    assert np.all(np.diff(y) > 0)


def test_library_metrics_match_oracle(mesh):
    """fmap (1 / (dy/deta) of the compact scheme), hy and the trapezoidal
    half-weights trp = (y(j+1) - y(j-1)) / 4 (trunk/lomacte3/src/main.f:
    689-697), from the library's host code, against the oracle and against
    their definitions."""
    y, o = mesh
    m = y_metrics(y)
    assert np.allclose(m["fmap"], o.coefs()["fmap"], rtol=1e-12, atol=0)
    assert np.array_equal(m["hy"][1:-1], 0.5 * (y[2:] - y[:-2]))
    L = y[-1] - y[0]
    assert 2 * m["trp"].sum() == pytest.approx(L, rel=1e-13)
    assert 2 * (m["trp"] * y).sum() == pytest.approx(0.5 * (y[-1] ** 2 - y[0] ** 2), abs=1e-10 * L * L)


def test_derivatives_on_reference_mesh(mesh):
    y, o = mesh
    assert np.abs(o.deryr(y) - 1).max() < 1e-13
    assert np.abs(o.deryyr(y ** 2) - 2).max() < 1e-6
    f = np.tanh(y / 8)
    d1 = (1 - f ** 2) / 8
    d2 = -2 * f * (1 - f ** 2) / 64
    assert np.abs(o.deryr(f) - d1).max() < 1e-4 * np.abs(d1).max()
    assert np.abs(o.deryyr(f) - d2).max() < 1e-6 * np.abs(d2).max()
    g = np.exp(-(y / 8) ** 2)
    u = o.inty8(-2 * y / 64 * g)
    assert u[0] == 0.0 and np.abs(u - (g - g[0])).max() < 1e-5


@pytest.mark.parametrize("k2", [0.0625, 1.0])
def test_poisson_systems_on_reference_mesh(mesh, k2):
    """Lapvdvhom: (dt22 - k^2 dt21) v = dt21 phi on the interior rows with
    v = 0 at the walls, and dv/dy its compact derivative; solvepsi: the same
    interior system with dv/dy = 0 at both walls."""
    y, o = mesh
    c = o.coefs()
    phi = np.sin(np.pi * (y - y[0]) / (y[-1] - y[0])) * (1 + 0.5j)
    rhs = _band(c["dt21"], phi, 2)
    scale = np.abs(rhs).max()
    v, dv = o.lapvdvhom(phi, k2)
    assert v[0] == 0 and v[-1] == 0
    lhs = _band(c["dt22"], v, 2) - k2 * _band(c["dt21"], v, 2)
    assert np.abs(lhs - rhs)[1:-1].max() < 1e-12 * scale
    assert np.abs(dv - (o.deryr(v.real) + 1j * o.deryr(v.imag))).max() < 1e-12 * np.abs(dv).max()
    p, dp = o.solvepsi(phi, k2)
    lhs = _band(c["dt22"], p, 2) - k2 * _band(c["dt21"], p, 2)
    assert np.abs(lhs - rhs)[1:-1].max() < 1e-12 * scale
    assert abs(dp[0]) < 1e-14 * np.abs(dp).max() and abs(dp[-1]) < 1e-14 * np.abs(dp).max()
