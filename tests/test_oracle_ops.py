"""Known-answer tests of the oracle's y-operators, following the reference's
own numerical harnesses: analytic derivatives on a stretched mesh
(trunk/mixing/test/test.f:182-200, branches/reactml/benchmark_fft/main.f:46-74)
and manufactured Poisson problems (laps.f:319-764)."""
import numpy as np
import pytest

from loma_phd_b200 import stretched_mesh
from oracle.oracle import Oracle


@pytest.fixture(scope="module")
def o():
    y = stretched_mesh(129)
    return Oracle(96, 96, y, 160.0, 0.25, 0.25, nthreads=2)


def test_derivatives_of_polynomials_are_exact(o):
    y = o.y
    # the first derivative acts on uniform eta with the metric fmap, so it is
    # exact for y itself; the second acts on the actual mesh (Taylor matched)
    assert np.abs(o.deryr(y) - 1).max() < 1e-13
    assert np.abs(o.deryyr(y ** 2) - 2).max() < 1e-9
    assert np.abs(o.deryyr(y ** 3) - 6 * y).max() < 1e-8


def test_derivative_of_windowed_sine_converges(o):
    # benchmark_fft/main.f:48-59: f = exp(-(y/swin)^2) sin(ky y)
    swin = 8.0
    errs1, errs2 = [], []
    for my in (65, 129, 257):
        yy = stretched_mesh(my)
        oo = Oracle(96, 96, yy, 160.0, 0.25, 0.25, nthreads=1)
        ky = 0.4
        g = np.exp(-(yy / swin) ** 2)
        f = g * np.sin(ky * yy)
        df = g * (ky * np.cos(ky * yy) - 2 * yy / swin ** 2 * np.sin(ky * yy))
        d2f = g * (-2 / swin ** 2 * np.sin(ky * yy) + 4 * yy ** 2 / swin ** 4 * np.sin(ky * yy)
                   - 4 * yy / swin ** 2 * ky * np.cos(ky * yy) - ky ** 2 * np.sin(ky * yy))
        errs1.append(np.abs(oo.deryr(f) - df).max())
        errs2.append(np.abs(oo.deryyr(f) - d2f).max())
    assert errs1[-1] < errs1[0] / 8 and errs1[-1] < 5e-4  # 2nd-order wall closures
    assert errs2[-1] < errs2[0] / 8 and errs2[-1] < 1e-5


def test_inty8_inverts_derivative(o):
    y = o.y
    g = np.exp(-(y / 4) ** 2)
    u = o.inty8(-2 * y / 16 * g)
    assert u[0] == 0.0
    assert np.abs(u - (g - g[0])).max() < 1e-5


def test_lapvdvhom_dirichlet(o):
    y = o.y
    phi = np.sin(np.pi * (y - y[0]) / (y[-1] - y[0])) * (1 + 0.5j)
    for k2 in (0.0625, 0.5, 4.0):
        v, dv = o.lapvdvhom(phi, k2)
        assert v[0] == 0 and v[-1] == 0
        assert np.abs(dv - (o.deryr(v.real) + 1j * o.deryr(v.imag))).max() < 1e-12
        r = o.deryyr(v.real) - k2 * v.real - phi.real
        assert np.abs(r[3:-3]).max() < 1e-6
    v, dv = o.lapvdvhom(phi, 0.0)
    assert not v.any() and not dv.any()


def test_solvepsi_neumann(o):
    y = o.y
    phi = np.exp(-(y / 3) ** 2) * (0.3 - 1.2j)
    for k2 in (0.0625, 1.0):
        v, dv = o.solvepsi(phi, k2)
        assert abs(dv[0]) < 1e-12 and abs(dv[-1]) < 1e-12
        r = o.deryyr(v.real) - k2 * v.real - phi.real
        assert np.abs(r[4:-4]).max() < 1e-4 * np.abs(phi).max()
