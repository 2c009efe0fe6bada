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


def _band(B, v, h):
    """Rows of a band matrix (entry c of row j at column j - h + c) times v."""
    n = len(v)
    out = np.zeros(n, dtype=np.result_type(B, v))
    for c in range(2 * h + 1):
        lo, hi = max(0, h - c), min(n, n + h - c)
        out[lo:hi] += B[lo:hi, c] * v[lo - h + c:hi - h + c]
    return out


def test_initloma3_divergence_residual():
    """initloma3's check of the decomposition it writes
    (trunk/initloma3/src/main.f:473-523): the divergence of the seeded
    momentum, div = i kx rho u + d(rho v)/dy + i kz rho w, is the source of
    the Dirichlet Poisson problem whose solution is the state's psi
    (Lapvdvhom).  Known answer: zero residual of the compact-scheme system
    (dt22 - k^2 dt21) psi = dt21 div on the interior rows, psi = 0 at the
    walls; solvepsi on the same source has the same interior residual and a
    zero dpsi/dy at both walls (laps.f:580-764)."""
    from oracle.ic import make_ic
    y = stretched_mesh(97)
    o = Oracle(48, 48, y, 160.0, 0.25, 0.25, nthreads=1)
    st = make_ic(48, 48, y, s=4.0, seed=5, momentum=True)
    c = o.coefs()
    nkx, mz, my = st["psi"].shape
    kx = 0.25 * np.arange(nkx)
    kz = 0.25 * np.array([k if k <= (mz - 1) // 2 else k - mz for k in range(mz)])
    worst = [0.0, 0.0, 0.0]
    checked = 0
    for i in range(nkx):
        for k in range(mz):
            k2 = kx[i] ** 2 + kz[k] ** 2
            rv = st["rv"][i, k]
            if k2 == 0.0 or not np.any(rv):
                continue
            dv = o.deryr(rv.real) + 1j * o.deryr(rv.imag)
            div = 1j * kx[i] * st["ru"][i, k] + dv + 1j * kz[k] * st["rw"][i, k]
            psi = st["psi"][i, k]
            lhs = _band(c["dt22"], psi, 2) - k2 * _band(c["dt21"], psi, 2)
            rhs = _band(c["dt21"], div, 2)
            scale = np.abs(rhs).max()
            worst[0] = max(worst[0], np.abs(lhs - rhs)[1:-1].max() / scale)
            assert psi[0] == 0 and psi[-1] == 0
            p2, dp2 = o.solvepsi(div, k2)
            lhs2 = _band(c["dt22"], p2, 2) - k2 * _band(c["dt21"], p2, 2)
            worst[1] = max(worst[1], np.abs(lhs2 - rhs)[1:-1].max() / scale)
            worst[2] = max(worst[2], abs(dp2[0]) / np.abs(dp2).max(), abs(dp2[-1]) / np.abs(dp2).max())
            checked += 1
    assert checked > 50
    assert worst[0] < 1e-12 and worst[1] < 1e-12 and worst[2] < 1e-12, worst
