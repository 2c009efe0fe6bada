"""Variable viscosity mu = k = rho D = T^sigma on the CPU: the oracle's
restatement (lmo_set_viscosity) checked without the device.

No lomacte code carries a variable viscosity; the physics follows
branches/loma/src/cross.f:1591-1596 (conduction) and 2177-2196 (stress
tau_ij = 2 T^sigma S_ij, isotropic part in the pressure).  The checks:

* sigma = 0 with the extension on reproduces the constant-viscosity
  substep bit for bit;
* 1-D state (00 modes only), one substep: the increments of T and of the
  00 mode of rho u against an independent evaluation of
  T^sigma (T T'' + sigma T'^2) / Pe - v T' and d/dy((T^sigma - 1) du/dy)/Re;
* uniform T = T0: the run equals a constant-viscosity run at Re / T0^sigma
  up to the truncation difference between d/dy(d/dy) and d2/dy2 (the
  three-dimensional stress, x and z derivatives included);
* x <-> z mirror: swapping the two periodic directions (u <-> w,
  Omega_y -> -Omega_y) commutes with the substep to round-off;
* the passive scalar follows T under the affine map when Re Sc = Pe
  (both equations carry the same T^sigma terms);
* a motionless state with a 3-D temperature perturbation: one substep's
  Delta T equals numpy's dealiased transform of T^sigma (T lap T + sigma
  |grad T|^2) / Pe from the stored spectral T (x and z gradients
  included);
* Omega_y in two modes over a 3-D temperature: the sigma-part of one
  substep's Omega_y increment equals the curl of the divergence of tau'
  formed by numpy (the x and z temperature-gradient terms of the stress
  and its diagonal factor 2 included);
* a motionless state with 3-D T and Z: one substep's Delta Z equals
  numpy's T^sigma (T lap Z + sigma grad T . grad Z) / (Re Sc).
"""
import numpy as np

from oracle.oracle import Oracle
from tests.helpers import FIELDS, case, oracle_for, rel_l2

PR = float(np.float32(0.7))  # Pe = Re*0.7f (main.f:569)


def _run(p, y, st, sigma, n=1, sub=None, Re=None, peclet=None):
    """n RK3 steps (or substep sub) of the oracle; Re, peclet override p's."""
    if Re is None:
        o = oracle_for(p, y, st, nthreads=4)
    else:
        o = Oracle(p.mgalx, p.mgalz, y, Re, p.alp, p.bet, peclet=peclet, cfl=p.cfl, ncfl=p.ncfl, dtmode=1,
                   dt0=p.dt, nthreads=4)
        o.set_state(st["vor"], st["phi"], st["psi"], st["scal"], st["u00"], st["v00"], st["w00"], 0.0)
    if sigma is not None:
        o.set_viscosity(sigma)
    if sub is not None:
        o.substep(sub)
    else:
        o.step(n)
    return o.get_state(), o


def test_sigma_zero_is_the_constant_viscosity_substep():
    p, y, st = case(24, 24, 33)
    a, _ = _run(p, y, st, None, 3)
    b, _ = _run(p, y, st, 0.0, 3)
    c, _ = _run(p, y, st, 0.7, 3)
    for k in FIELDS + ("u00", "v00", "w00"):
        assert np.array_equal(a[k], b[k]), k
    assert rel_l2(c["vor"], a["vor"]) > 1e-5 and rel_l2(c["scal"], a["scal"]) > 1e-6


def _one_d(p, y, st):
    s = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in st.items()}
    for k in ("vor", "phi", "psi", "scal"):
        keep = s[k][0, 0, :].copy()
        s[k][:] = 0
        s[k][0, 0, :] = keep
    s["u00"] = 0.5 * np.tanh(y / 2)
    s["v00"] = 0.01 * np.exp(-y ** 2 / 4)
    return s


def test_one_dimensional_increments():
    sig = 0.7
    p, y, st = case(24, 24, 65, dt=1e-3)
    s = _one_d(p, y, st)
    r0, o = _run(p, y, s, None, sub=0)
    r1, _ = _run(p, y, s, sig, sub=0)
    T, ru, rv = s["scal"][0, 0, :].real, s["u00"], s["v00"]
    h = p.dt * 8.0 / 15.0  # first substep: gamma_1 Deltat, xi_1 = 0
    pe, ire = p.Re * PR, 1.0 / p.Re
    Ty, Tyy = o.deryr(T), o.deryyr(T)
    inner = slice(1, -1)
    dT = (r1["scal"][0, 0, :].real - T) / h
    pred = -T * rv * Ty + T ** sig * (T * Tyy + sig * Ty ** 2) / pe
    assert np.abs(dT - pred)[inner].max() < 1e-8 * np.abs(pred[inner]).max()
    # the 00 mode of rho u: only the stress differs between the two runs
    du = (r1["u00"] - r0["u00"]) / h
    tau = ire * (T ** sig - 1.0) * (T * o.deryr(ru) + ru * Ty)
    pu = o.deryr(tau)
    assert np.abs(pu).max() > 1e-4
    assert np.abs(du - pu)[inner].max() < 1e-8 * np.abs(pu[inner]).max()


def test_uniform_temperature_rescales_reynolds():
    T0, sig, Re = 2.0, 0.7, 160.0
    p, y, st = case(24, 24, 65, dt=0.002)
    s = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in st.items()}
    s["scal"][:] = 0
    s["scal"][0, 0, :] = T0
    pe = Re * 0.7
    a, _ = _run(p, y, s, sig, 5, Re=Re, peclet=pe)
    b, _ = _run(p, y, s, None, 5, Re=Re / T0 ** sig, peclet=pe)
    c, _ = _run(p, y, s, None, 5, Re=Re, peclet=pe)
    for k in ("vor", "phi", "u00", "w00"):
        eff = rel_l2(a[k], c[k])
        assert eff > 1e-6, k
        assert rel_l2(a[k], b[k]) < 1e-3 * eff, (k, rel_l2(a[k], b[k]), eff)


def _swap(a, sign=1.0):
    """f(kx, kz) -> f(kz, kx) on the stored half spectrum [kx >= 0][kz][y]
    (a negative kx taken from the conjugate mode)."""
    nkx, mz, _ = a.shape
    nz1 = (mz - 1) // 2
    assert nkx == nz1 + 1
    out = np.zeros_like(a)
    for i in range(nkx):
        for k in range(mz):
            b = k if k <= nz1 else k - mz
            out[i, k] = a[b, i] if b >= 0 else np.conj(a[-b, (-i) % mz])
    return sign * out


def test_mirror_x_z():
    p, y, st = case(24, 24, 33)
    s2 = dict(st)
    s2["vor"] = _swap(st["vor"], -1.0)
    for k in ("phi", "psi", "scal"):
        s2[k] = _swap(st[k])
    s2["u00"], s2["w00"] = st["w00"].copy(), st["u00"].copy()
    a, _ = _run(p, y, st, 0.7, 3)
    b, _ = _run(p, y, s2, 0.7, 3)
    assert rel_l2(_swap(a["vor"], -1.0), b["vor"]) < 1e-12
    for k in ("phi", "psi", "scal"):
        assert rel_l2(_swap(a[k]), b[k]) < 1e-12, k
    assert np.abs(a["u00"] - b["w00"]).max() < 1e-12 * np.abs(a["u00"]).max()


def test_scalar_follows_temperature_with_sigma():
    p, y, st = case(24, 24, 33)
    o = oracle_for(p, y, st, nthreads=4)
    T = st["scal"]
    tb, tt = T[0, 0, 0].real, T[0, 0, -1].real
    a, b = -tb / (tt - tb), 1.0 / (tt - tb)
    Z = b * T.copy()
    Z[0, 0, :] += a
    o.set_scalar(Z, p.Re * PR / p.Re)
    o.set_viscosity(0.7)
    o.step(5)
    s = o.get_state()
    pred = b * s["scal"]
    pred[0, 0, :] += a
    assert np.abs(o.get_scalar() - pred).max() < 1e-13 * np.abs(pred).max()


def test_viscosity_arguments_checked():
    p, y, st = case(24, 24, 33)
    o = oracle_for(p, y, st, nthreads=1)
    for bad in (-0.1, 4.5, float("nan")):
        try:
            o.set_viscosity(bad)
        except ValueError:
            continue
        raise AssertionError(f"sigma {bad} accepted")


def _phys(c, mgalx, mgalz):
    """half spectrum c[kx >= 0][kz signed] -> real plane [z][x] (e^{+i})"""
    nkx, mz = c.shape
    nz1 = (mz - 1) // 2
    F = np.zeros((mgalz, mgalx), dtype=complex)
    for i in range(nkx):
        for k in range(mz):
            kk = k if k <= nz1 else k - mz
            F[kk % mgalz, i] += c[i, k]
            if i > 0:
                F[(-kk) % mgalz, (-i) % mgalx] += np.conj(c[i, k])
    return np.real(np.fft.ifft2(F)) * mgalx * mgalz


def test_three_dimensional_conduction():
    """A motionless state (rho u = 0) with a 3-D temperature perturbation:
    one substep's Delta T equals the dealiased transform of
    T^sigma (T lap T + sigma |grad T|^2) / Pe, evaluated with numpy from
    the stored spectral T (compact d/dy, d2/dy2 of the oracle per mode)."""
    sig = 0.7
    p, y, st = case(24, 24, 33, dt=1e-3)
    s = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in st.items()}
    for k in ("vor", "phi", "psi"):
        s[k][:] = 0
    for k in ("u00", "v00", "w00"):
        s[k] = np.zeros_like(s[k])
    T = s["scal"]
    T[:, :, :] = 0
    T[0, 0, :] = st["scal"][0, 0, :]
    env = np.exp(-y ** 2 / 8) * (1 - (y / y[-1]) ** 2)      # zero at the walls
    rng = np.random.default_rng(3)
    nkx, mz, my = T.shape
    for (i, k) in ((1, 0), (0, 2), (2, 1), (1, mz - 1), (3, 3)):
        T[i, k, :] = 0.01 * (rng.standard_normal() + 1j * rng.standard_normal()) * env
    r1, o = _run(p, y, s, sig, sub=0)
    dT = r1["scal"] - T
    pe = p.Re * PR
    kxv = p.alp * np.arange(nkx)
    kzv = p.bet * np.array([k if k <= (mz - 1) // 2 else k - mz for k in range(mz)])
    Ty = np.zeros_like(T)
    Tyy = np.zeros_like(T)
    for i in range(nkx):
        for k in range(mz):
            Ty[i, k] = o.deryr(T[i, k].real) + 1j * o.deryr(T[i, k].imag)
            Tyy[i, k] = o.deryyr(T[i, k].real) + 1j * o.deryyr(T[i, k].imag)
    k2 = kxv[:, None, None] ** 2 + kzv[None, :, None] ** 2
    lap = Tyy - k2 * T
    Tx = 1j * kxv[:, None, None] * T
    Tz = 1j * kzv[None, :, None] * T
    h = p.dt * 8.0 / 15.0
    pred = np.zeros_like(T)
    for j in range(1, my - 1):
        ph = {n: _phys(a[:, :, j], p.mgalx, p.mgalz) for n, a in (("T", T), ("x", Tx), ("y", Ty), ("z", Tz), ("l", lap))}
        rhs = ph["T"] ** sig * (ph["T"] * ph["l"] + sig * (ph["x"] ** 2 + ph["y"] ** 2 + ph["z"] ** 2)) / pe
        F = np.fft.fft2(rhs) / (p.mgalx * p.mgalz)
        for i in range(nkx):
            for k in range(mz):
                pred[i, k, j] = h * F[(k if k <= (mz - 1) // 2 else k - mz) % p.mgalz, i]
    inner = (slice(None), slice(None), slice(1, my - 1))
    assert np.abs(pred[inner]).max() > 1e-7
    assert np.abs(dT[inner] - pred[inner]).max() < 1e-9 * np.abs(pred[inner]).max()


def _spec(plane, nkx, mz):
    """real plane [z][x] -> the stored half spectrum [kx][kz] (dealiased)"""
    mgalz, mgalx = plane.shape
    F = np.fft.fft2(plane) / (mgalx * mgalz)
    out = np.zeros((nkx, mz), dtype=complex)
    for k in range(mz):
        out[:, k] = F[(k if k <= (mz - 1) // 2 else k - mz) % mgalz, :nkx]
    return out


def test_three_dimensional_stress():
    """Omega_y in two modes (so rho u = -i kz Omega/k^2, rho w = i kx
    Omega/k^2), u00 a shear profile and a 3-D temperature: the sigma-part
    of one substep's Omega_y increment equals i kz div(tau')_x - i kx
    div(tau')_z with tau'_ij = (T^sigma - 1)(d(u_i)/dx_j + d(u_j)/dx_i)/Re
    formed by numpy (x and z temperature gradients included)."""
    sig = 0.7
    p, y, st = case(24, 24, 33, dt=1e-3)
    nkx, mz, my = st["vor"].shape
    kxv = p.alp * np.arange(nkx)
    kzv = p.bet * np.array([k if k <= (mz - 1) // 2 else k - mz for k in range(mz)])
    env = np.exp(-y ** 2 / 8) * (1 - (y / y[-1]) ** 2)
    rng = np.random.default_rng(4)
    s = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in st.items()}
    s["phi"][:] = 0
    s["psi"][:] = 0
    s["vor"][:] = 0
    for (i, k) in ((1, 2), (2, mz - 1)):
        s["vor"][i, k, :] = 0.05 * (rng.standard_normal() + 1j * rng.standard_normal()) * env
    s["u00"] = 0.5 * np.tanh(y / 2)
    s["v00"] = np.zeros(my)
    s["w00"] = np.zeros(my)
    T = np.zeros_like(s["scal"])
    T[0, 0, :] = st["scal"][0, 0, :]
    for (i, k) in ((1, 0), (0, 2), (2, 1), (1, mz - 1)):
        T[i, k, :] = 0.01 * (rng.standard_normal() + 1j * rng.standard_normal()) * env
    s["scal"] = T
    r1, o = _run(p, y, s, sig, sub=0)
    r0, _ = _run(p, y, s, None, sub=0)
    h = p.dt * 8.0 / 15.0
    got = (r1["vor"] - r0["vor"]) / h

    def dy(a):
        out = np.zeros_like(a)
        for i in range(nkx):
            for k in range(mz):
                out[i, k] = o.deryr(a[i, k].real) + 1j * o.deryr(a[i, k].imag)
        return out

    vo = s["vor"].copy()
    vo[:, :, 0], vo[:, :, -1] = vo[:, :, 1], vo[:, :, -2]  # the wall condition of Omega_y (cross.f:315-327)
    k2 = kxv[:, None, None] ** 2 + kzv[None, :, None] ** 2
    k2[0, 0] = 1.0
    IX, IZ = 1j * kxv[:, None, None], 1j * kzv[None, :, None]
    ru, rw = -IZ * vo / k2, IX * vo / k2
    ru[0, 0], rw[0, 0] = s["u00"], 0.0
    rv = np.zeros_like(ru)
    dru, drw = dy(ru), dy(rw)
    g = {"xx": IX * ru, "yy": dy(rv), "zz": IZ * rw, "xy": dru + IX * rv, "xz": IZ * ru + IX * rw,
         "yz": IZ * rv + drw}
    grads = {"x": IX * T, "y": dy(T), "z": IZ * T}
    tau = {n: np.zeros_like(T) for n in g}
    ire = 1.0 / p.Re
    for j in range(my):
        P = lambda a: _phys(a[:, :, j], p.mgalx, p.mgalz)  # noqa: E731
        Tp, u, v, w = P(T), P(ru), P(rv), P(rw)
        tx, ty, tz = P(grads["x"]), P(grads["y"]), P(grads["z"])
        c = ire * (Tp ** sig - 1.0)
        phys = {"xx": 2 * c * (Tp * P(g["xx"]) + u * tx), "yy": 2 * c * (Tp * P(g["yy"]) + v * ty),
                "zz": 2 * c * (Tp * P(g["zz"]) + w * tz), "xy": c * (Tp * P(g["xy"]) + u * ty + v * tx),
                "xz": c * (Tp * P(g["xz"]) + u * tz + w * tx), "yz": c * (Tp * P(g["yz"]) + v * tz + w * ty)}
        for n in tau:
            tau[n][:, :, j] = _spec(phys[n], nkx, mz)
    fx = IX * tau["xx"] + dy(tau["xy"]) + IZ * tau["xz"]
    fz = IX * tau["xz"] + dy(tau["yz"]) + IZ * tau["zz"]
    pred = IZ * fx - IX * fz
    inner = (slice(None), slice(None), slice(1, my - 1))
    assert np.abs(pred[inner]).max() > 1e-6
    assert np.abs(got[inner] - pred[inner]).max() < 1e-8 * np.abs(pred[inner]).max()


def test_three_dimensional_scalar_diffusion():
    """A motionless state with 3-D T and Z: one substep's Delta Z equals
    numpy's dealiased transform of T^sigma (T lap Z + sigma grad T . grad
    Z) / (Re Sc)."""
    sig, sc = 0.7, 1.3
    p, y, st = case(24, 24, 33, dt=1e-3)
    nkx, mz, my = st["vor"].shape
    s = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in st.items()}
    for k in ("vor", "phi", "psi"):
        s[k][:] = 0
    for k in ("u00", "v00", "w00"):
        s[k] = np.zeros_like(s[k])
    env = np.exp(-y ** 2 / 8) * (1 - (y / y[-1]) ** 2)
    rng = np.random.default_rng(7)
    T = np.zeros_like(s["scal"])
    T[0, 0, :] = st["scal"][0, 0, :]
    Z = np.zeros_like(T)
    Z[0, 0, :] = 0.5 * (1 + np.tanh(y / 2))
    Z[0, 0, 0], Z[0, 0, -1] = 0.0, 1.0
    for (i, k) in ((1, 0), (0, 2), (2, 1)):
        T[i, k, :] = 0.01 * (rng.standard_normal() + 1j * rng.standard_normal()) * env
    for (i, k) in ((1, 0), (1, mz - 1), (3, 2)):
        Z[i, k, :] = 0.02 * (rng.standard_normal() + 1j * rng.standard_normal()) * env
    s["scal"] = T
    o = oracle_for(p, y, s, nthreads=4)
    o.set_scalar(Z, sc)
    o.set_viscosity(sig)
    o.substep(0)
    dZ = o.get_scalar() - Z
    kxv = p.alp * np.arange(nkx)
    kzv = p.bet * np.array([k if k <= (mz - 1) // 2 else k - mz for k in range(mz)])
    IX, IZ = 1j * kxv[:, None, None], 1j * kzv[None, :, None]

    def dy(a, f):
        r = np.zeros_like(a)
        for i in range(nkx):
            for k in range(mz):
                r[i, k] = f(a[i, k].real) + 1j * f(a[i, k].imag)
        return r

    lapZ = dy(Z, o.deryyr) - (kxv[:, None, None] ** 2 + kzv[None, :, None] ** 2) * Z
    tg = (IX * T, dy(T, o.deryr), IZ * T)
    zg = (IX * Z, dy(Z, o.deryr), IZ * Z)
    h = p.dt * 8.0 / 15.0
    pred = np.zeros_like(Z)
    for j in range(1, my - 1):
        P = lambda a: _phys(a[:, :, j], p.mgalx, p.mgalz)  # noqa: E731
        Tp = P(T)
        rhs = Tp ** sig * (Tp * P(lapZ) + sig * sum(P(a) * P(b) for a, b in zip(tg, zg))) / (p.Re * sc)
        pred[:, :, j] = h * _spec(rhs, nkx, mz)
    inner = (slice(None), slice(None), slice(1, my - 1))
    assert np.abs(pred[inner]).max() > 1e-8
    assert np.abs(dZ[inner] - pred[inner]).max() < 1e-9 * np.abs(pred[inner]).max()


def test_mass_with_variable_viscosity():
    """Impermeable walls: the total mass (masst, the integral of the plane
    mean of rho = 1/T) stays within 1e-5 of its start over 30 steps with
    mu = T^0.7, as it does with constant viscosity."""
    p, y, st = case(24, 24, 65)
    out = []
    for sig in (None, 0.7):
        o = oracle_for(p, y, st, nthreads=4)
        if sig is not None:
            o.set_viscosity(sig)
        m = []
        for _ in range(30):
            o.step(1)
            m.append(o.diag()["masst"])
        out.append(abs(m[-1] - m[0]) / m[0])
    assert out[1] < 1e-5 and out[0] < 1e-5


def test_extensions_golden():
    """The oracle's scalar and variable-viscosity run against its committed
    regression pin (tests/golden/make_extension_golden.py)."""
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_extension_golden as g
    ref = np.load(os.path.join(os.path.dirname(__file__), "golden", "extensions_24x33x24.npz"))
    s = g.run()
    assert np.allclose(s["u00"], ref["u00"], rtol=0, atol=1e-13 * np.abs(ref["u00"]).max())
    for k in g.FIELDS:
        n = float(ref[k + "_norm"])
        assert abs(np.linalg.norm(s[k]) - n) <= 1e-12 * n, k
        got = s[k][g.sample_index(s[k].shape)]
        assert np.abs(got - ref[k + "_sample"]).max() <= 1e-12 * n, k
