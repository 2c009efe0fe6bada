"""The oracle's Omega_y and phi equations (trunk/lomacte3/src/
cross.f:652-921) and T equation (cross.f:1625-1647) against the physics
evaluated independently with numpy, on the CPU.

State: Omega_y in two modes (so rho u = -i kz Omega/k^2, rho w = i kx
Omega/k^2, rho v = 0), a shear profile in the 00 mode of rho u, a 3-D
temperature.  numpy forms the velocity u_i = T rho u_i and the fluxes
rho u_i u_j on the 3/2 grid, transforms and truncates them, and builds
RHS(Omega_y) = i kz N_x - i kx N_z + lap(omega_y)/Re with N_i = -d_j(rho
u_i u_j) and omega_y = i kz u - i kx w from the dealiased velocity (d/dy
and d2/dy2 by the compact schemes the oracle exposes).  One substep's
Omega_y increment (gamma_1 Deltat RHS, xi_1 = 0) must match it; the same
for phi and for T with RHS(T) = -u.grad T + T lap T / Pe; and the
divergence constraint: the d(rho)/dt source of the psi solve from the T
update through rho = 1/T.
"""
import numpy as np

from tests.helpers import case, oracle_for


def _phys(c, mgalx, mgalz):
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


def _spec(plane, nkx, mz):
    mgalz, mgalx = plane.shape
    F = np.fft.fft2(plane) / (mgalx * mgalz)
    out = np.zeros((nkx, mz), dtype=complex)
    for k in range(mz):
        out[:, k] = F[(k if k <= (mz - 1) // 2 else k - mz) % mgalz, :nkx]
    return out


def _state():
    """Omega_y in three modes, a shear profile in rho u00, a 3-D T."""
    p, y, st = case(24, 24, 33, dt=1e-3)
    nkx, mz, my = st["vor"].shape
    kxv = p.alp * np.arange(nkx)
    kzv = p.bet * np.array([k if k <= (mz - 1) // 2 else k - mz for k in range(mz)])
    env = np.exp(-y ** 2 / 8) * (1 - (y / y[-1]) ** 2)
    rng = np.random.default_rng(8)
    s = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in st.items()}
    s["phi"][:] = 0
    s["psi"][:] = 0
    s["vor"][:] = 0
    for (i, k) in ((1, 2), (2, mz - 1), (1, 0)):
        s["vor"][i, k, :] = 0.05 * (rng.standard_normal() + 1j * rng.standard_normal()) * env
    s["u00"], s["v00"], s["w00"] = 0.5 * np.tanh(y / 2), np.zeros(my), np.zeros(my)
    T = np.zeros_like(s["scal"])
    T[0, 0, :] = st["scal"][0, 0, :]
    for (i, k) in ((1, 0), (0, 2), (2, 1)):
        T[i, k, :] = 0.01 * (rng.standard_normal() + 1j * rng.standard_normal()) * env
    s["scal"] = T
    return p, y, s, kxv, kzv


def _dy(o, a, f):
    nkx, mz, _ = a.shape
    r = np.zeros_like(a)
    for i in range(nkx):
        for k in range(mz):
            r[i, k] = f(a[i, k].real) + 1j * f(a[i, k].imag)
    return r


def _momentum(p, s, kxv, kzv):
    """rho u_i of the state (rho v = 0): -i kz Omega/k^2, i kx Omega/k^2,
    the 00 profile in rho u; Omega_y with its wall values (cross.f:315-327)"""
    vo = s["vor"].copy()
    vo[:, :, 0], vo[:, :, -1] = vo[:, :, 1], vo[:, :, -2]
    k2 = kxv[:, None, None] ** 2 + kzv[None, :, None] ** 2
    k2[0, 0] = 1.0
    IX, IZ = 1j * kxv[:, None, None], 1j * kzv[None, :, None]
    m = {"x": -IZ * vo / k2, "y": np.zeros_like(vo), "z": IX * vo / k2}
    m["x"][0, 0], m["z"][0, 0] = s["u00"], 0.0
    return m


def test_vorticity_equation_against_numpy():
    p, y, s, kxv, kzv = _state()
    nkx, mz, my = s["vor"].shape
    T = s["scal"]
    o = oracle_for(p, y, s, nthreads=2)
    o.substep(0)
    h = p.dt * 8.0 / 15.0
    got = (o.get_state()["vor"] - s["vor"]) / h

    def dy(a, f):
        return _dy(o, a, f)

    k2 = kxv[:, None, None] ** 2 + kzv[None, :, None] ** 2
    IX, IZ = 1j * kxv[:, None, None], 1j * kzv[None, :, None]
    m = _momentum(p, s, kxv, kzv)
    pairs = ("xx", "xy", "xz", "yz", "zz")
    M = {n: np.zeros_like(T) for n in pairs}
    U = {c: np.zeros_like(T) for c in "xz"}
    for j in range(my):
        P = lambda a: _phys(a[:, :, j], p.mgalx, p.mgalz)  # noqa: E731
        Tp = P(T)
        mp = {c: P(m[c]) for c in "xyz"}
        up = {c: mp[c] * Tp for c in "xyz"}
        for n in pairs:
            M[n][:, :, j] = _spec(mp[n[0]] * up[n[1]], nkx, mz)
        for c in "xz":
            U[c][:, :, j] = _spec(up[c], nkx, mz)
    Nx = -(IX * M["xx"] + dy(M["xy"], o.deryr) + IZ * M["xz"])
    Nz = -(IX * M["xz"] + dy(M["yz"], o.deryr) + IZ * M["zz"])
    wy = IZ * U["x"] - IX * U["z"]
    lap = dy(wy, o.deryyr) - k2 * wy
    pred = IZ * Nx - IX * Nz + lap / p.Re
    inner = (slice(None), slice(None), slice(1, my - 1))
    assert np.abs(pred[inner]).max() > 1e-4
    assert np.abs(got[inner] - pred[inner]).max() < 1e-9 * np.abs(pred[inner]).max()


def test_temperature_equation_against_numpy():
    """RHS(T) = -u.grad T + T lap T / Pe (cross.f:1631-1637) on the 3/2 grid,
    transformed and truncated: one substep's Delta T (gamma_1 Deltat
    RHS(T), the physical accumulator starting at zero)."""
    p, y, s, kxv, kzv = _state()
    nkx, mz, my = s["vor"].shape
    T = s["scal"]
    o = oracle_for(p, y, s, nthreads=2)
    o.substep(0)
    h = p.dt * 8.0 / 15.0
    got = (o.get_state()["scal"] - T) / h
    IX, IZ = 1j * kxv[:, None, None], 1j * kzv[None, :, None]
    k2 = kxv[:, None, None] ** 2 + kzv[None, :, None] ** 2
    m = _momentum(p, s, kxv, kzv)
    ty = _dy(o, T, o.deryr)
    lap = _dy(o, T, o.deryyr) - k2 * T
    pe = p.Re * float(np.float32(0.7))
    pred = np.zeros_like(T)
    for j in range(1, my - 1):
        P = lambda a: _phys(a[:, :, j], p.mgalx, p.mgalz)  # noqa: E731
        Tp = P(T)
        rhs = -(P(m["x"]) * Tp * P(IX * T) + P(m["y"]) * Tp * P(ty) + P(m["z"]) * Tp * P(IZ * T)) + Tp * P(lap) / pe
        pred[:, :, j] = _spec(rhs, nkx, mz)
    inner = (slice(None), slice(None), slice(1, my - 1))
    assert np.abs(pred[inner]).max() > 1e-5
    assert np.abs(got[inner] - pred[inner]).max() < 1e-9 * np.abs(pred[inner]).max()


def test_phi_equation_against_numpy():
    """RHS(phi) = -k^2 N_y - d/dy(i kx N_x + i kz N_z) - lap(i kz omega_x -
    i kx omega_z)/Re (cross.f:748-921) with N_i = -d_j(rho u_i u_j) and the
    vorticity of the dealiased velocity; here rho v = 0, so N_y = 0,
    omega_x = dw/dy and omega_z = -du/dy."""
    p, y, s, kxv, kzv = _state()
    nkx, mz, my = s["vor"].shape
    T = s["scal"]
    o = oracle_for(p, y, s, nthreads=2)
    o.substep(0)
    h = p.dt * 8.0 / 15.0
    got = (o.get_state()["phi"] - s["phi"]) / h
    IX, IZ = 1j * kxv[:, None, None], 1j * kzv[None, :, None]
    k2 = kxv[:, None, None] ** 2 + kzv[None, :, None] ** 2
    m = _momentum(p, s, kxv, kzv)
    pairs = ("xx", "xy", "xz", "yz", "zz")
    M = {n: np.zeros_like(T) for n in pairs}
    U = {c: np.zeros_like(T) for c in "xz"}
    for j in range(my):
        P = lambda a: _phys(a[:, :, j], p.mgalx, p.mgalz)  # noqa: E731
        Tp = P(T)
        mp = {c: P(m[c]) for c in "xyz"}
        up = {c: mp[c] * Tp for c in "xyz"}
        for n in pairs:
            M[n][:, :, j] = _spec(mp[n[0]] * up[n[1]], nkx, mz)
        for c in "xz":
            U[c][:, :, j] = _spec(up[c], nkx, mz)
    Nx = -(IX * M["xx"] + _dy(o, M["xy"], o.deryr) + IZ * M["xz"])
    Nz = -(IX * M["xz"] + _dy(o, M["yz"], o.deryr) + IZ * M["zz"])
    wx, wz = _dy(o, U["z"], o.deryr), -_dy(o, U["x"], o.deryr)
    cc = IZ * wx - IX * wz
    lap = _dy(o, cc, o.deryyr) - k2 * cc
    pred = -_dy(o, IX * Nx + IZ * Nz, o.deryr) - lap / p.Re
    inner = (slice(None), slice(None), slice(1, my - 1))
    assert np.abs(pred[inner]).max() > 1e-5
    assert np.abs(got[inner] - pred[inner]).max() < 1e-9 * np.abs(pred[inner]).max()


def test_divergence_constraint_against_numpy():
    """A motionless state with a 3-D temperature: the d(rho)/dt source of
    the psi solve (cross.f:1669-1673, rho = 1/T with T advanced by one
    substep of conduction) evaluated with numpy on the 3/2 grid and
    transformed; psi(n+1) of the oracle's substep equals the oracle's
    Neumann Poisson solve (solvepsi) of that source, mode by mode."""
    p, y, st = case(24, 24, 33, dt=1e-3)
    nkx, mz, my = st["vor"].shape
    kxv = p.alp * np.arange(nkx)
    kzv = p.bet * np.array([k if k <= (mz - 1) // 2 else k - mz for k in range(mz)])
    env = np.exp(-y ** 2 / 8) * (1 - (y / y[-1]) ** 2)
    rng = np.random.default_rng(9)
    s = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in st.items()}
    for k in ("vor", "phi", "psi"):
        s[k][:] = 0
    for k in ("u00", "v00", "w00"):
        s[k] = np.zeros_like(s[k])
    T = np.zeros_like(s["scal"])
    T[0, 0, :] = st["scal"][0, 0, :]
    for (i, k) in ((1, 0), (0, 2), (2, 1), (1, mz - 1)):
        T[i, k, :] = 0.01 * (rng.standard_normal() + 1j * rng.standard_normal()) * env
    s["scal"] = T
    o = oracle_for(p, y, s, nthreads=2)
    o.substep(0)
    psi = o.get_state()["psi"]
    # RK3 coefficients of the first substep (modulos.f:193-209)
    gama0, p0 = 8.0 / 15.0, 5.0 / 66.0
    beta0, alpha0 = gama0 - p0, p0
    dtg, dtb, ab = p.dt * gama0, p.dt * beta0, alpha0 / beta0
    pe = p.Re * float(np.float32(0.7))
    k2 = kxv[:, None, None] ** 2 + kzv[None, :, None] ** 2
    lap = _dy(o, T, o.deryyr) - k2 * T
    drho = np.zeros_like(T)
    for j in range(my):
        P = lambda a: _phys(a[:, :, j], p.mgalx, p.mgalz)  # noqa: E731
        Tp = P(T)
        rhs = Tp * P(lap) / pe
        d8 = dtg * rhs
        tn = Tp + d8
        drho[:, :, j] = _spec((d8 / (Tp * tn)) / dtb - ab * rhs / (Tp * Tp), nkx, mz)
    pred = np.zeros_like(psi)
    for i in range(nkx):
        for k in range(mz):
            if i == 0 and k == 0:
                continue
            pred[i, k], _ = o.solvepsi(drho[i, k], float(k2[i, k, 0]))
    mask = np.ones((nkx, mz), bool)
    mask[0, 0] = False
    assert np.abs(pred[mask]).max() > 1e-8
    assert np.abs(psi[mask] - pred[mask]).max() < 1e-9 * np.abs(pred[mask]).max()


def test_all_terms_with_phi():
    """Omega_y and phi in several modes (rho v from the oracle's Lapvdvhom,
    cross.f:365-372: rho u = (i kx dm_y/dy - i kz Omega)/k^2, rho v = m_y,
    rho w = (i kz dm_y/dy + i kx Omega)/k^2), a shear profile, a 3-D T:
    every advective term active.  One substep's increments of Omega_y, phi,
    T and the 00 mode of rho u (its RHS -d(rho u v)_00/dy + d2(u_00)/dy2 /
    Re, cross.f:686-722) against numpy."""
    p, y, st = case(24, 24, 33, dt=1e-3)
    nkx, mz, my = st["vor"].shape
    kxv = p.alp * np.arange(nkx)
    kzv = p.bet * np.array([k if k <= (mz - 1) // 2 else k - mz for k in range(mz)])
    env = np.exp(-y ** 2 / 8) * (1 - (y / y[-1]) ** 2)
    rng = np.random.default_rng(10)
    s = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in st.items()}
    for k in ("vor", "phi", "psi"):
        s[k][:] = 0
    for (i, k) in ((1, 2), (2, mz - 1)):
        s["vor"][i, k, :] = 0.05 * (rng.standard_normal() + 1j * rng.standard_normal()) * env
    for (i, k) in ((1, 1), (0, 3), (2, mz - 2)):
        s["phi"][i, k, :] = 0.05 * (rng.standard_normal() + 1j * rng.standard_normal()) * env
    s["u00"], s["v00"], s["w00"] = 0.5 * np.tanh(y / 2), np.zeros(my), np.zeros(my)
    T = np.zeros_like(s["scal"])
    T[0, 0, :] = st["scal"][0, 0, :]
    for (i, k) in ((1, 0), (0, 2), (2, 1)):
        T[i, k, :] = 0.01 * (rng.standard_normal() + 1j * rng.standard_normal()) * env
    s["scal"] = T
    o = oracle_for(p, y, s, nthreads=2)
    o.substep(0)
    new = o.get_state()
    h = p.dt * 8.0 / 15.0
    IX, IZ = 1j * kxv[:, None, None], 1j * kzv[None, :, None]
    k2 = kxv[:, None, None] ** 2 + kzv[None, :, None] ** 2
    k2s = k2.copy()
    k2s[0, 0] = 1.0
    vo = s["vor"].copy()
    vo[:, :, 0], vo[:, :, -1] = vo[:, :, 1], vo[:, :, -2]
    my_, dmy = np.zeros_like(T), np.zeros_like(T)
    for i in range(nkx):
        for k in range(mz):
            my_[i, k], dmy[i, k] = o.lapvdvhom(s["phi"][i, k], float(k2[i, k, 0]))
    m = {"x": (IX * dmy - IZ * vo) / k2s, "y": my_, "z": (IZ * dmy + IX * vo) / k2s}
    m["x"][0, 0], m["y"][0, 0], m["z"][0, 0] = s["u00"], 0.0, 0.0
    pairs = ("xx", "xy", "xz", "yy", "yz", "zz")
    M = {n: np.zeros_like(T) for n in pairs}
    U = {c: np.zeros_like(T) for c in "xyz"}
    RT = np.zeros_like(T)
    ty = _dy(o, T, o.deryr)
    lapT = _dy(o, T, o.deryyr) - k2 * T
    pe = p.Re * float(np.float32(0.7))
    for j in range(my):
        P = lambda a: _phys(a[:, :, j], p.mgalx, p.mgalz)  # noqa: E731
        Tp = P(T)
        mp = {c: P(m[c]) for c in "xyz"}
        up = {c: mp[c] * Tp for c in "xyz"}
        for n in pairs:
            M[n][:, :, j] = _spec(mp[n[0]] * up[n[1]], nkx, mz)
        for c in "xyz":
            U[c][:, :, j] = _spec(up[c], nkx, mz)
        RT[:, :, j] = _spec(-(up["x"] * P(IX * T) + up["y"] * P(ty) + up["z"] * P(IZ * T)) + Tp * P(lapT) / pe,
                            nkx, mz)
    D = lambda a: _dy(o, a, o.deryr)  # noqa: E731
    D2 = lambda a: _dy(o, a, o.deryyr)  # noqa: E731
    Nx = -(IX * M["xx"] + D(M["xy"]) + IZ * M["xz"])
    Ny = -(IX * M["xy"] + D(M["yy"]) + IZ * M["yz"])
    Nz = -(IX * M["xz"] + D(M["yz"]) + IZ * M["zz"])
    wx = D(U["z"]) - IZ * U["y"]
    wy = IZ * U["x"] - IX * U["z"]
    wz = IX * U["y"] - D(U["x"])
    rhs_vor = IZ * Nx - IX * Nz + (D2(wy) - k2 * wy) / p.Re
    cc = IZ * wx - IX * wz
    rhs_phi = -k2 * Ny - D(IX * Nx + IZ * Nz) - (D2(cc) - k2 * cc) / p.Re
    inner = (slice(None), slice(None), slice(1, my - 1))
    for name, got, pred in (("vor", (new["vor"] - s["vor"]) / h, rhs_vor),
                            ("phi", (new["phi"] - s["phi"]) / h, rhs_phi),
                            ("scal", (new["scal"] - T) / h, RT)):
        assert np.abs(pred[inner]).max() > 1e-5, name
        assert np.abs(got[inner] - pred[inner]).max() < 1e-9 * np.abs(pred[inner]).max(), name
    u00 = (new["u00"] - s["u00"]) / h
    pred00 = -o.deryr(M["xy"][0, 0].real) + o.deryyr(U["x"][0, 0].real) / p.Re
    assert np.abs(u00[1:-1] - pred00[1:-1]).max() < 1e-9 * np.abs(pred00[1:-1]).max()
