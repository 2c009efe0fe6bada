"""Physical-field export on the CPU: the oracle's restatement
(lmo_physical) of the quantities tofis_loma writes (escrphys,
trunk/tofis_loma/src/escru.f:11-314), from the solver's own rho u_i.

Checks: T on a plane equals numpy's inverse 2-D transform of the spectral T
as stored, so the natural z/x order and the normalisation are pinned
independently; for a state whose rho u_i is known in closed form (Omega_y
only), u, w and the vorticity equal numpy's pointwise products of the
inverse-transformed fields; plane means of T and of rho u =
u / T equal the 00 profiles; the mean of omega_y vanishes; the export
leaves the state alone.
"""
import numpy as np

from tests.helpers import case, oracle_for


def _to_physical(c, mgalx, mgalz):
    """numpy: half spectrum c[kx >= 0][kz signed] -> real field [z][x]
    with samples e^{+i(kx x + kz z)}."""
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


def test_temperature_plane_matches_numpy_transform():
    p, y, st = case(24, 24, 33)
    o = oracle_for(p, y, st, nthreads=4)
    o.step(2)
    s = o.get_state()
    planes = [2, 17, 30]
    out = o.physical(planes)
    assert out.shape == (3, 7, p.mgalz, p.mgalx)
    for n, j in enumerate(planes):
        ref = _to_physical(s["scal"][:, :, j - 1], p.mgalx, p.mgalz)
        assert np.abs(out[n, 3] - ref).max() < 1e-13 * np.abs(ref).max()


def test_plane_means_and_state_untouched():
    p, y, st = case(24, 24, 33)
    o = oracle_for(p, y, st, nthreads=4)
    o.step(2)
    before = o.get_state()
    planes = list(range(1, p.my + 1))
    out = o.physical(planes)
    after = o.get_state()
    for k in ("vor", "phi", "psi", "scal", "u00", "v00", "w00"):
        assert np.array_equal(before[k], after[k]), k
    rows = np.array(planes) - 1
    T = out[:, 3]
    assert np.allclose(T.mean(axis=(1, 2)), before["scal"][0, 0, rows].real, rtol=0, atol=1e-13)
    for q, k in ((0, "u00"), (1, "v00"), (2, "w00")):
        m = (out[:, q] / T).mean(axis=(1, 2))
        assert np.abs(m - before[k][rows]).max() < 1e-12 * max(1.0, np.abs(before[k]).max()), k
    assert np.abs(out[:, 5].mean(axis=(1, 2))).max() < 1e-14


def test_velocity_and_vorticity_against_numpy():
    """Omega_y in two modes (rho u = -i kz Omega/k^2, rho w = i kx
    Omega/k^2, rho v = 0), u00 a shear profile, a 3-D temperature: u, w
    and omega against numpy's pointwise products of the inverse-transformed
    fields (u = T rho u, omega = T curl(rho u) + grad T x rho u)."""
    p, y, st = case(24, 24, 33)
    nkx, mz, my = st["vor"].shape
    kxv = p.alp * np.arange(nkx)
    kzv = p.bet * np.array([k if k <= (mz - 1) // 2 else k - mz for k in range(mz)])
    env = np.exp(-y ** 2 / 8) * (1 - (y / y[-1]) ** 2)
    rng = np.random.default_rng(6)
    s = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in st.items()}
    s["phi"][:] = 0
    s["psi"][:] = 0
    s["vor"][:] = 0
    for (i, k) in ((1, 2), (2, mz - 1)):
        s["vor"][i, k, :] = 0.05 * (rng.standard_normal() + 1j * rng.standard_normal()) * env
    s["u00"], s["v00"], s["w00"] = 0.5 * np.tanh(y / 2), np.zeros(my), np.zeros(my)
    T = np.zeros_like(s["scal"])
    T[0, 0, :] = st["scal"][0, 0, :]
    for (i, k) in ((1, 0), (0, 2), (2, 1)):
        T[i, k, :] = 0.01 * (rng.standard_normal() + 1j * rng.standard_normal()) * env
    s["scal"] = T
    o = oracle_for(p, y, s, nthreads=2)
    planes = [5, 17, 29]
    out = o.physical(planes)

    def dy(a):
        r = np.zeros_like(a)
        for i in range(nkx):
            for k in range(mz):
                r[i, k] = o.deryr(a[i, k].real) + 1j * o.deryr(a[i, k].imag)
        return r

    vo = s["vor"].copy()
    vo[:, :, 0], vo[:, :, -1] = vo[:, :, 1], vo[:, :, -2]  # the wall condition of Omega_y (cross.f:315-327)
    k2 = kxv[:, None, None] ** 2 + kzv[None, :, None] ** 2
    k2[0, 0] = 1.0
    IX, IZ = 1j * kxv[:, None, None], 1j * kzv[None, :, None]
    ru, rw = -IZ * vo / k2, IX * vo / k2
    ru[0, 0], rw[0, 0] = s["u00"], 0.0
    cx, cz = dy(rw), -dy(ru)            # curl(rho u) with rho v = 0
    cy = IZ * ru - IX * rw
    tx, ty, tz = IX * T, dy(T), IZ * T
    for n, j in enumerate(planes):
        P = lambda a: _to_physical(a[:, :, j - 1], p.mgalx, p.mgalz)  # noqa: E731
        Tp, u, w = P(T), P(ru), P(rw)
        want = {0: u * Tp, 2: w * Tp, 4: Tp * P(cx) + P(ty) * w, 5: Tp * P(cy) + P(tz) * u - P(tx) * w,
                6: Tp * P(cz) - P(ty) * u}
        for q, ref in want.items():
            assert np.abs(out[n, q] - ref).max() < 1e-12 * max(np.abs(ref).max(), 1e-300), (j, q)
        assert np.abs(out[n, 1]).max() < 1e-14  # rho v = 0
