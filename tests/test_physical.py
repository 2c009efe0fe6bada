"""Physical-field export on the CPU: the oracle's restatement
(lmo_physical) of the quantities tofis_loma writes (escrphys,
trunk/tofis_loma/src/escru.f:11-314), from the solver's own rho u_i.

Checks: T on a plane equals numpy's inverse 2-D transform of the spectral T
as stored, so the natural z/x order and the normalisation are pinned
independently; plane means of T and of rho u =
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
