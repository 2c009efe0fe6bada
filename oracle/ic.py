"""Seeded initial condition on the oracle side (test infrastructure only).

A restatement, with the oracle's own y operators (pred1m6o / prederiv2 /
Lapvdvhom of lomacte_oracle.c), of the library's seeded initial condition:
the structure of the reference generator trunk/initloma3/src/main.f:95-609
(random velocity modes with nymax y-harmonics, curl for a solenoidal field,
rms scaling at the mid plane, mean profiles, then psi, Omega_y and phi)
with a counter-based random number per (seed, kx, kz, component, draw)
instead of initloma3's wall-clock seed.  It lets the CPU arms of bench.py
build their state without loading the product library, and tests pin it to
the library's generator.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline and
reference legs use this module.
"""
from __future__ import annotations

import numpy as np

from oracle.oracle import Oracle

_M64 = (1 << 64) - 1


def _splitmix64(x: int) -> int:
    x = (x + 0x9E3779B97F4A7C15) & _M64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & _M64
    return x ^ (x >> 31)


def urand(seed: int, a: int, b: int, c: int, d: int) -> float:
    """Uniform in [0, 1) from a hash chain of the counters (order- and
    thread-independent)."""
    h = _splitmix64(seed & _M64)
    h = _splitmix64(h ^ ((a * 0x100000001B3) & _M64))
    h = _splitmix64(h ^ ((b * 0xC2B2AE3D27D4EB4F) & _M64))
    h = _splitmix64(h ^ ((c * 0x165667B19E3779F9) & _M64))
    h = _splitmix64(h ^ ((d * 0x27D4EB2F165667C5) & _M64))
    return (h >> 11) * (1.0 / 9007199254740992.0)


def make_ic(mgalx, mgalz, y, alp=0.25, bet=0.25, s=4.0, u0=-0.5, dm0=1.0, amp=1e-2, swin=2.0,
            nkmax=8, nymax=4, seed=0, momentum=False):
    """State dict (vor, phi, psi, scal [nkx, mz, my] complex, u00, v00, w00)
    of the seeded mixing layer: rho00 = 1 + (s-1)/(s+1) tanh(-y/(2 dm0)),
    T00 = 1/rho00, rho u00 = rho00 u0 tanh(y/(2 dm0)); solenoidal noise on
    1 <= |k| <= nkmax (mode-index units) windowed by exp(-(y/swin)^2),
    scaled to rms amp at the mid plane.  momentum: also return the spectral
    rho u, rho v, rho w the state was built from (keys ru, rv, rw)."""
    y = np.ascontiguousarray(y, dtype=np.float64)
    my = len(y)
    nkx = (2 * (mgalx // 3)) // 2
    mz = 2 * (mgalz // 3) - 1
    nz1 = (mz - 1) // 2
    kzi = np.array([k if k <= nz1 else k - mz for k in range(mz)])
    kxv = alp * np.arange(nkx)
    kzv = bet * kzi
    o = Oracle(6, 3, y, 160.0, alp, bet, nthreads=1)  # the y operators depend on y alone

    def d1(u):
        return o.deryr(u.real) + 1j * o.deryr(u.imag)

    def d2(u):
        return o.deryyr(u.real) + 1j * o.deryyr(u.imag)

    win = np.exp(-(y / swin) ** 2)
    band = []
    for m in range(nkx * mz):
        i, kz = m // mz, kzi[m % mz]
        nh = np.sqrt(float(i * i + kz * kz))
        if 1.0 <= nh <= nkmax:
            band.append(m)
    slot = {m: b for b, m in enumerate(band)}
    nym = nymax if nymax > 0 else 1
    # 1) random velocity per mode (initloma3/src/main.f:128-226)
    vel = np.zeros((len(band), 3, my), dtype=np.complex128)
    for b, m in enumerate(band):
        i, k = m // mz, m % mz
        kz = int(kzi[k])
        if i == 0 and kz < 0:
            continue
        kh = np.sqrt(kxv[i] ** 2 + kzv[k] ** 2)
        for c in range(3):
            for jj in range(1, nym + 1):
                a = 2.0 * (0.5 - urand(seed, i, kz + 100000, c, 2 * jj))
                ph = urand(seed, i, kz + 100000, c, 2 * jj + 1)
                ky = 2.0 * kh / nym * jj
                vel[b, c] += a * np.exp(1j * (ky * y + 2.0 * np.pi * ph)) * win
    for b, m in enumerate(band):  # kx = 0, kz < 0: the conjugate of the kz > 0 partner
        if m // mz == 0 and kzi[m % mz] < 0:
            vel[b] = np.conj(vel[slot[-int(kzi[m % mz])]])
    # 2) solenoidal: curl (initloma3/src/main.f:231-256)
    cur = np.zeros_like(vel)
    for b, m in enumerate(band):
        i, k = m // mz, m % mz
        ikx, ikz = 1j * kxv[i], 1j * kzv[k]
        uf, vf, wf = vel[b]
        cur[b, 0] = d1(wf) - ikz * vf
        cur[b, 1] = ikz * uf - ikx * wf
        cur[b, 2] = ikx * vf - d1(uf)
    # 3) rms amp at the mid plane (initloma3/src/main.f:291-356)
    jm = int(np.argmin(np.abs(y)))
    e = 0.0
    for b, m in enumerate(band):
        e += (1.0 if m // mz == 0 else 2.0) * abs(cur[b, 0, jm]) ** 2
    fac = amp / np.sqrt(e) if e > 0 else 0.0
    # 4) mean profiles (initloma3/src/main.f:362-374, 572-600)
    rho00 = 1.0 + (s - 1.0) / (s + 1.0) * np.tanh(-y / (2.0 * dm0))
    # 5) psi, Omega_y, phi (initloma3/src/main.f:473-561); zero outside the band
    shp = (nkx, mz, my)
    vor, phi, psi, scal = (np.zeros(shp, dtype=np.complex128) for _ in range(4))
    mom = [np.zeros(shp, dtype=np.complex128) for _ in range(3)] if momentum else None
    for b, m in enumerate(band):
        i, k = m // mz, m % mz
        ikx, ikz = 1j * kxv[i], 1j * kzv[k]
        k2 = kxv[i] ** 2 + kzv[k] ** 2
        ru, rv, rw = (rho00 * fac * cur[b, c] for c in range(3))
        if momentum:
            mom[0][i, k], mom[1][i, k], mom[2][i, k] = ru, rv, rw
        div = ikx * ru + ikz * rw + d1(rv)
        ps = o.lapvdvhom(div, k2)[0] if k2 != 0.0 else np.zeros(my, dtype=np.complex128)
        myv = rv - d1(ps)
        psi[i, k] = ps
        vor[i, k] = -ikx * rw + ikz * ru
        phi[i, k] = -k2 * myv + d2(myv)
    scal[0, 0] = 1.0 / rho00
    u00 = rho00 * u0 * np.tanh(y / (2.0 * dm0))
    out = dict(vor=vor, phi=phi, psi=psi, scal=scal, u00=u00, v00=np.zeros(my), w00=np.zeros(my), time=0.0)
    if momentum:
        out.update(ru=mom[0], rv=mom[1], rw=mom[2])
    return out
