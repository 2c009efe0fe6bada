"""ctypes front-end of the FP64 CPU oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline and
reference legs use this module, as the checker or as the timed CPU
baseline.  The product package ``loma_phd_b200`` never imports it.

The oracle restates the reference lomacte3 substep in FP64
(Beovulfo/LoMa_phD trunk/lomacte3/src/cross.f:307-1141 and the routines it
calls); see lomacte_oracle.h for the file-by-file list.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liblomacte_oracle.so")
_lib = None

NDIAG = 13
DIAG_NAMES = ("time", "Deltat", "dm", "dw", "Redw", "trapz", "masst",
              "massu", "massv", "massw", "H00u", "H00w", "Deltat_next")

_dp = ctypes.POINTER(ctypes.c_double)


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc, OpenMP)."""
    src = [os.path.join(_HERE, f) for f in ("lomacte_oracle.c", "lomacte_oracle.h")]
    stale = not os.path.exists(_LIB_PATH) or any(
        os.path.getmtime(f) > os.path.getmtime(_LIB_PATH) for f in src)
    if force or stale:
        subprocess.run(["make", "-C", _HERE], check=True,
                       stdout=subprocess.DEVNULL)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        L.lmo_create.restype = ctypes.c_void_p
        L.lmo_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp,
                                 ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                 ctypes.c_int, ctypes.c_double, ctypes.c_int]
        L.lmo_destroy.argtypes = [ctypes.c_void_p]
        L.lmo_set_state.argtypes = [ctypes.c_void_p] + [_dp] * 7 + [ctypes.c_double]
        L.lmo_get_state.argtypes = [ctypes.c_void_p] + [_dp] * 8
        L.lmo_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.lmo_set_variant.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.lmo_substep.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.lmo_set_sample.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.lmo_get_diag.argtypes = [ctypes.c_void_p, _dp]
        L.lmo_get_coefs.argtypes = [ctypes.c_void_p] + [_dp] * 7
        for n in ("lmo_deryr", "lmo_deryyr", "lmo_inty8"):
            getattr(L, n).argtypes = [ctypes.c_void_p, _dp, _dp]
        for n in ("lmo_lapvdvhom", "lmo_solvepsi"):
            getattr(L, n).argtypes = [ctypes.c_void_p, _dp, _dp, _dp, ctypes.c_double]
        L.lmo_stats_reset.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                      ctypes.c_double]
        L.lmo_stats_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.lmo_stats_read.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, ctypes.POINTER(ctypes.c_int), ctypes.c_int]
        L.lmo_set_scalar.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]
        L.lmo_set_scalar_state.argtypes = [ctypes.c_void_p, _dp]
        L.lmo_get_scalar_state.argtypes = [ctypes.c_void_p, _dp]
        L.lmo_set_viscosity.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]
        L.lmo_physical.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int), _dp]
        L.lmo_cft.argtypes = [ctypes.c_int, _dp, ctypes.c_int]
        L.lmo_rft.argtypes = [ctypes.c_int, _dp, ctypes.c_int]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


class Oracle:
    """FP64 CPU restatement of one lomacte run (cross1's time loop)."""

    def __init__(self, mgalx, mgalz, y, Re, alp, bet, peclet=None, cfl=0.5,
                 ncfl=10, dtmode=1, dt0=0.01, nthreads=None, variant=0):
        self.y = np.ascontiguousarray(y, dtype=np.float64)
        self.my = len(self.y)
        self.mgalx, self.mgalz = mgalx, mgalz
        self.mx = 2 * (mgalx // 3)
        self.nkx = self.mx // 2
        self.mz = 2 * (mgalz // 3) - 1
        if peclet is None:
            # main.f:569 -- Re*0.7 with 0.7 a single-precision literal
            peclet = Re * float(np.float32(0.7))
        if nthreads is None:
            nthreads = os.cpu_count() or 1
        self.nthreads = nthreads
        self._scalar = False
        self.h = lib().lmo_create(mgalx, mgalz, self.my, _p(self.y), Re, alp, bet,
                                  peclet, cfl, ncfl, dtmode, dt0, nthreads)
        if not self.h:
            raise ValueError("oracle: bad grid")
        if variant:
            lib().lmo_set_variant(self.h, int(variant))

    def __del__(self):
        if getattr(self, "h", None):
            lib().lmo_destroy(self.h)
            self.h = None

    @property
    def shape(self):
        return (self.nkx, self.mz, self.my)

    def set_state(self, vor, phi, psi, scal, u00, v00, w00, time=0.0):
        c = [np.ascontiguousarray(a, dtype=np.complex128).view(np.float64)
             for a in (vor, phi, psi, scal)]
        r = [np.ascontiguousarray(a, dtype=np.float64) for a in (u00, v00, w00)]
        for a in c:
            assert a.size == 2 * self.nkx * self.mz * self.my
        lib().lmo_set_state(self.h, *[_p(a) for a in c], *[_p(a) for a in r], time)

    def get_state(self):
        n = self.nkx * self.mz * self.my
        c = [np.zeros(2 * n) for _ in range(4)]
        r = [np.zeros(self.my) for _ in range(3)]
        t = np.zeros(1)
        lib().lmo_get_state(self.h, *[_p(a) for a in c], *[_p(a) for a in r], _p(t))
        out = {k: a.view(np.complex128).reshape(self.shape)
               for k, a in zip(("vor", "phi", "psi", "scal"), c)}
        out.update(u00=r[0], v00=r[1], w00=r[2], time=float(t[0]))
        return out

    def step(self, n=1):
        lib().lmo_step(self.h, n)

    def substep(self, r=0):
        lib().lmo_substep(self.h, r)

    def set_sample(self, stride, phase=0):
        """Later substeps do 1/stride of their work (timing samples only)."""
        if lib().lmo_set_sample(self.h, int(stride), int(phase)) != 0:
            raise ValueError("lmo_set_sample rejected its arguments")

    # passive scalar Z, advanced as T (lomacte_oracle.h)
    def set_scalar(self, z, schmidt):
        if lib().lmo_set_scalar(self.h, 1, float(schmidt)) != 0:
            raise ValueError("lmo_set_scalar rejected its arguments")
        self._scalar = True
        a = np.ascontiguousarray(np.asarray(z, dtype=np.complex128).reshape(self.shape)).view(np.float64)
        lib().lmo_set_scalar_state(self.h, _p(a.ravel()))

    def get_scalar(self):
        a = np.zeros(self.shape, dtype=np.complex128)
        lib().lmo_get_scalar_state(self.h, _p(a.view(np.float64).ravel()))
        return a

    # variable viscosity mu = k = rho D = T^sigma (lomacte_oracle.h)
    def set_viscosity(self, sigma):
        """sigma = None: constant viscosity (the lomacte3 substep)."""
        on = sigma is not None
        if lib().lmo_set_viscosity(self.h, int(on), float(sigma or 0.0)) != 0:
            raise ValueError("lmo_set_viscosity rejected its arguments")

    # physical fields on y planes (lomacte_oracle.h: lmo_physical)
    def physical(self, planes):
        """[nplanes, nq, mgalz, mgalx]: u, v, w, T, omega_x, omega_y,
        omega_z (and Z with the scalar) on the 1-based rows planes."""
        pl = np.ascontiguousarray(planes, dtype=np.int32)
        nq = 8 if self._scalar else 7
        out = np.zeros((len(pl), nq, self.mgalz, self.mgalx))
        rc = lib().lmo_physical(self.h, len(pl), pl.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _p(out.ravel()))
        if rc != 0:
            raise ValueError("lmo_physical rejected its arguments")
        return out

    # statistics: addstats1/2 and the phys2 sums (cross.f:578-585, 794-812,
    # 1583-1607), resetstats (escru.f:485-580)
    def stats_reset(self, planes, sigma=0.0):
        jsp = (ctypes.c_int * max(1, len(planes)))(*[int(j) for j in planes])
        if lib().lmo_stats_reset(self.h, len(planes), jsp, float(sigma)) != 0:
            raise ValueError("lmo_stats_reset rejected its arguments")
        self._nsp = len(planes)

    def stats_step(self, n=1):
        if lib().lmo_stats_step(self.h, n) != 0:
            raise RuntimeError("lmo_stats_step: no statistics set up")

    def stats_read(self, clear_spectra=False):
        """(profiles [33, my], spectra [nkx, 12, nsp, nz1+1], uner [9],
        nacum, nacumsp) -- the raw accumulators, .sta order."""
        nkx, mz, _ = self.shape
        nz1 = (mz - 1) // 2
        prof = np.zeros((33, self.my))
        spec = np.zeros((nkx, 12, self._nsp, nz1 + 1))
        uner = np.zeros(9)
        cnt = (ctypes.c_int * 2)()
        if lib().lmo_stats_read(self.h, _p(prof), _p(spec), _p(uner), cnt, int(bool(clear_spectra))) != 0:
            raise RuntimeError("lmo_stats_read: no statistics set up")
        return prof, spec, uner, cnt[0], cnt[1]

    def diag(self):
        d = np.zeros(NDIAG)
        lib().lmo_get_diag(self.h, _p(d))
        return dict(zip(DIAG_NAMES, d.tolist()))

    def coefs(self):
        my = self.my
        a = [np.zeros(7 * my) for _ in range(3)] + [np.zeros(5 * my) for _ in range(3)] + [np.zeros(my)]
        lib().lmo_get_coefs(self.h, *[_p(x) for x in a])
        names = ("prem1_lu", "dt11", "dt12", "prem3_lu", "dt21", "dt22", "fmap")
        out = {}
        for n_, x in zip(names, a):
            out[n_] = x if n_ == "fmap" else x.reshape(my, -1)
        return out

    def deryr(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        du = np.zeros_like(u)
        lib().lmo_deryr(self.h, _p(u), _p(du))
        return du

    def deryyr(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        du = np.zeros_like(u)
        lib().lmo_deryyr(self.h, _p(u), _p(du))
        return du

    def inty8(self, du):
        du = np.ascontiguousarray(du, dtype=np.float64)
        u = np.zeros_like(du)
        lib().lmo_inty8(self.h, _p(du), _p(u))
        return u

    def _pois(self, fn, phi, rk):
        phi = np.ascontiguousarray(phi, dtype=np.complex128)
        v = np.zeros_like(phi)
        dv = np.zeros_like(phi)
        fn(self.h, _p(phi.view(np.float64)), _p(v.view(np.float64)),
           _p(dv.view(np.float64)), rk)
        return v, dv

    def lapvdvhom(self, phi, rk):
        return self._pois(lib().lmo_lapvdvhom, phi, rk)

    def solvepsi(self, phi, rk):
        return self._pois(lib().lmo_solvepsi, phi, rk)


def cft(c: np.ndarray, iopt: int) -> np.ndarray:
    """cftsingle.f cft on one complex vector (forward scaled by 1/n)."""
    x = np.ascontiguousarray(c, dtype=np.complex128).copy()
    lib().lmo_cft(len(x), _p(x.view(np.float64)), iopt)
    return x


def rft(c: np.ndarray, iopt: int, n: int) -> np.ndarray:
    """rftsingle.f rft on one line: forward takes n reals and returns the
    packed n+2 reals; inverse takes n+2 packed reals and returns n reals."""
    buf = np.zeros(n + 2)
    buf[: len(c)] = c
    lib().lmo_rft(n, _p(buf), iopt)
    return buf[:n] if iopt >= 0 else buf
