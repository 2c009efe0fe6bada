"""Host-side mirror of the reference lomacte driver interface over the C ABI.

``Lomacte`` plays the role of the reference's ``cross1`` time loop
(Beovulfo/LoMa_phD trunk/lomacte3/src/cross.f:24-45, called from
trunk/lomacte3/src/main.f:215): it owns one case on one GPU and advances it
by full RK3 steps.  All compute runs in liblomacte_b200.so on the GPU; there
is no CPU fallback -- without the library or without a CUDA device the
constructor raises.

The spectral fields use the reference layout ``vor(0:my-1, 0:mz-1,
1:nplanes)``; as numpy arrays they are complex arrays of shape
``(nplanes, mz, my)``.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liblomacte_b200.so")

LMC_OK, LMC_EINVAL, LMC_ENOMEM, LMC_ENAN, LMC_ETIMEOUT, LMC_ECUDA, LMC_ENODEV = 0, -1, -2, -3, -4, -5, -6

# Exported symbols of include/lomacte_b200.h.
SYMBOLS = (
    "lmc_create", "lmc_destroy", "lmc_load_state_f64", "lmc_load_state_f32",
    "lmc_get_state_f64", "lmc_get_state_f32", "lmc_step", "lmc_sync",
    "lmc_get_diag", "lmc_status", "lmc_strerror", "lmc_stream",
    "lmc_state_device_ptrs", "lmc_make_ic", "lmc_op_y", "lmc_profile_start",
    "lmc_profile_read", "lmc_deryr2_noalloc", "lmc_wait_selftest", "lmc_step_split",
    "lmc_op_y_dense", "lmc_yop_tune", "lmc_y_metrics", "lmc_use_graphs", "lmc_query",
    "lmc_device_bytes", "lmc_footprint", "lmc_launches_per_step", "lmc_y_family",
    "lmc_stats_reset", "lmc_stats_step", "lmc_stats_read", "lmc_load_scalar_f64", "lmc_get_scalar_f64",
    "lmc_physical_f64",
)

# quantities of lmc_physical_f64, in order (the scalar adds "Z")
PHYSICAL_NAMES = ("u", "v", "w", "T", "omega_x", "omega_y", "omega_z")

KERNEL_NAMES = ("lapv", "assemble", "tder", "zinv", "xphys", "zfwd", "post1", "post2", "psi", "memset", "stats")


class LomacteError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        msg = _lib().lmc_strerror(code).decode() if _LIB is not None else str(code)
        super().__init__(f"{what}: {msg} ({code})" if what else f"{msg} ({code})")


class lmc_params(ctypes.Structure):
    _fields_ = [("mgalx", ctypes.c_int), ("mgalz", ctypes.c_int), ("my", ctypes.c_int),
                ("Re", ctypes.c_double), ("alp", ctypes.c_double), ("bet", ctypes.c_double),
                ("peclet", ctypes.c_double), ("cfl", ctypes.c_double), ("ncfl", ctypes.c_int),
                ("dt_mode", ctypes.c_int), ("dt", ctypes.c_double), ("precision", ctypes.c_int),
                ("device", ctypes.c_int), ("variant", ctypes.c_int), ("scalar", ctypes.c_int),
                ("schmidt", ctypes.c_double), ("visc", ctypes.c_int), ("sigma", ctypes.c_double)]


class lmc_diag(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "time", "Deltat", "dm", "dw", "Redw", "trapz", "masst", "massu", "massv", "massw",
        "H00u", "H00w", "Deltat_next")] + [("step", ctypes.c_int), ("status", ctypes.c_int)]


class lmc_ic_params(ctypes.Structure):
    _fields_ = [("s", ctypes.c_double), ("u0", ctypes.c_double), ("dm0", ctypes.c_double),
                ("amp", ctypes.c_double), ("swin", ctypes.c_double), ("nkmax", ctypes.c_int),
                ("nymax", ctypes.c_int), ("seed", ctypes.c_ulonglong)]


_LIB = None
_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)


def _lib():
    """Load liblomacte_b200.so (building it first when the sources are newer)."""
    global _LIB
    if _LIB is None:
        from . import build as _build
        try:
            _build.build()
        except Exception:
            if not os.path.exists(LIB_PATH):
                raise
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        L.lmc_create.argtypes = [ctypes.POINTER(lmc_params), _dp, ctypes.POINTER(vp)]
        L.lmc_destroy.argtypes = [vp]
        L.lmc_load_state_f64.argtypes = [vp] + [_dp] * 7 + [ctypes.c_double]
        L.lmc_load_state_f32.argtypes = [vp] + [_fp] * 4 + [_dp] * 3 + [ctypes.c_double]
        L.lmc_get_state_f64.argtypes = [vp] + [_dp] * 8
        L.lmc_get_state_f32.argtypes = [vp] + [_fp] * 4 + [_dp] * 4
        L.lmc_step.argtypes = [vp, ctypes.c_int]
        L.lmc_sync.argtypes = [vp]
        L.lmc_get_diag.argtypes = [vp, ctypes.POINTER(lmc_diag)]
        L.lmc_status.argtypes = [vp]
        L.lmc_strerror.restype = ctypes.c_char_p
        L.lmc_strerror.argtypes = [ctypes.c_int]
        L.lmc_stream.restype = vp
        L.lmc_stream.argtypes = [vp]
        L.lmc_state_device_ptrs.argtypes = [vp] + [ctypes.POINTER(_dp)] * 4
        L.lmc_make_ic.argtypes = [ctypes.POINTER(lmc_params), _dp, ctypes.POINTER(lmc_ic_params)] + [_dp] * 7
        L.lmc_op_y.argtypes = [vp, ctypes.c_int, vp, vp, vp]
        L.lmc_profile_start.argtypes = [vp]
        L.lmc_profile_read.argtypes = [vp, ctypes.c_int, _dp, ctypes.POINTER(ctypes.c_int)]
        L.lmc_deryr2_noalloc.argtypes = [ctypes.c_int, _dp, ctypes.c_int, vp, vp, vp]
        L.lmc_wait_selftest.argtypes = [vp, ctypes.c_uint]
        L.lmc_step_split.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.lmc_op_y_dense.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, vp]
        L.lmc_yop_tune.argtypes = [vp, ctypes.c_int, _dp]
        L.lmc_y_metrics.argtypes = [ctypes.c_int, _dp, _dp, _dp, _dp]
        L.lmc_use_graphs.argtypes = [vp, ctypes.c_int]
        L.lmc_launches_per_step.argtypes = [vp]
        L.lmc_y_family.argtypes = [vp]
        L.lmc_query.argtypes = [vp]
        L.lmc_device_bytes.argtypes = [vp]
        L.lmc_device_bytes.restype = ctypes.c_size_t
        L.lmc_stats_reset.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_double]
        L.lmc_stats_step.argtypes = [vp, ctypes.c_int]
        L.lmc_stats_read.argtypes = [vp, _dp, _dp, _dp, ctypes.POINTER(ctypes.c_int), ctypes.c_int]
        L.lmc_load_scalar_f64.argtypes = [vp, _dp]
        L.lmc_get_scalar_f64.argtypes = [vp, _dp]
        L.lmc_physical_f64.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), _dp]
        L.lmc_footprint.argtypes = [ctypes.POINTER(lmc_params)]
        L.lmc_footprint.restype = ctypes.c_size_t
        _LIB = L
    return _LIB


def lib():
    return _lib()


def _ptr(a: np.ndarray, t=_dp):
    return a.ctypes.data_as(t)


def _check(rc: int, what: str):
    if rc != LMC_OK:
        raise LomacteError(rc, what)


def stretched_mesh(my: int, ly: float = 24.0, a: float = 2.0) -> np.ndarray:
    """y = (ly/2) sinh(a eta)/sinh(a), eta uniform on [-1, 1]."""
    eta = np.linspace(-1.0, 1.0, my)
    return 0.5 * ly * np.sinh(a * eta) / np.sinh(a)


@dataclasses.dataclass
class Params:
    """hre.dat-equivalent run parameters (main.f:502-570)."""
    mgalx: int
    mgalz: int
    my: int
    Re: float = 160.0
    alp: float = 0.25
    bet: float = 0.25
    peclet: float = 0.0       # <= 0: Re*0.7f as the reference
    cfl: float = 0.5
    ncfl: int = 10
    dt_mode: int = 1          # 0 reference CFL, 1 fixed Deltat
    dt: float = 0.01
    precision: int = 0
    device: int = 0
    variant: int = 0          # 0 trunk/lomacte3 (2017), 1 trunk/lomacte (2014)
    scalar: int = 0           # 1: carry a passive scalar Z (lmc_load_scalar_f64)
    schmidt: float = 0.0      # Sc of Z; <= 0: Sc = Pr = 0.7f
    visc: int = 0             # 1: mu = k = rho D = T^sigma (0: constant viscosity)
    sigma: float = 0.0        # the exponent, in [0, 4]

    def c(self) -> lmc_params:
        return lmc_params(*[getattr(self, f.name) for f in dataclasses.fields(self)])

    @property
    def nplanes(self) -> int:
        return (2 * (self.mgalx // 3)) // 2

    @property
    def mz(self) -> int:
        return 2 * (self.mgalz // 3) - 1

    @property
    def shape(self):
        return (self.nplanes, self.mz, self.my)

    @staticmethod
    def from_modes(nx: int, nz: int, ny: int, **kw) -> "Params":
        """Grid from nominal Fourier-mode counts (nx = mx, nz = mz+1); nz = 1
        is a 2-D run (mz = 1, mgalz = 3)."""
        return Params(mgalx=3 * nx // 2, mgalz=3 if nz == 1 else 3 * nz // 2, my=ny, **kw)


@dataclasses.dataclass
class ICParams:
    s: float = 4.0
    u0: float = -0.5
    dm0: float = 1.0
    amp: float = 1e-2
    swin: float = 2.0
    nkmax: int = 8
    nymax: int = 4
    seed: int = 0

    def c(self) -> lmc_ic_params:
        return lmc_ic_params(self.s, self.u0, self.dm0, self.amp, self.swin, self.nkmax,
                             self.nymax, self.seed)


def make_ic(p: Params, y: np.ndarray, ic: ICParams):
    """Seeded initial condition (host only).  Returns a state dict."""
    y = np.ascontiguousarray(y, dtype=np.float64)
    shp = p.shape
    f = [np.zeros(shp, dtype=np.complex128) for _ in range(4)]
    r = [np.zeros(p.my) for _ in range(3)]
    pc, icc = p.c(), ic.c()
    rc = _lib().lmc_make_ic(ctypes.byref(pc), _ptr(y), ctypes.byref(icc),
                            *[_ptr(a.view(np.float64)) for a in f], *[_ptr(a) for a in r])
    _check(rc, "lmc_make_ic")
    return dict(vor=f[0], phi=f[1], psi=f[2], scal=f[3], u00=r[0], v00=r[1], w00=r[2], time=0.0)


def y_metrics(y: np.ndarray):
    """fmap = 1/(dy/deta), hy and trp of a mesh (host only; lmc_y_metrics)."""
    y = np.ascontiguousarray(y, dtype=np.float64)
    out = [np.zeros(len(y)) for _ in range(3)]
    _check(_lib().lmc_y_metrics(len(y), _ptr(y), *[_ptr(a) for a in out]), "lmc_y_metrics")
    return dict(fmap=out[0], hy=out[1], trp=out[2])


def footprint(p: "Params") -> int:
    """Device bytes a case with these parameters holds (lmc_footprint)."""
    pc = p.c()
    return int(_lib().lmc_footprint(ctypes.byref(pc)))


def deryr2_noalloc(y: np.ndarray, npencil: int, in_ptr: int, out_ptr: int, stream: int = 0) -> int:
    """d/dy of npencil device pencils without any device allocation (see
    lmc_deryr2_noalloc in include/lomacte_b200.h).  Returns the status."""
    y = np.ascontiguousarray(y, dtype=np.float64)
    return _lib().lmc_deryr2_noalloc(len(y), _ptr(y), int(npencil), ctypes.c_void_p(in_ptr),
                                     ctypes.c_void_p(out_ptr), ctypes.c_void_p(stream))


class Lomacte:
    """One lomacte case resident on one GPU (the cross1 time loop)."""

    def __init__(self, params: Params, y: np.ndarray):
        self.p = params
        self.y = np.ascontiguousarray(y, dtype=np.float64)
        if len(self.y) != params.my:
            raise ValueError("len(y) != my")
        self._h = ctypes.c_void_p()
        pc = params.c()
        _check(_lib().lmc_create(ctypes.byref(pc), _ptr(self.y), ctypes.byref(self._h)), "lmc_create")

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _lib().lmc_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def shape(self):
        return self.p.shape

    def load_state(self, st: dict):
        f = [np.ascontiguousarray(st[k], dtype=np.complex128).view(np.float64) for k in ("vor", "phi", "psi", "scal")]
        for a in f:
            if a.size != 2 * int(np.prod(self.shape)):
                raise ValueError("field size does not match the grid")
        r = [np.ascontiguousarray(st[k], dtype=np.float64) for k in ("u00", "v00", "w00")]
        _check(_lib().lmc_load_state_f64(self._h, *[_ptr(a) for a in f], *[_ptr(a) for a in r],
                                         float(st.get("time", 0.0))), "lmc_load_state_f64")

    def load_state_f32(self, fields: dict, u00, v00, w00, time: float = 0.0):
        """Load complex*8 fields (the reference's storage type, e.g. from
        files.read_restart) through lmc_load_state_f32."""
        f = [np.ascontiguousarray(fields[k], dtype=np.complex64).view(np.float32) for k in ("vor", "phi", "psi", "scal")]
        for a in f:
            if a.size != 2 * int(np.prod(self.shape)):
                raise ValueError("field size does not match the grid")
        r = [np.ascontiguousarray(v, dtype=np.float64) for v in (u00, v00, w00)]
        _check(_lib().lmc_load_state_f32(self._h, *[_ptr(a, _fp) for a in f], *[_ptr(a) for a in r], float(time)),
               "lmc_load_state_f32")

    def use_graphs(self, on: bool):
        _check(_lib().lmc_use_graphs(self._h, int(bool(on))), "lmc_use_graphs")

    def done(self) -> bool:
        """True when the enqueued steps have finished (never blocks)."""
        rc = _lib().lmc_query(self._h)
        if rc < 0:
            raise LomacteError(rc, "lmc_query")
        return rc == 1

    @property
    def launches_per_step(self) -> int:
        return int(_lib().lmc_launches_per_step(self._h))

    @property
    def y_family(self) -> str:
        """'mode' (one thread per mode) or 'warp' (one warp per mode)."""
        return "mode" if _lib().lmc_y_family(self._h) == 1 else "warp"

    @property
    def device_bytes(self) -> int:
        return int(_lib().lmc_device_bytes(self._h))

    def get_state(self) -> dict:
        f = [np.zeros(self.shape, dtype=np.complex128) for _ in range(4)]
        r = [np.zeros(self.p.my) for _ in range(3)]
        t = np.zeros(1)
        _check(_lib().lmc_get_state_f64(self._h, *[_ptr(a.view(np.float64)) for a in f],
                                        *[_ptr(a) for a in r], _ptr(t)), "lmc_get_state_f64")
        return dict(vor=f[0], phi=f[1], psi=f[2], scal=f[3], u00=r[0], v00=r[1], w00=r[2], time=float(t[0]))

    def step(self, n: int = 1):
        _check(_lib().lmc_step(self._h, int(n)), "lmc_step")

    # passive scalar Z (Params.scalar = 1): reference layout, complex
    def step_split(self, nblocks: int, n: int = 1):
        """n RK3 steps with the transform stage split into nblocks slab
        blocks exchanged by device copies (lmc_step_split)."""
        _check(_lib().lmc_step_split(self._h, int(nblocks), int(n)), "lmc_step_split")

    def load_scalar(self, z):
        a = np.ascontiguousarray(np.asarray(z, dtype=np.complex128).reshape(self.shape))
        _check(_lib().lmc_load_scalar_f64(self._h, _ptr(a.view(np.float64))), "lmc_load_scalar_f64")

    def get_scalar(self) -> np.ndarray:
        a = np.zeros(self.shape, dtype=np.complex128)
        _check(_lib().lmc_get_scalar_f64(self._h, _ptr(a.view(np.float64))), "lmc_get_scalar_f64")
        return a

    def physical(self, planes) -> dict:
        """Physical fields on the 1-based y rows planes (lmc_physical_f64):
        a dict of [nplanes, mgalz, mgalx] arrays u, v, w, T, omega_x,
        omega_y, omega_z (and Z with the scalar), x fastest."""
        pl = np.ascontiguousarray(planes, dtype=np.int32)
        names = PHYSICAL_NAMES + (("Z",) if self.p.scalar else ())
        out = np.zeros((len(pl), len(names), self.p.mgalz, self.p.mgalx))
        _check(_lib().lmc_physical_f64(self._h, len(pl), pl.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                       _ptr(out.ravel())), "lmc_physical_f64")
        return {k: out[:, q] for q, k in enumerate(names)}

    def sync(self):
        _check(_lib().lmc_sync(self._h), "lmc_sync")

    # statistics: addstats1/2 and the phys2 sums on the device
    # (cross.f:578-585, 794-812, 1583-1607), resetstats (escru.f:485-580)
    def stats_reset(self, planes=None, sigma: float = 0.0):
        """Zero the accumulators; planes are 1-based y rows of the spectra
        (default: the centre row (my+1)/2, the reference's jsptot(nspec+1))."""
        planes = [(self.p.my + 1) // 2] if planes is None else [int(j) for j in planes]
        arr = (ctypes.c_int * max(1, len(planes)))(*planes)
        _check(_lib().lmc_stats_reset(self._h, len(planes), arr, float(sigma)), "lmc_stats_reset")
        self._stats_planes = planes
        self._stats_sigma = float(sigma)

    def stats_step(self, n: int = 1):
        """n RK3 steps that accumulate statistics (istati = 1)."""
        _check(_lib().lmc_stats_step(self._h, int(n)), "lmc_stats_step")

    def stats_read(self, clear_spectra: bool = False):
        """Read the accumulators back as a StatsData; clear_spectra zeroes the
        spectra and nacumsp afterwards, as writestats does."""
        from .stats import NSTAT, StatsData
        planes = getattr(self, "_stats_planes", None)
        if planes is None:
            raise LomacteError(LMC_EINVAL, "stats_read before stats_reset")
        nkx, mz, my = self.shape
        prof = np.zeros((NSTAT, my))
        spec = np.zeros((nkx, 12, len(planes), (mz - 1) // 2 + 1))
        uner = np.zeros(9)
        cnt = (ctypes.c_int * 2)()
        _check(_lib().lmc_stats_read(self._h, _ptr(prof), _ptr(spec), _ptr(uner), cnt, int(bool(clear_spectra))),
               "lmc_stats_read")
        return StatsData(prof=prof, spec=spec, uner=uner, nacum=int(cnt[0]), nacumsp=int(cnt[1]),
                         planes=list(planes), sigma=self._stats_sigma)

    def wait_selftest(self, polls: int = 1000):
        """One bounded device wait that nothing completes (lmc_wait_selftest);
        lmc_status reads LMC_ETIMEOUT afterwards."""
        _check(_lib().lmc_wait_selftest(self._h, int(polls)), "lmc_wait_selftest")

    def status(self) -> int:
        """The device status word (lmc_status): 0 or an LMC_E* code."""
        return int(_lib().lmc_status(self._h))

    def diag(self) -> dict:
        d = lmc_diag()
        _check(_lib().lmc_get_diag(self._h, ctypes.byref(d)), "lmc_get_diag")
        return {n: getattr(d, n) for n, _ in lmc_diag._fields_}

    def op_y(self, op: int, inp, out, out2=None):
        """Single y-operator on device buffers (torch CUDA tensors or raw
        device pointers) holding all modes in the reference layout."""
        def p(x):
            if x is None:
                return None
            return ctypes.c_void_p(x.data_ptr() if hasattr(x, "data_ptr") else int(x))
        _check(_lib().lmc_op_y(self._h, op, p(inp), p(out), p(out2)), "lmc_op_y")

    def op_y_dense(self, op: int, method: int, inp, out):
        """The y operator op (1 d/dy, 2 d2/dy2) as a dense GEMM (method 1
        FP64, 2 3xTF32) on device buffers in the reference layout."""
        p = lambda x: ctypes.c_void_p(x.data_ptr() if hasattr(x, "data_ptr") else int(x))
        _check(_lib().lmc_op_y_dense(self._h, int(op), int(method), p(inp), p(out)), "lmc_op_y_dense")

    def yop_tune(self, op: int = 1) -> dict:
        """Banded solve against the dense GEMMs for the y operator op on the
        current state (lmc_yop_tune): times in ms, errors, the choice."""
        out = np.zeros(6)
        _check(_lib().lmc_yop_tune(self._h, int(op), _ptr(out)), "lmc_yop_tune")
        names = ("banded", "dense_fp64", "dense_3xtf32")
        return {"op": op, "ms": dict(zip(names, out[:3].tolist())),
                "rel_err_vs_banded": {"dense_fp64": float(out[3]), "dense_3xtf32": float(out[4])},
                "choice": names[int(out[5])]}

    def profile_start(self):
        _check(_lib().lmc_profile_start(self._h), "lmc_profile_start")

    def profile_read(self) -> dict:
        n = len(KERNEL_NAMES)
        ms = np.zeros(n)
        cnt = (ctypes.c_int * n)()
        _check(_lib().lmc_profile_read(self._h, n, _ptr(ms), cnt), "lmc_profile_read")
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(KERNEL_NAMES)}

    def load_state_ptrs(self, vor, phi, psi, scal, u00, v00, w00, time=0.0):
        """Load from raw host pointers (e.g. pinned torch tensors)."""
        P = lambda x: ctypes.cast(ctypes.c_void_p(x), _dp)
        _check(_lib().lmc_load_state_f64(self._h, P(vor), P(phi), P(psi), P(scal), P(u00), P(v00), P(w00),
                                         float(time)), "lmc_load_state_f64")

    def get_state_ptrs(self, vor, phi, psi, scal, u00, v00, w00):
        P = lambda x: ctypes.cast(ctypes.c_void_p(x), _dp)
        t = np.zeros(1)
        _check(_lib().lmc_get_state_f64(self._h, P(vor), P(phi), P(psi), P(scal), P(u00), P(v00), P(w00),
                                        _ptr(t)), "lmc_get_state_f64")
        return float(t[0])

    def load_scalar_ptr(self, z):
        """Load Z from a raw host pointer (reference layout, complex*16)."""
        _check(_lib().lmc_load_scalar_f64(self._h, ctypes.cast(ctypes.c_void_p(z), _dp)), "lmc_load_scalar_f64")

    def get_scalar_ptr(self, z):
        _check(_lib().lmc_get_scalar_f64(self._h, ctypes.cast(ctypes.c_void_p(z), _dp)), "lmc_get_scalar_f64")

    @property
    def stream(self) -> int:
        return int(_lib().lmc_stream(self._h) or 0)
