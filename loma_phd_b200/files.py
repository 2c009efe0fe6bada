"""The reference's file formats, read and written by the host side.

* Restart / image files (Fortran unformatted sequential, little endian,
  4-byte record markers), written by escru (trunk/lomacte3/src/escru.f:
  121-139) and read by getfil (trunk/lomacte3/src/main.f:361-406):
    record 1: time, Re, alp, bet, a0 (real*4), mx, my, mz (integer*4),
              (y_j, fmap_j) real*8 pairs for j = 1..my,
              (u00_j, v00_j, w00_j) real*4 triples for j = 1..my
    then one record per kx plane i = 0..mx/2-1:
              ((vor, phi, psi, scal)(j, k), j = 0..2my-1, k = 0..mz-1) real*4,
              the four fields interleaved per real scalar, j running over
              the (re, im) pairs of the y pencil.
  Reading into a grid with another mz keeps the kz = 0..klen-1 and the last
  klen-1 (negative) modes, as assign does (main.f:841-882).
* hre.dat (main.f:502-545): lines that start with "CC" are comments; then
  Re alp bet a0 / nstep nimag nhist / CFL ncfl / id22 nstart ntimes /
  output, input and statistics file names.
* Statistics (.sta) and spectra (.spe) files of writestats (escru.f:276-484),
  Fortran unformatted sequential like the images:
    .sta record 1: my (i4), time, Re, alp, bet, a0 (real*4), nacum (i4)
         record 2: (y_j, fmap_j) real*8 pairs, j = 1..my
         record 3: 33 real*8 per row j = 1..my: um vm wm rum rvm rwm Tm w1m
                   w2m w3m them up vp wp uvr uwr vwr w1p w2p w3p Tp ep and
                   fac * (ruu ruv ruw rvv rvw rww rhom thep theup mum num),
                   fac = 1/(mgalx*mgalz) in real*4
    .spe record 1: time, Re, alp, bet (real*4), mx, my, mz, nspec+1,
                   nacumsp (i4)
         record 2: the nspec+1 planes jsptot (i4), then (y_j, fmap_j) real*8
         then one record per kx plane: 12*(nz1+1)*(nspec+1) real*4, |kz|
                   fastest, then spectra plane, then field
* The .cf history line (cross.f:1172-1176): 21 values in format 21(d22.14):
  time, dm, dw, Re*dw, trapz, masst, enerdis, energy(1..9), massu, massv,
  massw, wall time, communication time.
"""
from __future__ import annotations

import dataclasses
import math
import struct
from typing import Dict, Iterable, List, Optional

import numpy as np

_FIELDS = ("vor", "phi", "psi", "scal")


# --------------------------------------------------------------------------
# Fortran sequential records
# --------------------------------------------------------------------------
def _write_record(f, payload: bytes) -> None:
    n = struct.pack("<i", len(payload))
    f.write(n)
    f.write(payload)
    f.write(n)


def _read_record(f) -> Optional[bytes]:
    head = f.read(4)
    if not head:
        return None
    if len(head) != 4:
        raise ValueError("truncated record marker")
    (n,) = struct.unpack("<i", head)
    if n < 0:
        raise ValueError("negative record length (not a little-endian sequential file?)")
    payload = f.read(n)
    tail = f.read(4)
    if len(payload) != n or len(tail) != 4 or struct.unpack("<i", tail)[0] != n:
        raise ValueError("record markers do not match")
    return payload


# --------------------------------------------------------------------------
# restart / image files
# --------------------------------------------------------------------------
@dataclasses.dataclass
class RestartHeader:
    time: float
    Re: float
    alp: float
    bet: float
    a0: float
    mx: int
    my: int
    mz: int
    y: np.ndarray
    fmap: np.ndarray


def write_restart(path: str, state: Dict[str, np.ndarray], y: np.ndarray, fmap: np.ndarray, *, time: float,
                  Re: float, alp: float, bet: float, a0: float = 0.0) -> None:
    """Write a state dict (vor, phi, psi, scal complex [nkx][mz][my]; u00,
    v00, w00 [my]) as the reference writes its images (escru.f:121-139).
    Values are stored in real*4 like the reference; y and fmap in real*8.
    With a passive scalar under "mfz" the plane records carry it as a fifth
    interleaved field, as the scalar-carrying branch reads them
    (branches/lomaHZ/src/main.f:432-433: ntotr = 5*2*my*mz)."""
    vor = np.asarray(state["vor"])
    nkx, mz, my = vor.shape
    y = np.asarray(y, dtype=np.float64)
    fmap = np.asarray(fmap, dtype=np.float64)
    if y.shape != (my,) or fmap.shape != (my,):
        raise ValueError("y and fmap must have my entries")
    head = struct.pack("<5f3i", time, Re, alp, bet, a0, 2 * nkx, my, mz)
    yf = np.empty((my, 2), dtype="<f8")
    yf[:, 0] = y
    yf[:, 1] = fmap
    w00 = np.empty((my, 3), dtype="<f4")
    w00[:, 0] = state["u00"]
    w00[:, 1] = state["v00"]
    w00[:, 2] = state["w00"]
    names = _FIELDS + (("mfz",) if "mfz" in state else ())
    with open(path, "wb") as f:
        _write_record(f, head + yf.tobytes() + w00.tobytes())
        plane = np.empty((mz, 2 * my, len(names)), dtype="<f4")
        for i in range(nkx):
            for q, name in enumerate(names):
                a = np.ascontiguousarray(state[name][i], dtype=np.complex64)  # [mz][my]
                plane[:, :, q] = a.view(np.float32).reshape(mz, 2 * my)
            _write_record(f, plane.tobytes())


def _assign_kz(a: np.ndarray, mz: int) -> np.ndarray:
    """kz re-mapping of a [..][mze][..] array to mz modes (main.f:857-882)."""
    mze = a.shape[-2]
    if mze == mz:
        return a
    out = np.zeros(a.shape[:-2] + (mz, a.shape[-1]), dtype=a.dtype)
    klen = (min(mz, mze) + 1) // 2
    out[..., :klen, :] = a[..., :klen, :]
    if klen > 1:
        out[..., mz - klen + 1:, :] = a[..., mze - klen + 1:, :]
    return out


def read_restart(path: str, mz: Optional[int] = None) -> Dict[str, object]:
    """Read a restart / image file.  Returns a dict with the header
    (RestartHeader under "header") and the state: vor, phi, psi, scal as
    complex128 [nplanes][mz][my] (real*4 values widened), u00, v00, w00, and
    "mfz" when the plane records carry a fifth field (the passive scalar).
    With mz given, the kz modes are re-mapped as the reference does."""
    with open(path, "rb") as f:
        r1 = _read_record(f)
        if r1 is None or len(r1) < 32:
            raise ValueError("missing header record")
        time, Re, alp, bet, a0, mx, my, mze = struct.unpack("<5f3i", r1[:32])
        need = 32 + 16 * my + 12 * my
        if len(r1) != need:
            raise ValueError(f"header record has {len(r1)} bytes, expected {need} for my={my}")
        yf = np.frombuffer(r1, dtype="<f8", count=2 * my, offset=32).reshape(my, 2)
        w00 = np.frombuffer(r1, dtype="<f4", count=3 * my, offset=32 + 16 * my).reshape(my, 3)
        planes: List[np.ndarray] = []
        nf = 4
        while True:
            rec = _read_record(f)
            if rec is None:
                break
            if not planes and len(rec) == 5 * 8 * my * mze:
                nf = 5
            if len(rec) != nf * 8 * my * mze:
                raise ValueError("plane record of unexpected length")
            planes.append(np.frombuffer(rec, dtype="<f4").reshape(mze, 2 * my, nf))
    data = np.stack(planes) if planes else np.zeros((0, mze, 2 * my, nf), dtype=np.float32)
    out: Dict[str, object] = {
        "header": RestartHeader(time, Re, alp, bet, a0, mx, my, mze, yf[:, 0].copy(), yf[:, 1].copy()),
        "u00": w00[:, 0].astype(np.float64), "v00": w00[:, 1].astype(np.float64),
        "w00": w00[:, 2].astype(np.float64), "time": float(time),
    }
    for q, name in enumerate(_FIELDS + (("mfz",) if nf == 5 else ())):
        re_im = np.ascontiguousarray(data[:, :, :, q]).reshape(data.shape[0], mze, my, 2)
        c = (re_im[..., 0].astype(np.float64) + 1j * re_im[..., 1].astype(np.float64))
        out[name] = _assign_kz(c, mz) if mz is not None else c
    return out


# --------------------------------------------------------------------------
# hre.dat
# --------------------------------------------------------------------------
@dataclasses.dataclass
class HreData:
    Re: float
    alp: float
    bet: float
    a0: float
    nstep: int
    nimag: int
    nhist: int
    cfl: float
    ncfl: int
    id22: int
    nstart: int
    ntimes: int
    filout: str
    filinp: str
    filstt: str


def _fortran_values(text: str) -> List[str]:
    return [t for t in text.replace(",", " ").split() if t]


def _ffloat(t: str) -> float:
    return float(t.replace("D", "E").replace("d", "e"))


def read_hre(path: str) -> HreData:
    """Parse hre.dat as initcr does (main.f:502-545)."""
    with open(path) as f:
        lines = [ln.rstrip("\n") for ln in f]
    data = [ln for ln in lines if not ln[:2] == "CC"]
    if len(data) < 7:
        raise ValueError("hre.dat needs 4 parameter lines and 3 file names")
    v = _fortran_values(data[0])
    Re, alp, bet, a0 = (_ffloat(t) for t in v[:4])
    nstep, nimag, nhist = (int(_ffloat(t)) for t in _fortran_values(data[1])[:3])
    v = _fortran_values(data[2])
    cfl, ncfl = _ffloat(v[0]), int(_ffloat(v[1]))
    id22, nstart, ntimes = (int(_ffloat(t)) for t in _fortran_values(data[3])[:3])
    # a70 read, then the name up to the first blank (filout(1:index(filout,' ')-1))
    names = [data[4 + q][:70].split(" ")[0] for q in range(3)]
    return HreData(Re, alp, bet, a0, nstep, nimag, nhist, cfl, ncfl, id22, nstart, ntimes, *names)


# --------------------------------------------------------------------------
# .cf history
# --------------------------------------------------------------------------
def fortran_d(x: float, w: int = 22, d: int = 14) -> str:
    """Fortran Dw.d edit of one value (0.ddd...D+ee, right-justified)."""
    x = float(x)
    if not math.isfinite(x):
        return ("NaN" if math.isnan(x) else ("-Infinity" if x < 0 else "Infinity")).rjust(w)
    sign = "-" if (x < 0 or (x == 0 and math.copysign(1.0, x) < 0)) else ""
    a = abs(x)
    if a == 0.0:
        mant, e = "0" * d, 0
    else:
        s = f"{a:.{d - 1}e}"  # d significant digits: m.mmm e+XX
        digits, exp = s.split("e")
        mant = digits.replace(".", "")
        e = int(exp) + 1
    if abs(e) <= 99:
        ex = f"D{'+' if e >= 0 else '-'}{abs(e):02d}"
    else:
        ex = f"{'+' if e >= 0 else '-'}{abs(e):03d}"
    s = f"{sign}0.{mant}{ex}"
    return s.rjust(w) if len(s) <= w else "*" * w


def cf_line(diag: Dict[str, float], energies: Optional[Iterable[float]] = None, enerdis: float = 0.0,
            wall: float = 0.0, comm: float = 0.0) -> str:
    """One .cf record (cross.f:1172-1176) from a diag dict of Lomacte.diag().
    energy(1..9) and enerdis come from the statistics module of the
    reference; without them they are written as zeros."""
    en = list(energies) if energies is not None else [0.0] * 9
    if len(en) != 9:
        raise ValueError("energy has 9 entries")
    vals = [diag["time"], diag["dm"], diag["dw"], diag["Redw"], diag["trapz"], diag["masst"], enerdis] + en + \
        [diag["massu"], diag["massv"], diag["massw"], wall, comm]
    return "".join(fortran_d(v) for v in vals)


# --------------------------------------------------------------------------
# statistics and spectra files (writestats, escru.f:276-484)
# --------------------------------------------------------------------------
def write_sta(path: str, data, y: np.ndarray, fmap: np.ndarray, *, time: float, Re: float, alp: float,
              bet: float, mgalx: int, mgalz: int, a0: float = 0.0) -> None:
    """Write a .sta file from a StatsData read-back (escru.f:381-402)."""
    from .stats import FAC_FROM, NSTAT, fac32
    prof = np.asarray(data.prof, dtype=np.float64)
    if prof.ndim != 2 or prof.shape[0] != NSTAT:
        raise ValueError("prof must be [33, my]")
    my = prof.shape[1]
    if np.shape(y) != (my,) or np.shape(fmap) != (my,):
        raise ValueError("y and fmap must have my entries")
    rows = np.array(prof.T, dtype="<f8")  # [my][33]
    rows[:, FAC_FROM:] *= fac32(mgalx, mgalz)
    yf = np.empty((my, 2), dtype="<f8")
    yf[:, 0] = y
    yf[:, 1] = fmap
    with open(path, "wb") as f:
        _write_record(f, struct.pack("<i5fi", my, time, Re, alp, bet, a0, int(data.nacum)))
        _write_record(f, yf.tobytes())
        _write_record(f, rows.tobytes())


def read_sta(path: str) -> Dict[str, object]:
    """Read a .sta file: header values, y, fmap and the [33, my] profiles as
    written (the last eleven times fac)."""
    with open(path, "rb") as f:
        r1, r2, r3 = _read_record(f), _read_record(f), _read_record(f)
    if r1 is None or r2 is None or r3 is None or len(r1) != 28:
        raise ValueError("not a .sta file")
    my, time, Re, alp, bet, a0, nacum = struct.unpack("<i5fi", r1)
    yf = np.frombuffer(r2, dtype="<f8").reshape(my, 2)
    rows = np.frombuffer(r3, dtype="<f8").reshape(my, -1)
    return dict(my=my, time=time, Re=Re, alp=alp, bet=bet, a0=a0, nacum=nacum, y=yf[:, 0].copy(),
                fmap=yf[:, 1].copy(), prof=rows.T.copy())


def write_spe(path: str, data, y: np.ndarray, fmap: np.ndarray, *, time: float, Re: float, alp: float,
              bet: float, mx: int, mz: int) -> None:
    """Write a .spe file from a StatsData read-back (escru.f:435-448); the
    spectra are stored in real*4 as the reference accumulates them."""
    spec = np.asarray(data.spec, dtype=np.float64)
    nkx, nf, nsp, nk = spec.shape
    my = len(y)
    if nf != 12 or nsp != len(data.planes) or nkx != mx // 2 or nk != (mz - 1) // 2 + 1:
        raise ValueError("spectra shape does not match the grid")
    yf = np.empty((my, 2), dtype="<f8")
    yf[:, 0] = y
    yf[:, 1] = fmap
    with open(path, "wb") as f:
        _write_record(f, struct.pack("<4f5i", time, Re, alp, bet, mx, my, mz, nsp, int(data.nacumsp)))
        _write_record(f, np.asarray(data.planes, dtype="<i4").tobytes() + yf.tobytes())
        for i in range(nkx):
            _write_record(f, np.ascontiguousarray(spec[i], dtype="<f4").tobytes())


def read_spe(path: str) -> Dict[str, object]:
    """Read a .spe file: header values, planes, y, fmap and the spectra
    [mx/2, 12, nspec+1, nz1+1] (real*4)."""
    with open(path, "rb") as f:
        r1 = _read_record(f)
        if r1 is None or len(r1) != 36:
            raise ValueError("not a .spe file")
        time, Re, alp, bet, mx, my, mz, nsp, nacumsp = struct.unpack("<4f5i", r1)
        r2 = _read_record(f)
        planes = np.frombuffer(r2[:4 * nsp], dtype="<i4").copy()
        yf = np.frombuffer(r2[4 * nsp:], dtype="<f8").reshape(my, 2)
        nk = (mz - 1) // 2 + 1
        spec = np.empty((mx // 2, 12, nsp, nk), dtype=np.float32)
        for i in range(mx // 2):
            r = _read_record(f)
            if r is None:
                raise ValueError("truncated .spe file")
            spec[i] = np.frombuffer(r, dtype="<f4").reshape(12, nsp, nk)
    return dict(time=time, Re=Re, alp=alp, bet=bet, mx=mx, my=my, mz=mz, nacumsp=nacumsp, planes=planes,
                y=yf[:, 0].copy(), fmap=yf[:, 1].copy(), spec=spec)


# tofis_loma's physical-field files (escrphys, trunk/tofis_loma/src/
# escru.f:11-314): per quantity (u, v, w, T, omega_x, omega_y, omega_z) a yz
# file, a yx file and an xz file, each opening with the header record
# time, Re, alp, bet (real*4), mgalx, my, mgalz, nspec, nacum (int) and the
# record of the spectra rows and (y, fmap) pairs (escru.f:88-92); then per
# row j = 1..my the yz line (x = plyz) over z and the yx line (z = plyx)
# over x, and for the rows jspec the whole xz plane (x fastest), real*4.
TOFIS_EXT = (".upyz", ".upyx", ".upxz", ".vpyz", ".vpyx", ".vpxz", ".wpyz", ".wpyx", ".wpxz",
             ".Tfyz", ".Tfyx", ".Tfxz", ".o1yz", ".o1yx", ".o1xz", ".o2yz", ".o2yx", ".o2xz",
             ".o3yz", ".o3yx", ".o3xz")
TOFIS_FIELDS = ("u", "v", "w", "T", "omega_x", "omega_y", "omega_z")


def write_tofis(base: str, fields: Dict[str, np.ndarray], y: np.ndarray, fmap: np.ndarray, *, time: float,
                Re: float, alp: float, bet: float, jspec: Iterable[int], plyz: int = 1, plyx: int = 48,
                nacum: int = 1) -> List[str]:
    """Write the 21 files of escrphys from whole fields [my][mgalz][mgalx]
    (e.g. Lomacte.physical(range(1, my + 1))).  jspec: 1-based rows of the
    xz files; plyz, plyx: 1-based x index of the yz files and z index of
    the yx files (escru.f:86-87).  Returns the paths."""
    my, mgalz, mgalx = np.asarray(fields["u"]).shape
    jspec = [int(j) for j in jspec]
    if not (1 <= plyz <= mgalx and 1 <= plyx <= mgalz) or any(not 1 <= j <= my for j in jspec):
        raise ValueError("plane indices outside the grid")
    head = struct.pack("<4f5i", time, Re, alp, bet, mgalx, my, mgalz, len(jspec), nacum)
    yf = np.empty(2 * my)
    yf[0::2], yf[1::2] = np.asarray(y, dtype=np.float64), np.asarray(fmap, dtype=np.float64)
    head2 = np.asarray(jspec, dtype="<i4").tobytes() + yf.astype("<f8").tobytes()
    paths = []
    for q, name in enumerate(TOFIS_FIELDS):
        a = np.asarray(fields[name], dtype=np.float64)
        for kind in range(3):
            path = base + TOFIS_EXT[3 * q + kind]
            with open(path, "wb") as f:
                _write_record(f, head)
                _write_record(f, head2)
                for j in range(my):
                    if kind == 0:
                        _write_record(f, a[j, :, plyz - 1].astype("<f4").tobytes())
                    elif kind == 1:
                        _write_record(f, a[j, plyx - 1, :].astype("<f4").tobytes())
                    elif j + 1 in jspec:
                        _write_record(f, a[j].astype("<f4").tobytes())
            paths.append(path)
    return paths


def read_tofis(path: str) -> Dict[str, object]:
    """One escrphys file: header values and its records as float32 arrays
    (yz and yx: [my][n]; xz: [nspec][mgalz][mgalx])."""
    with open(path, "rb") as f:
        h = struct.unpack("<4f5i", _read_record(f))
        mgalx, my, mgalz, nspec = h[4], h[5], h[6], h[7]
        r2 = _read_record(f)
        jspec = np.frombuffer(r2[:4 * nspec], dtype="<i4")
        yf = np.frombuffer(r2[4 * nspec:], dtype="<f8")
        recs = []
        while True:
            r = _read_record(f)
            if r is None:
                break
            recs.append(np.frombuffer(r, dtype="<f4"))
    out = {"time": h[0], "Re": h[1], "alp": h[2], "bet": h[3], "mgalx": mgalx, "my": my, "mgalz": mgalz,
           "nspec": nspec, "nacum": h[8], "jspec": jspec, "y": yf[0::2], "fmap": yf[1::2]}
    if path.endswith("xz"):
        out["data"] = np.array(recs).reshape(len(recs), mgalz, mgalx)
    else:
        out["data"] = np.array(recs)
    return out
