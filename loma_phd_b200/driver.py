"""The reference's run on the library: what trunk/lomacte3/src/main.f does
around cross1, and the bookkeeping of cross1's time loop
(cross.f:225-1226), with the three substeps of each step on the device.

    run("hre.dat")

reads hre.dat (main.f:502-570) and the restart file it names, advances
nstep RK3 steps in the reference's CFL mode (Deltat starting at 1e-4,
main.f:559, recomputed every ncfl steps), and writes what the reference
writes: an image every nimag steps (filout.NNN, escru.f:11-193), the
statistics of the ntimes steps before each nhist boundary when nstart /= 0
(filstt_NNN.sta / .spe, escru.f:276-484), and a .cf line every nhist steps
(filstt.cf, cross.f:1172-1176).  A restart file whose plane records carry
a fifth field (the passive scalar, "mfz") runs with the scalar and writes
it into its images; sigma selects the variable viscosity mu = T^sigma
(branches/loma reads it as hre.dat's fourth value, main.f:543).
"""
from __future__ import annotations

import dataclasses
import os
import time as _time
from typing import Callable, Dict, List, Optional

import numpy as np

from . import files, stats as stats_mod
from .lomacte import Lomacte, Params, y_metrics


@dataclasses.dataclass
class StepFlags:
    image: bool        # write an image before the step (cross.f:244)
    stats: bool        # the step accumulates statistics (istati = 1)
    write_stats: bool  # write .sta/.spe after the step (cross.f:1145)
    hist: bool         # write a .cf line after the step (cross.f:1168)


def step_flags(istep: int, nimag: int, nhist: int, ntimes: int, nstart: int, istati: bool):
    """Flags of step istep (1-based) and the next istati (cross.f:236-260,
    1145-1162)."""
    if nstart != 0 and (istep - 1) % nhist == nhist - ntimes:
        istati = True
    hist = istep % nhist == 0
    image = (istep - 1) % nimag == 0 and istep != 1
    fl = StepFlags(image=image, stats=istati, write_stats=hist and istati, hist=hist)
    return fl, (False if fl.write_stats else istati)


def grid_of(mx: int, mz: int):
    """mgalx, mgalz of a restart header's mx, mz (ctes3D:26-27 inverted)."""
    return 3 * mx // 2, 3 * (mz + 1) // 2


def run(hre_path: str, workdir: Optional[str] = None, precision: int = 0, device: int = 0,
        planes: Optional[List[int]] = None, nstep: Optional[int] = None,
        log: Optional[Callable[[str], None]] = None, sigma: Optional[float] = None,
        schmidt: float = 0.0) -> Dict[str, object]:
    """Run a case as the reference's main program does.  File names in
    hre.dat are relative to workdir (default: the directory of hre.dat).
    planes: 1-based rows of the spectra (default: the centre row, the
    reference's jsptot(nspec+1)); nstep overrides hre.dat's; sigma: mu =
    T^sigma (None: constant viscosity); schmidt: Sc of a scalar the restart
    carries (<= 0: Sc = Pr)."""
    wd = workdir or os.path.dirname(os.path.abspath(hre_path))
    h = files.read_hre(hre_path)
    r = files.read_restart(os.path.join(wd, h.filinp))
    hd = r["header"]
    mgalx, mgalz = grid_of(hd.mx, hd.mz)
    has_z = "mfz" in r
    p = Params(mgalx=mgalx, mgalz=mgalz, my=hd.my, Re=h.Re, alp=h.alp, bet=h.bet, cfl=h.cfl, ncfl=h.ncfl,
               dt_mode=0, dt=1e-4, precision=precision, device=device, scalar=int(has_z), schmidt=schmidt,
               visc=0 if sigma is None else 1, sigma=sigma or 0.0)
    y = np.asarray(hd.y)
    met = y_metrics(y)
    fmap = met["fmap"]
    case = Lomacte(p, y)
    case.load_state_f32({k: r[k] for k in ("vor", "phi", "psi", "scal")}, r["u00"], r["v00"], r["w00"], r["time"])
    if has_z:
        case.load_scalar(np.asarray(r["mfz"], dtype=np.complex128))
    planes = planes or [(hd.my + 1) // 2]
    case.stats_reset(planes)
    id22, ista = h.id22, h.id22  # main.f:565-566
    out = {"images": [], "sta": [], "spe": [], "cf": os.path.join(wd, h.filstt + ".cf"), "steps": 0}
    n = h.nstep if nstep is None else nstep
    istati = False
    t0 = _time.perf_counter()
    with open(out["cf"], "a") as cf:
        for istep in range(1, n + 1):
            fl, istati = step_flags(istep, h.nimag, h.nhist, h.ntimes, h.nstart, istati)
            if fl.image:
                st = case.get_state()
                if has_z:
                    st["mfz"] = case.get_scalar()
                path = os.path.join(wd, f"{h.filout}.{id22:03d}")
                files.write_restart(path, st, y, fmap, time=st["time"], Re=h.Re, alp=h.alp, bet=h.bet, a0=h.a0)
                out["images"].append(path)
                id22 += 1
            if fl.stats:
                case.stats_step(1)
            else:
                case.step(1)
            energies, enerdis = None, 0.0
            if fl.write_stats:
                data = case.stats_read(clear_spectra=True)
                d = case.diag()
                base = os.path.join(wd, f"{h.filstt}_{ista:03d}")
                files.write_sta(base + ".sta", data, y, fmap, time=d["time"], Re=h.Re, alp=h.alp,
                                bet=h.bet, mgalx=mgalx, mgalz=mgalz, a0=h.a0)
                files.write_spe(base + ".spe", data, y, fmap, time=d["time"], Re=h.Re, alp=h.alp,
                                bet=h.bet, mx=hd.mx, mz=hd.mz)
                out["sta"].append(base + ".sta")
                out["spe"].append(base + ".spe")
                ista += 1
                energies = stats_mod.energies(data.uner)
                enerdis = stats_mod.enerdis(data, met["hy"])
                case.stats_reset(planes)  # resetstats after writing (cross.f:1160)
            if fl.hist:
                d = case.diag()
                line = files.cf_line(d, energies, enerdis, wall=_time.perf_counter() - t0)
                cf.write(line + "\n")
                cf.flush()
                if log:
                    log(f"step {istep} time {d['time']:.6f} Deltat {d['Deltat']:.3e} dm {d['dm']:.6f}")
            out["steps"] = istep
    out["state"] = case.get_state()
    if has_z:
        out["state"]["mfz"] = case.get_scalar()
    case.close()
    return out
