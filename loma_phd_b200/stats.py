"""Statistics of an accumulating run: names, layout and the derived numbers
the reference prints (trunk/lomacte3/src/cross.f:1145-1176,
escru.f:276-484).

The device accumulates, while a step runs through ``Lomacte.stats_step``,
what addstats1 / addstats2 (cross.f:1981-2290) and the physical sums of
phys2 (cross.f:1583-1607) accumulate while istati = 1.  ``StatsData`` holds
one read-back of those accumulators.
"""
from __future__ import annotations

import dataclasses
from typing import List

import numpy as np

# Profiles in the order of the .sta record (escru.f:381-402): eleven means
# of 00 modes, then wkstats(j, 1..22).  Indices >= FAC_FROM are multiplied by
# 1/(mgalx*mgalz) when written (sums over physical planes, plus thep and
# theup, which writestats scales the same way).
STAT_NAMES = (
    "um", "vm", "wm", "rum", "rvm", "rwm", "Tm", "w1m", "w2m", "w3m", "them",
    "up", "vp", "wp", "uvr", "uwr", "vwr", "w1p", "w2p", "w3p", "Tp", "ep",
    "ruu", "ruv", "ruw", "rvv", "rvw", "rww", "rhom", "thep", "theup", "mum", "num",
)
NSTAT = len(STAT_NAMES)
FAC_FROM = STAT_NAMES.index("ruu")

# Fields of the spectra (cross.f:2097-2098, 2001-2002)
SPEC_FIELDS = ("u", "v", "w", "uv_re", "uv_im", "o1", "o2", "o3", "rhou", "rhov", "rhow", "T")

# The nine energies of uner (cross.f:2153-2182)
ENERGY_NAMES = ("up", "vp", "wp", "uvr", "uwr", "vwr", "w1p", "w2p", "w3p")


@dataclasses.dataclass
class StatsData:
    """One read-back of the accumulators.

    prof   [33, my]                raw profiles, STAT_NAMES order
    spec   [nplanes, 12, nsp, nz1+1] spectra, SPEC_FIELDS order, |kz| fastest
    uner   [9]                     hy-weighted energies of the last step
    nacum, nacumsp                 accumulated steps (profiles, spectra)
    planes                         1-based y rows of the spectra
    sigma                          exponent of mu/mu0 = T^sigma
    """
    prof: np.ndarray
    spec: np.ndarray
    uner: np.ndarray
    nacum: int
    nacumsp: int
    planes: List[int]
    sigma: float = 0.0

    def profile(self, name: str) -> np.ndarray:
        return self.prof[STAT_NAMES.index(name)]

    def spectrum(self, field: str) -> np.ndarray:
        """[nplanes, nsp, nz1+1] spectrum of one field."""
        return self.spec[:, SPEC_FIELDS.index(field)]


def fac32(mgalx: int, mgalz: int) -> float:
    """writestats' fac = 1/(mgalx*mgalz), a real*4 variable (escru.f:371, 380)."""
    return float(np.float32(1.0 / (mgalx * mgalz)))


def energies(uner) -> np.ndarray:
    """energy(i) = sqrt(|uner(i)|), the nine .cf energies (cross.f:808-815)."""
    return np.sqrt(np.abs(np.asarray(uner, dtype=np.float64)))


def enerdis(data: StatsData, hy) -> float:
    """Mean dissipation sum_j ep(j)/nacum hy(j) (cross.f:1152-1157)."""
    if data.nacum <= 0:
        return 0.0
    return float(np.sum(data.profile("ep") / data.nacum * np.asarray(hy)))


def masst(data: StatsData, hy, mgalx: int, mgalz: int) -> float:
    """masst = sum_j fac rhom(j) hy(j) (escru.f:371-375).  The reference's
    loop runs j = 0..my-1 over wkstats(j, 18) * hy(j+1), one row off (its
    j = 0 term reads outside the rhom column); this is the aligned sum."""
    return float(np.sum(fac32(mgalx, mgalz) * data.profile("rhom") * np.asarray(hy)))
