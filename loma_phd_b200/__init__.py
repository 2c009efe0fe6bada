"""B200-native lomacte RK3 substep (low-Mach temporal mixing-layer DNS).

The compute lives in liblomacte_b200.so (sm_100a CUDA + C++ host set-up);
``lomacte.Lomacte`` is the host-side mirror of the reference cross1 loop.
Beside it: ``files`` (restart, hre.dat, .cf, .sta/.spe and tofis_loma's
physical-field files), ``stats`` (the statistics' derived quantities),
``driver`` (the reference's main program on the library), ``serve``
(continuous batching of independent runs on one GPU), ``replicas`` and
``slab`` (multi-rank plumbing).
"""
from .lomacte import (PHYSICAL_NAMES, ICParams, Lomacte, LomacteError, Params, lib, make_ic,  # noqa: F401
                      footprint, stretched_mesh, y_metrics)
