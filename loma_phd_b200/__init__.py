"""B200-native lomacte RK3 substep (low-Mach temporal mixing-layer DNS).

The compute lives in liblomacte_b200.so (sm_100a CUDA + C++ host set-up);
``lomacte.Lomacte`` is the host-side mirror of the reference cross1 loop.
"""
from .lomacte import (ICParams, Lomacte, LomacteError, Params, lib, make_ic,  # noqa: F401
                      footprint, stretched_mesh, y_metrics)
