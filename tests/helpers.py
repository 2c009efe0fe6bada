"""Shared set-up of the parity tests: grids, seeded initial conditions and
the relative L2 error used against the FP64 oracle."""
import numpy as np

from loma_phd_b200 import ICParams, Params, make_ic, stretched_mesh
from oracle.oracle import Oracle

FIELDS = ("vor", "phi", "psi", "scal")


def case(nx=32, nz=32, ny=65, seed=0, s=4.0, dt_mode=1, dt=0.01, Re=160.0, **kw):
    p = Params.from_modes(nx, nz, ny, Re=Re, dt_mode=dt_mode, dt=dt, **kw)
    y = stretched_mesh(p.my)
    st = make_ic(p, y, ICParams(s=s, seed=seed))
    return p, y, st


def oracle_for(p, y, st, nthreads=None):
    o = Oracle(p.mgalx, p.mgalz, y, p.Re, p.alp, p.bet, peclet=None if p.peclet <= 0 else p.peclet,
               cfl=p.cfl, ncfl=p.ncfl, dtmode=p.dt_mode, dt0=p.dt, nthreads=nthreads,
               variant=getattr(p, "variant", 0))
    o.set_state(st["vor"], st["phi"], st["psi"], st["scal"], st["u00"], st["v00"], st["w00"], st.get("time", 0.0))
    return o


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.linalg.norm(b.ravel())
    num = np.linalg.norm((a - b).ravel())
    return num / den if den > 0 else num


def mixing_scalar(p, y):
    """The passive scalar of the mixing-layer workloads: Z = 0.5 (1 +
    tanh(y/2)) in the kx = kz = 0 mode, no fluctuation."""
    z = np.zeros(p.shape, dtype=np.complex128)
    z[0, 0, :] = 0.5 * (1.0 + np.tanh(np.asarray(y) / 2.0))
    return z
