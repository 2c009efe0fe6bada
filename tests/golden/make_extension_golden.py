"""Regenerate tests/golden/extensions_24x33x24.npz: a regression pin of the
oracle's restatement of the two extensions that no lomacte code carries
(the passive scalar and mu = k = rho D = T^sigma), so that later changes to
the oracle cannot move them unnoticed.

Case: 24 x 24 Fourier modes x 33 rows, the seeded initial condition (s = 4,
seed 0), Z = (T - T_bot)/(T_top - T_bot), Sc = 1.3, sigma = 0.7, Deltat =
0.01; three RK3 steps.  Stored per field (vor, phi, psi, scal, Z) the L2
norm and 40 sampled complex values at fixed indices, and u00.

Usage: python tests/golden/make_extension_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

FIELDS = ("vor", "phi", "psi", "scal", "Z")


def run():
    from tests.helpers import case, oracle_for
    p, y, st = case(24, 24, 33)
    T = st["scal"]
    tb, tt = T[0, 0, 0].real, T[0, 0, -1].real
    z = T / (tt - tb)
    z[0, 0, :] -= tb / (tt - tb)
    o = oracle_for(p, y, st, nthreads=1)
    o.set_scalar(z, 1.3)
    o.set_viscosity(0.7)
    o.step(3)
    s = o.get_state()
    s["Z"] = o.get_scalar()
    return s


def sample_index(shape, n=40, seed=11):
    rng = np.random.default_rng(seed)
    return tuple(rng.integers(0, d, n) for d in shape)


def main():
    s = run()
    out = {"u00": s["u00"]}
    for k in FIELDS:
        idx = sample_index(s[k].shape)
        out[k + "_norm"] = np.array(np.linalg.norm(s[k]))
        out[k + "_sample"] = s[k][idx]
    np.savez(os.path.join(HERE, "extensions_24x33x24.npz"), **out)


if __name__ == "__main__":
    main()
