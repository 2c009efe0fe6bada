"""Pins the oracle's FFT conventions to the reference's own golden vectors
(branches/reactml/benchmark_fft/{cft,rfft}test_double.txt, committed as
tests/golden/fft_rect_double.npz by tests/golden/make_golden.py)."""
import os

import numpy as np

from oracle.oracle import cft, rft

GOLD = os.path.join(os.path.dirname(__file__), "golden", "fft_rect_double.npz")
# the files print 7 significant digits (Fortran E14.7)
TOL = 6e-8


def test_cft_rectangle_matches_reference_golden():
    g = np.load(GOLD)
    x = g["cft_phys"].astype(np.complex128)
    assert len(x) == 384
    X = cft(x, -1)
    assert np.abs(X.real - g["cft_re"]).max() < TOL
    assert np.abs(X.imag - g["cft_im"]).max() < TOL


def test_rft_rectangle_matches_reference_golden():
    g = np.load(GOLD)
    n = 768
    # benchmark_fft/main.f:128-138: four(257:511)=1 except the stale-index
    # element four(385)=0.5; four(256), four(512) stay 0.
    x = np.zeros(n)
    x[256:511] = 1.0
    x[384] = 0.5
    p = rft(x, -1, n)
    assert np.abs(p[:n] - g["rft_four"]).max() < TOL
    # the element after the 768-long array received the Nyquist slot
    assert abs(p[n] - g["rft_physx"][0]) < TOL


def test_fft_round_trips():
    rng = np.random.default_rng(1)
    for n in (96, 144, 384):
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        assert np.allclose(cft(cft(x, -1), 1), x, atol=1e-13)
        xr = rng.standard_normal(n)
        assert np.allclose(rft(rft(xr, -1, n), 1, n), xr, atol=1e-13)
        assert np.allclose(cft(x, -1), np.fft.fft(x) / n, atol=1e-14)
