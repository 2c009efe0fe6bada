"""Host-side checks that need no GPU: the C ABI library loads and exports
every symbol of include/lomacte_b200.h, the seeded initial condition is
deterministic and consistent, and the oracle advances it stably."""
import ctypes
import os
import re

import numpy as np
import pytest

from loma_phd_b200 import ICParams, Params, make_ic, stretched_mesh
from loma_phd_b200 import lomacte as lm
from tests.helpers import case, oracle_for

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, "include", "lomacte_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(lmc_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_header_symbol():
    L = lm.lib()
    syms = header_symbols()
    assert set(syms) == set(lm.SYMBOLS)
    for s in syms:
        assert hasattr(L, s), s


def test_strerror_and_nodev_paths():
    L = lm.lib()
    assert L.lmc_strerror(0) == b"ok"
    assert L.lmc_strerror(-6) == b"no CUDA device"


def test_noalloc_rejects_bad_pointers_before_any_launch():
    """lmc_deryr2_noalloc checks alignment and overlap on the host: these
    pointer values are never dereferenced, so no device is needed."""
    y = stretched_mesh(65)
    n = 4
    nb = n * 65 * 16
    base = 1 << 20
    # an input one double off the 16-byte grid
    assert lm.deryr2_noalloc(y, n, base + 8, base + 4 * nb) == lm.LMC_EINVAL
    # in place, and overlapping by one complex value
    assert lm.deryr2_noalloc(y, n, base, base) == lm.LMC_EINVAL
    assert lm.deryr2_noalloc(y, n, base, base + nb - 16) == lm.LMC_EINVAL
    # beyond the scratch array's largest pencil
    assert lm.deryr2_noalloc(stretched_mesh(545), 1, base, base + 4 * nb) == lm.LMC_EINVAL


def test_create_without_gpu_fails_loudly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("GPU present")
    except Exception:
        pass
    p = Params.from_modes(32, 32, 65)
    with pytest.raises(lm.LomacteError) as e:
        lm.Lomacte(p, stretched_mesh(p.my))
    assert e.value.code == lm.LMC_ENODEV


def test_ic_is_seeded_and_hermitian():
    p, y, a = case(seed=3)
    _, _, b = case(seed=3)
    _, _, c = case(seed=4)
    for k in ("vor", "phi", "psi", "scal"):
        assert np.array_equal(a[k], b[k])
    assert not np.array_equal(a["vor"], c["vor"])
    # kx = 0 plane: field(-kz) = conj(field(kz)) so the physical field is real
    mz = p.mz
    for k in ("vor", "phi", "psi"):
        f = a[k][0]
        for kk in range(1, (mz - 1) // 2 + 1):
            assert np.allclose(f[mz - kk], np.conj(f[kk]), atol=1e-15)
    # T carries only the 00 mode, 1/rho00 with rho_bot/rho_top = s
    assert np.count_nonzero(a["scal"]) == p.my
    T = a["scal"][0, 0].real
    assert abs(T[-1] / T[0] - 4.0) < 1e-3


def test_oracle_runs_ic_stably():
    p, y, st = case(nx=24, nz=24, ny=33)
    o = oracle_for(p, y, st, nthreads=2)
    o.step(3)
    d = o.diag()
    s = o.get_state()
    for k in ("vor", "phi", "psi", "scal"):
        assert np.isfinite(s[k]).all()
    assert abs(d["masst"] - (y[-1] - y[0])) < 0.05
    assert 3.5 < d["dw"] < 4.5


def test_params_struct_matches_header():
    src = open(os.path.join(ROOT, "include", "lomacte_b200.h")).read()
    body = re.search(r"typedef struct lmc_params \{(.*?)\} lmc_params;", src, flags=re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    names = []
    for decl in body.split(";"):
        decl = decl.strip()
        if decl:
            names += [n.strip() for n in decl.split(None, 1)[1].split(",")]
    assert names == [f[0] for f in lm.lmc_params._fields_]


def test_footprint_counts_the_viscosity_buffers():
    base = Params.from_modes(64, 64, 65)
    vis = Params.from_modes(64, 64, 65, visc=1, sigma=0.7)
    zp = (64 // 2) * 65 * 96 * 16  # one FP64 z-physical buffer
    assert lm.footprint(vis) - lm.footprint(base) >= 3 * zp
    both = Params.from_modes(64, 64, 65, visc=1, sigma=0.7, scalar=1)
    sc = Params.from_modes(64, 64, 65, scalar=1)
    assert lm.footprint(both) - lm.footprint(sc) >= 6 * zp


def test_viscosity_x_grid_limit():
    # the x stage's shared memory: mgalx 1152 with the scalar, 1536 without
    ok = Params.from_modes(768, 1, 65, visc=1, sigma=0.7, scalar=1)
    big = Params.from_modes(1024, 1, 65, visc=1, sigma=0.7, scalar=1)
    big_ns = Params.from_modes(1024, 1, 65, visc=1, sigma=0.7)
    assert lm.footprint(ok) > 0 and lm.footprint(big_ns) > 0
    assert lm.footprint(big) == 0
    assert lm.footprint(Params.from_modes(1024, 1, 65, scalar=1)) > 0


@pytest.mark.parametrize("lang,cc", [("c", "gcc"), ("c++", "g++")])
def test_header_compiles_alone(lang, cc, tmp_path):
    import shutil
    import subprocess
    if not shutil.which(cc):
        pytest.skip(f"no {cc}")
    r = subprocess.run([cc, "-fsyntax-only", "-Wall", "-Wextra", "-Werror", "-x", lang,
                        os.path.join(ROOT, "include", "lomacte_b200.h")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.parametrize("grid,s,seed", [((32, 32, 65), 4.0, 0), ((64, 64, 129), 8.0, 1), ((48, 1, 65), 4.0, 2)])
def test_oracle_side_ic_matches_the_library(grid, s, seed):
    """The CPU arms of bench.py build the initial condition with the oracle's
    own restatement (oracle/ic.py) so that they never load the library; it
    is the library's lmc_make_ic up to the round-off of the two y-operator
    builds."""
    from oracle.ic import make_ic as oracle_ic
    p, y, a = case(*grid, s=s, seed=seed)
    b = oracle_ic(p.mgalx, p.mgalz, y, alp=p.alp, bet=p.bet, s=s, seed=seed)
    for k in ("vor", "phi", "psi", "scal", "u00"):
        den = np.linalg.norm(a[k])
        assert np.linalg.norm(a[k] - b[k]) <= 1e-12 * den, k
    for k in ("v00", "w00"):
        assert not np.any(b[k])
