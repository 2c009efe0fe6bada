"""The reference's run loop on the library (loma_phd_b200/driver.py): the
step schedule of cross.f:236-260 and 1145-1162 on the CPU, and a short
run from hre.dat and a restart file on the GPU that writes the reference's
images, .sta/.spe and .cf files and ends on the state plain steps reach."""
import os

import numpy as np
import pytest

from loma_phd_b200 import Lomacte, y_metrics
from loma_phd_b200 import files
from loma_phd_b200.driver import grid_of, run, step_flags
from tests.helpers import FIELDS, case


def _schedule(n, nimag, nhist, ntimes, nstart):
    istati, out = False, []
    for istep in range(1, n + 1):
        fl, istati = step_flags(istep, nimag, nhist, ntimes, nstart, istati)
        out.append(fl)
    return out


def test_step_schedule():
    fl = _schedule(12, 5, 4, 2, 1)
    assert [i + 1 for i, f in enumerate(fl) if f.stats] == [3, 4, 7, 8, 11, 12]
    assert [i + 1 for i, f in enumerate(fl) if f.write_stats] == [4, 8, 12]
    assert [i + 1 for i, f in enumerate(fl) if f.hist] == [4, 8, 12]
    assert [i + 1 for i, f in enumerate(fl) if f.image] == [6, 11]
    assert not any(f.stats for f in _schedule(12, 5, 4, 2, 0))  # nstart = 0: no statistics


def test_grid_of_header():
    p, _, _ = case(64, 96, 33)
    assert grid_of(2 * p.nplanes, p.mz) == (p.mgalx, p.mgalz)


def _write_case(tmp, p, y, st):
    files.write_restart(os.path.join(tmp, "start.000"), st, y, y_metrics(y)["fmap"], time=0.0, Re=p.Re, alp=p.alp,
                        bet=p.bet, a0=0.0)
    with open(os.path.join(tmp, "hre.dat"), "w") as f:
        f.write("CC run of the driver test\n")
        f.write(f"{p.Re} {p.alp} {p.bet} 0.0\n12 5 4\n0.5 2\n1 1 2\nrun\nstart.000\nrunst\n")


@pytest.mark.gpu
def test_driver_run(gpu, tmp_path):
    p, y, st = case(24, 24, 33)
    tmp = str(tmp_path)
    _write_case(tmp, p, y, st)
    out = run(os.path.join(tmp, "hre.dat"))
    assert out["steps"] == 12
    assert [os.path.basename(x) for x in out["images"]] == ["run.001", "run.002"]
    assert [os.path.basename(x) for x in out["sta"]] == ["runst_001.sta", "runst_002.sta", "runst_003.sta"]
    lines = open(out["cf"]).read().splitlines()
    assert len(lines) == 3 and all(len(ln) == 21 * 22 for ln in lines)
    energy = [float(v.replace("D", "E")) for v in [lines[0][22 * k:22 * (k + 1)] for k in range(7, 16)]]
    assert energy[0] > 0  # from the statistics of the steps before the line
    s = files.read_sta(out["sta"][0])
    assert s["nacum"] == 2 and s["my"] == p.my
    img = files.read_restart(out["images"][0])
    assert img["header"].mz == p.mz
    # the same steps without the driver (CFL mode, Deltat from 1e-4)
    r = files.read_restart(os.path.join(tmp, "start.000"))
    q = type(p)(**{**p.__dict__, "dt_mode": 0, "dt": 1e-4, "cfl": 0.5, "ncfl": 2})
    g = Lomacte(q, y)
    g.load_state_f32({k: r[k] for k in FIELDS}, r["u00"], r["v00"], r["w00"], 0.0)
    g.step(12)
    ref = g.get_state()
    g.close()
    for k in FIELDS:
        np.testing.assert_array_equal(out["state"][k], ref[k], err_msg=k)


@pytest.mark.gpu
def test_driver_run_with_scalar_and_viscosity(gpu, tmp_path):
    p, y, st = case(24, 24, 33)
    T = st["scal"]
    tb, tt = T[0, 0, 0].real, T[0, 0, -1].real
    z = T / (tt - tb)
    z[0, 0, :] -= tb / (tt - tb)
    st = dict(st, mfz=z)
    tmp = str(tmp_path)
    _write_case(tmp, p, y, st)
    out = run(os.path.join(tmp, "hre.dat"), sigma=0.7)
    assert out["steps"] == 12 and "mfz" in out["state"]
    img = files.read_restart(out["images"][0])
    assert "mfz" in img
    # the same steps without the driver
    r = files.read_restart(os.path.join(tmp, "start.000"))
    q = type(p)(**{**p.__dict__, "dt_mode": 0, "dt": 1e-4, "cfl": 0.5, "ncfl": 2, "scalar": 1, "visc": 1,
                   "sigma": 0.7})
    g = Lomacte(q, y)
    g.load_state_f32({k: r[k] for k in FIELDS}, r["u00"], r["v00"], r["w00"], 0.0)
    g.load_scalar(np.asarray(r["mfz"], dtype=np.complex128))
    g.step(12)
    ref, zr = g.get_state(), g.get_scalar()
    g.close()
    for k in FIELDS:
        np.testing.assert_array_equal(out["state"][k], ref[k], err_msg=k)
    np.testing.assert_array_equal(out["state"]["mfz"], zr)
