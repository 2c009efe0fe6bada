"""bench.py's algorithmic byte model (the roofline numerator) on the CPU:
the x stage's compulsory bytes of the bench workloads counted by hand, and
the JSON contract of the reference arm on a tiny case."""
import json
import os
import subprocess
import sys

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _sizes(nx, nz, ny):
    nplanes, mz, mgalx, mgalz = nx // 2, nz - 1, 3 * nx // 2, 3 * nz // 2
    return nplanes * mz * ny, nplanes * mgalz * ny, mgalx * mgalz * ny


def test_xstage_bytes_by_hand():
    S, Z, P = _sizes(256, 256, 257)
    # lomacte3 substep, mixed: 8 input lines read, 11 output lines written, RHS(T) read + written
    assert bench.ALGO["xphys"](S, Z, P, 8, 0, 0) == (8 + 11) * Z * 8 + 2 * P * 8
    # with the scalar and mu = T^sigma: 8 + 4 + 6 inputs, 12 outputs, RHS(T) and RHS(Z)
    assert bench.ALGO["xphys"](S, Z, P, 8, 1, 1) == (18 + 12) * Z * 8 + 4 * P * 8
    assert abs(bench.ALGO["xphys"](S, Z, P, 8, 1, 1) - 4.245e9) < 1e6
    assert abs(bench.ALGO["xphys"](S, Z, P, 16, 1, 1) - 7.276e9) < 1e6
    # z transforms: 6 (+3 scalar, +4 viscosity) spectral inputs read, 8 (+4, +6) z-padded written
    assert bench.ALGO["zinv"](S, Z, P, 8, 1, 1) == 13 * S * 8 + 18 * Z * 8


def test_reference_arm_line():
    """The reference arm: RK3-step accounting of its bounded samples, the
    JSON contract, and no product library in its process."""
    code = ("import runpy, sys, io, contextlib; sys.argv = ['bench.py', '--impl', 'reference', '--workload', "
            "'medium', '--ny', '33', '--steps', '3', '--warmup', '1']; buf = io.StringIO()\n"
            "with contextlib.redirect_stdout(buf): runpy.run_path('bench.py', run_name='__main__')\n"
            "print(buf.getvalue().strip().splitlines()[-1])\n"
            "print(sorted(set(l.split()[-1] for l in open('/proc/self/maps') if 'lomacte' in l)))")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    out = r.stdout.strip().splitlines()
    d = json.loads(out[-2])
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["e2e"]["value"] == d["value"] and d["cpu_baseline"]["kind"] == "port"
    assert "passive scalar" in d["config"]["workload"] and "T^0.7" in d["config"]["workload"]
    # each step is one sample of 1/16 of a substep of the 256^2 x 33 slab, i.e. 1/48 RK3 step
    w = bench.WORKLOADS["medium"]
    rk3 = 256 * 256 * 33 / 1e6 / (3 * w["ref_stride"])
    assert abs(d["value"] - rk3 / (d["ms_per_step"] / 1e3)) < 1e-9 * d["value"]
    assert d["steps"] == 3 and d["warmup"] == 1
    libs = eval(out[-1])
    assert libs and all("oracle" in x for x in libs), libs
