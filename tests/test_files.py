"""The reference's file formats: restart images (escru.f:121-139 /
main.f:361-406), hre.dat (main.f:502-545), the .cf line (cross.f:1172-1176)
and the y-metrics written into the restart header."""
import os
import struct

import numpy as np
import pytest

from loma_phd_b200 import Lomacte, y_metrics
from loma_phd_b200.files import cf_line, fortran_d, read_hre, read_restart, write_restart
from tests.helpers import FIELDS, case, oracle_for, rel_l2

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _f32(st):
    out = {k: np.asarray(st[k]).astype(np.complex64).astype(np.complex128) for k in FIELDS}
    out.update({k: np.asarray(st[k]).astype(np.float32).astype(np.float64) for k in ("u00", "v00", "w00")})
    return out


def test_restart_round_trip_and_layout(tmp_path):
    p, y, st = case(16, 16, 33)
    fm = y_metrics(y)["fmap"]
    path = str(tmp_path / "case.001")
    write_restart(path, st, y, fm, time=1.5, Re=p.Re, alp=p.alp, bet=p.bet, a0=0.0)
    r = read_restart(path)
    h = r["header"]
    assert (h.mx, h.my, h.mz) == (2 * p.nplanes, p.my, p.mz)
    assert h.time == pytest.approx(1.5) and h.Re == pytest.approx(p.Re)
    assert np.array_equal(h.y, y) and np.array_equal(h.fmap, fm)
    ref = _f32(st)
    for k in FIELDS + ("u00", "v00", "w00"):
        assert np.array_equal(r[k], ref[k]), k
    # byte layout: record markers, header size, one record per kx plane with
    # the four fields interleaved per real scalar
    raw = open(path, "rb").read()
    n1 = struct.unpack("<i", raw[:4])[0]
    assert n1 == 32 + 16 * p.my + 12 * p.my
    assert struct.unpack("<i", raw[4 + n1:8 + n1])[0] == n1
    off = 8 + n1
    n2 = struct.unpack("<i", raw[off:off + 4])[0]
    assert n2 == 4 * 8 * p.my * p.mz
    first = np.frombuffer(raw[off + 4:off + 4 + 16], dtype="<f4")
    v = np.asarray(st["vor"])[0, 0, 0], np.asarray(st["phi"])[0, 0, 0]
    assert first[0] == np.float32(v[0].real) and first[1] == np.float32(v[1].real)
    assert len(raw) == 8 + n1 + p.nplanes * (8 + n2)


def test_restart_with_scalar_field(tmp_path):
    p, y, st = case(16, 16, 33)
    fm = y_metrics(y)["fmap"]
    st = dict(st)
    st["mfz"] = 0.5 * np.asarray(st["scal"])
    path = str(tmp_path / "case_z.001")
    write_restart(path, st, y, fm, time=0.5, Re=p.Re, alp=p.alp, bet=p.bet)
    r = read_restart(path)
    assert np.array_equal(r["mfz"], np.asarray(st["mfz"]).astype(np.complex64).astype(np.complex128))
    assert np.array_equal(r["vor"], _f32(st)["vor"])
    raw = open(path, "rb").read()
    n1 = struct.unpack("<i", raw[:4])[0]
    assert struct.unpack("<i", raw[8 + n1:12 + n1])[0] == 5 * 8 * p.my * p.mz


def test_restart_kz_remapping(tmp_path):
    p, y, st = case(16, 16, 33)
    path = str(tmp_path / "case.002")
    write_restart(path, st, y, y_metrics(y)["fmap"], time=0.0, Re=p.Re, alp=p.alp, bet=p.bet)
    mz = p.mz
    big = read_restart(path, mz=mz + 6)["vor"]
    klen = (mz + 1) // 2
    src = _f32(st)["vor"]
    assert np.array_equal(big[:, :klen], src[:, :klen])
    assert np.array_equal(big[:, -(klen - 1):], src[:, -(klen - 1):])
    assert np.all(big[:, klen:mz + 6 - klen + 1] == 0)


def test_restart_rejects_bad_files(tmp_path):
    path = tmp_path / "bad"
    path.write_bytes(struct.pack("<i", 8) + b"\0" * 8 + struct.pack("<i", 9))
    with pytest.raises(ValueError):
        read_restart(str(path))


def test_hre_dat(tmp_path):
    text = "\n".join([
        "CC parameters", "CC   Re  alp  bet  a0",
        "   160.0   0.25  0.25   0.",
        "CC nstep nimag nhist",
        "   100   50   10",
        "CC CFL ncfl",
        "  0.5  10",
        "CC first image, stats, ntimes",
        " 3  1  5",
        "CC files",
        "runs/out/mix",
        "runs/in/mix.002",
        "runs/stats/mix_01",
    ])
    path = tmp_path / "hre.dat"
    path.write_text(text + "\n")
    h = read_hre(str(path))
    assert (h.Re, h.alp, h.bet, h.a0) == (160.0, 0.25, 0.25, 0.0)
    assert (h.nstep, h.nimag, h.nhist, h.cfl, h.ncfl) == (100, 50, 10, 0.5, 10)
    assert (h.id22, h.nstart, h.ntimes) == (3, 1, 5)
    assert (h.filout, h.filinp, h.filstt) == ("runs/out/mix", "runs/in/mix.002", "runs/stats/mix_01")


@pytest.mark.parametrize("code,want", [
    ("lomacte3", dict(Re=160.0, alp=0.0136295, bet=0.036319, a0=0.0, nstep=15001, nimag=1000, nhist=200, cfl=0.5,
                      ncfl=10, id22=6, nstart=1, ntimes=1, filout="/share/drive/toni/VDML/s20/01c/s20a",
                      filinp="/share/drive/toni/VDML/s20/01/s20a.005",
                      filstt="/share/drive/toni/VDML/s20/01c/s20a_02")),
    ("lomacte", dict(Re=160.0, alp=0.0182, bet=0.0731, a0=0.0, nstep=21, nimag=10, nhist=5, cfl=0.5, ncfl=10,
                     id22=1, nstart=1, ntimes=5, filout="/data2/toni/turb/3Dinc",
                     filinp="/home/toni/SVNlast/branches/initloma/data/finpinc.dat",
                     filstt="/data2/toni/turb/3Dinc_01")),
])
def test_reference_hre_dat(code, want):
    """The reference's own run-parameter files (trunk/lomacte3/hre.dat,
    trunk/lomacte/hre.dat, copied by tests/golden/make_golden.py), parsed as
    initcr does (main.f:502-545): 'CC' lines skipped, list-directed reads of
    the four parameter records, the first blank-free word of the three a70
    file-name records."""
    h = read_hre(os.path.join(GOLDEN, f"hre_{code}.dat"))
    for k, v in want.items():
        assert getattr(h, k) == v, (k, getattr(h, k), v)


def test_fortran_d_edit():
    assert fortran_d(1.0) == "  0.10000000000000D+01"
    assert fortran_d(-0.00123) == " -0.12300000000000D-02"
    assert fortran_d(0.0) == "  0.00000000000000D+00"
    assert fortran_d(123456.789) == "  0.12345678900000D+06"
    d = dict(time=1.0, dm=2.0, dw=3.0, Redw=480.0, trapz=0.0, masst=1.0, massu=0.0, massv=0.0, massw=0.0)
    line = cf_line(d)
    assert len(line) == 21 * 22
    assert line[22:44] == fortran_d(2.0)


def test_y_metrics_match_oracle():
    p, y, st = case(16, 16, 65)
    m = y_metrics(y)
    o = oracle_for(p, y, st, nthreads=1)
    assert np.allclose(m["fmap"], o.coefs()["fmap"], rtol=1e-13, atol=0)
    assert np.allclose(m["hy"][1:-1], 0.5 * (y[2:] - y[:-2]))


@pytest.mark.gpu
def test_restart_drives_the_gpu_path(gpu, tmp_path):
    """A restart written by the host side loads through the real*4 entry
    point, advances one step on the GPU and matches the FP64 oracle run
    from the same real*4 state; the result writes back to a restart."""
    p, y, st = case(24, 24, 33)
    path = str(tmp_path / "in.000")
    write_restart(path, st, y, y_metrics(y)["fmap"], time=0.0, Re=p.Re, alp=p.alp, bet=p.bet)
    r = read_restart(path)
    g = Lomacte(p, r["header"].y)
    g.load_state_f32({k: np.asarray(r[k]).astype(np.complex64) for k in FIELDS},
                     r["u00"], r["v00"], r["w00"], r["time"])
    g.step(1)
    sg = g.get_state()
    o = oracle_for(p, y, r)
    o.step(1)
    so = o.get_state()
    for k in FIELDS:
        assert rel_l2(sg[k], so[k]) < 1e-10, k
    out = str(tmp_path / "out.001")
    write_restart(out, sg, y, y_metrics(y)["fmap"], time=g.diag()["time"], Re=p.Re, alp=p.alp, bet=p.bet)
    assert np.array_equal(read_restart(out)["scal"], _f32(sg)["scal"])
    g.close()


def test_tofis_files_round_trip(tmp_path):
    """escrphys's 21 files (trunk/tofis_loma/src/escru.f:11-314) from the
    oracle's physical fields of a seeded state: headers, yz/yx lines and
    xz planes read back as written."""
    from loma_phd_b200 import files, y_metrics
    from tests.helpers import case, oracle_for
    p, y, st = case(24, 24, 33)
    o = oracle_for(p, y, st, nthreads=2)
    o.step(1)
    ph = o.physical(list(range(1, p.my + 1)))
    names = files.TOFIS_FIELDS
    fields = {k: ph[:, q] for q, k in enumerate(names)}
    fmap = y_metrics(y)["fmap"]
    base = str(tmp_path / "run")
    paths = files.write_tofis(base, fields, y, fmap, time=0.5, Re=p.Re, alp=p.alp, bet=p.bet, jspec=[16, 17],
                              plyz=3, plyx=5)
    assert len(paths) == 21
    for q, k in enumerate(names):
        a = fields[k].astype(np.float32)
        yz = files.read_tofis(base + files.TOFIS_EXT[3 * q])
        yx = files.read_tofis(base + files.TOFIS_EXT[3 * q + 1])
        xz = files.read_tofis(base + files.TOFIS_EXT[3 * q + 2])
        for r in (yz, yx, xz):
            assert (r["mgalx"], r["my"], r["mgalz"], r["nspec"]) == (p.mgalx, p.my, p.mgalz, 2)
            assert list(r["jspec"]) == [16, 17] and np.array_equal(r["y"], y)
        assert np.array_equal(yz["data"], a[:, :, 2])
        assert np.array_equal(yx["data"], a[:, 4, :])
        assert np.array_equal(xz["data"], a[[15, 16]])
