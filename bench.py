#!/usr/bin/env python
"""Benchmark of the lomacte RK3 step on B200 (Mpts.RK3-steps/s).

Workload (default, ``--workload large``): the large single run of the
low-Mach temporal mixing layer, nx = nz = 768 Fourier modes (3/2
dealiased: mgalx = mgalz = 1152), ny = 513 on y = 12 sinh(2 eta)/sinh(2),
Lx = Lz = 8 pi, seeded initial condition (density ratio s = T2/T1 = 8,
seed 1, rms 1e-2 on |k| <= 8 windowed by exp(-y^2/4)), Re = 800, Deltat
from CFL = 0.5 (recomputed every 10 steps, initial Deltat 1e-4 as the
reference), Pr = Sc = 0.7, mu = k = rho D = T^0.7 and a passive scalar
Z = 0.5 (1 + tanh(y/2)).  ``--workload medium`` is the 256^2 x 257 run
(s = 4, Re = 160, Deltat = 0.01, seed 0) with the same physics, and its
line is also reported beside the headline (``medium_grid``).  One "step"
= one full RK3 step (3 substeps).  The metric is (nx*ny*nz/1e6) * steps /
seconds, measured for the mixed-precision form (the headline value) and
the FP64 plain path (reported beside it, with the ratio and the relative
L2 difference of the two final states), and on the medium grid the
difference of the two forms after 1000 steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload large|medium] [--precision both|mixed|fp64]

N > 1 runs N independent replicas (one per GPU, launched by torchrun); the
time is the max over ranks and the value the aggregate over ranks.
``--impl reference`` times the CPU restatement of the reference algorithm
(the reference Fortran cannot be built in this environment: no Fortran
compiler, no MPI) on the host cores, on bounded samples of the same
workload (see ``cpu_sample``); it never loads the product library.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from loma_phd_b200.replicas import job_throughput, max_over_ranks  # noqa: E402

# The two mixing-layer workloads (hre.dat-equivalent parameters).  y_cpu
# and the strides are the bounded CPU samples: the oracle runs on the same
# x/z grid with y_cpu of the y points (its per-point cost does not depend
# on ny: every y solve is banded, every transform is per y row) and visits
# 1/stride of a substep's modes, planes and lines (lmo_set_sample).
WORKLOADS = {
    "large": dict(nx=768, nz=768, ny=513, s=8.0, Re=800.0, seed=1, dt_mode=0, dt=1e-4, cfl=0.5, ncfl=10,
                  y_cpu=65, cpu_stride=2, ref_stride=8,
                  desc="768^2 x 513 modes (mgal 1152^2), s=8, Re=800, seed 1, Deltat from CFL=0.5 every 10 steps"),
    "medium": dict(nx=256, nz=256, ny=257, s=4.0, Re=160.0, seed=0, dt_mode=1, dt=0.01, cfl=0.5, ncfl=10,
                   y_cpu=257, cpu_stride=4, ref_stride=16,
                   desc="256^2 x 257 modes (mgal 384^2), s=4, Re=160, Deltat=0.01"),
}
PR = float(np.float32(0.7))  # Pr = Sc = 0.7f (main.f:569)

# Algorithmic HBM bytes per launch, in units of the spectral (S = nplanes *
# mz * ny complex), z-padded (Z = nplanes * mgalz * ny complex) and physical
# (P = mgalx * mgalz * ny real) counts.  State fields (Omega_y, phi, psi, T,
# R_Omega, R_phi) are FP64 complex (16 B) in both forms; transform work
# buffers take w bytes per complex value (16 in the FP64 form, 8 in the mixed
# form).  Compulsory reads + writes of each kernel group (one profile id):
#   zinv : 6 spectral inputs read (rho u, rho v, rho w, lap T, dT/dy, T), 8 Z written
#   xphys: 8 Z read, 11 Z written, RHS(T) physical accumulator (FP64) read + written
#   zfwd : 11 Z read, 11 S written
#   lapv : phi read, m_y and dm_y/dy written (+ 7 doubles/point mode tables read)
#   assemble: vor, psi, R_om, phi, R_phi, m_y, dm_y read; rho u, rho v, rho w, vor, phi written
#   tder : T read and written; dT/dy, lap T written
#   post1: T, DT, rho vv, rho uv, rho vw, rho uu, rho uw, rho ww read; T, N_x, N_y, N_z written
#   post2: u, v, w, N_x, N_y, N_z, vor, phi read; R_om, R_phi, vor, phi written
#          (two launches, post2a and post2b, counted together as one stage)
#   psi  : drho read, psi written (+ 7 doubles/point mode tables read)
# The passive scalar (sc) adds to zinv lap Z, dZ/dy, Z read and 4 Z
# written; to xphys 4 Z read, 1 Z written (the twelfth output) and its
# physical accumulator; to zfwd the twelfth output; to tder (t_zder) Z read
# and written, dZ/dy, lap Z written; to zfwd's profile id (t_zupd) Z read
# and written, Delta Z read.  The variable viscosity (vs) adds to zinv the
# four strain-rate sums read and 6 Z written; to xphys 6 Z read; to the
# assemble id (t_sgrad) rho u, rho v, rho w read and the four sums written.
ALGO = {
    "zinv": lambda S, Z, P, w, sc, vs: (6 + 3 * sc + 4 * vs) * S * w + (8 + 4 * sc + 6 * vs) * Z * w,
    "xphys": lambda S, Z, P, w, sc, vs: (19 + 5 * sc + 6 * vs) * Z * w + 2 * (1 + sc) * P * 8,
    "zfwd": lambda S, Z, P, w, sc, vs: (11 + sc) * (Z + S) * w + sc * (2 * S * 16 + S * w),
    "lapv": lambda S, Z, P, w, sc, vs: S * 16 + 2 * S * w + S * 7 * 8 // 2,
    "assemble": lambda S, Z, P, w, sc, vs: 7 * S * 16 + 5 * S * w + vs * 7 * S * w,
    "tder": lambda S, Z, P, w, sc, vs: (1 + sc) * (2 * S * 16 + 2 * S * w),
    "post1": lambda S, Z, P, w, sc, vs: 2 * S * 16 + 10 * S * w,
    "post2": lambda S, Z, P, w, sc, vs: 6 * S * 16 + 6 * S * w,
    "psi": lambda S, Z, P, w, sc, vs: S * 16 + S * w + S * 7 * 8 // 2,
}

# DRAM bytes (read + write) per launch measured by ncu, by (workload, FP64
# form): full-set captures of one launch on a case of the same x/z grid
# with fewer y points (profiles/), scaled to a full launch by ny, as every
# kernel's traffic grows in proportion to ny at fixed x/z sizes.  None:
# not captured for that kernel.
NCU_TRAFFIC = {
    # 768^2 x 33 (mgal 1152^2), mu = T^0.7 + scalar: profiles/kernels_transforms_large_768x33x768.md
    ("large", False, 1, 1): {"xphys": (5.0270e9, 33)},
    ("large", True, 1, 1): {"xphys": (8.3872e9, 33)},
    # 256^2 x 65 (mgal 384^2), mu = T^0.7 + scalar: profiles/kernels_xphys_mu07_scalar_256x65x256.md
    ("medium", False, 1, 1): {"xphys": (1026.2e6, 65)},
    ("medium", True, 1, 1): {"xphys": (1791.0e6, 65)},
}

MIXED_NAMES = {1: "mixed (FP32 storage and FFTs, FP64 state/solves/00 modes)",
               2: "mixed (FP32 storage, FP64 FFT arithmetic, state/solves/00 modes)"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--workload", default="large", choices=tuple(WORKLOADS))
    ap.add_argument("--ny", type=int, default=0, help="override the workload's ny (profiling of small cases)")
    ap.add_argument("--precision", default="both", choices=("both", "mixed", "fp64"),
                    help="both: time the FP64 and the mixed form; the headline value is the mixed form")
    ap.add_argument("--mixed-form", type=int, default=1, choices=(1, 2),
                    help="1: FP32 FFT arithmetic; 2: FP64 FFT arithmetic on FP32 storage")
    ap.add_argument("--no-medium", action="store_true", help="skip the medium-grid line beside the headline")
    ap.add_argument("--error-steps", type=int, default=1000,
                    help="steps of the mixed-vs-FP64 error run (0: skip)")
    ap.add_argument("--error-workload", default="medium", choices=tuple(WORKLOADS),
                    help="workload of the error run (the large one takes about 25 GPU-minutes for 1000 steps)")
    ap.add_argument("--serve-requests", type=int, default=16,
                    help="requests of the synthetic serving stream (0: skip)")
    ap.add_argument("--serve-scale", type=float, default=0.05,
                    help="factor on the stream's step counts (log-uniform in [200, 2000])")
    ap.add_argument("--ensemble", type=int, default=0,
                    help="also run an ensemble of this many independent cases of uneven grids (0: skip)")
    ap.add_argument("--ensemble-steps", type=int, default=500)
    ap.add_argument("--no-scalar", dest="scalar", action="store_false",
                    help="without the passive scalar Z (the lomacte3 substep carries none)")
    ap.add_argument("--sigma", type=float, default=0.7,
                    help="mu = k = rho D = T^sigma; negative: the constant viscosity of lomacte3")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--json-only", action="store_true")
    a = ap.parse_args()
    if a.sigma < 0:
        a.sigma = None
    return a


def wl(a, name=None):
    """The workload's parameters (ny overridden by --ny for the main one)."""
    w = dict(WORKLOADS[name or a.workload])
    w["name"] = name or a.workload
    if name is None and a.ny:
        w["ny"] = a.ny
        w["y_cpu"] = min(w["y_cpu"], a.ny)
    return w


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        if self.proc is None:
            return out
        try:
            self.proc.terminate()
            self.proc.wait(timeout=5)
        except Exception:
            pass
        try:
            rows = [l.strip().split(",") for l in open(self.path) if l.strip()]
            os.unlink(self.path)
        except Exception:
            return out
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except ValueError:
                continue
            for n, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if sm:
            out = {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                   "samples": len(sm)}
        return out


def mpts(w, ny=None):
    return w["nx"] * (ny or w["ny"]) * w["nz"] / 1e6


def sizes(p):
    S = p.nplanes * p.mz * p.my
    Z = p.nplanes * p.mgalz * p.my
    P = p.mgalx * p.mgalz * p.my
    return S, Z, P


def mixing_scalar(shape, y):
    """Z = 0.5 (1 + tanh(y/2)): the kx = kz = 0 mode of the spectral Z."""
    z = np.zeros(shape, dtype=np.complex128)
    z[0, 0, :] = 0.5 * (1.0 + np.tanh(np.asarray(y) / 2.0))
    return z


def extensions(a):
    e = (" + passive scalar Z=0.5(1+tanh(y/2)), Sc=0.7" if a.scalar else "") + \
        (f" + mu = T^{a.sigma:g}" if a.sigma is not None else "")
    return e


def config(a, w, form):
    return {"workload": f"lomacte {form}{extensions(a)}, Pr=0.7, {w['desc']}",
            "grid": f"{w['nx']}x{w['ny']}x{w['nz']}", "parallelism": "replicas",
            "l2": "inputs larger than L2"}


def mesh(ny):
    eta = np.linspace(-1.0, 1.0, ny)
    return 12.0 * np.sinh(2.0 * eta) / np.sinh(2.0)


def cpu_sample(a, w, stride, nth, warmup, nsamples):
    """Bounded CPU samples of the workload with the FP64 oracle: the same
    x/z grid, y_cpu of its y points, 1/stride of each substep's modes,
    kx planes and physical lines (timing only; never the product library).
    Returns (value in Mpts*RK3-steps/s, seconds per sample, description)."""
    from oracle.ic import make_ic as oracle_ic
    from oracle.oracle import Oracle
    ny = w["y_cpu"]
    y = mesh(ny)
    mgx, mgz = 3 * w["nx"] // 2, 3 * w["nz"] // 2
    st = oracle_ic(mgx, mgz, y, s=w["s"], seed=w["seed"])
    o = Oracle(mgx, mgz, y, w["Re"], 0.25, 0.25, cfl=w["cfl"], ncfl=w["ncfl"], dtmode=w["dt_mode"], dt0=w["dt"],
               nthreads=nth)
    o.set_state(st["vor"], st["phi"], st["psi"], st["scal"], st["u00"], st["v00"], st["w00"])
    if a.scalar:
        o.set_scalar(mixing_scalar(o.shape, y), PR)
    if a.sigma is not None:
        o.set_viscosity(a.sigma)
    del st
    k = 0

    def one():
        nonlocal k
        o.set_sample(stride, k % stride)
        o.substep(k % 3)
        k += 1
    for _ in range(warmup):
        one()
    t0 = time.perf_counter()
    for _ in range(nsamples):
        one()
    dt = time.perf_counter() - t0
    val = mpts(w, ny) * nsamples / (3.0 * stride) / dt
    desc = (f"{nsamples} sample(s), each 1/{stride} of one RK3 substep (every {stride}th mode, kx plane and "
            f"physical line) of the {w['nx']}x{ny}x{w['nz']} case ({ny} of the workload's {w['ny']} y points; "
            f"per-point cost independent of ny), FP64 CPU restatement of cross.f:307-1141 with OpenMP "
            f"({nth} threads), {dt / nsamples:.2f} s per sample")
    return val, dt / nsamples, desc


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = wl(a)
    nth = os.cpu_count() or 1
    val, per, desc = cpu_sample(a, w, w["ref_stride"], nth, a.warmup, a.steps)
    line = {
        "impl": "reference", "metric": "Mpts*RK3-steps/s", "value": val, "unit": "Mpts*RK3-steps/s",
        "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * per,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded initial condition)",
        "config": dict(config(a, w, "FP64 CPU restatement"), sample="each step = one bounded sample (cpu_baseline)"),
        "cpu_baseline": {"value": val, "unit": "Mpts*RK3-steps/s", "cores": nth, "kind": "port",
                         "sample": desc + " (the Fortran reference cannot be compiled here)"},
        "e2e": {"value": val, "unit": "Mpts*RK3-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def make_case(a, w, prec, dev, rank):
    from loma_phd_b200 import ICParams, Lomacte, Params, make_ic, stretched_mesh
    p = Params.from_modes(w["nx"], w["nz"], w["ny"], Re=w["Re"], dt_mode=w["dt_mode"], dt=w["dt"], cfl=w["cfl"],
                          ncfl=w["ncfl"], device=dev, precision=prec, scalar=1 if a.scalar else 0,
                          visc=0 if a.sigma is None else 1, sigma=a.sigma or 0.0)
    y = stretched_mesh(p.my)
    st = make_ic(p, y, ICParams(s=w["s"], seed=w["seed"] + rank))
    g = Lomacte(p, y)
    g.load_state(st)
    z = mixing_scalar(p.shape, y) if a.scalar else None
    if a.scalar:
        g.load_scalar(z)
    return p, y, st, z, g


def run_arm(a, w, prec, dev, rank, world, dist, want_e2e, steps, warmup, stats_cost=True):
    """Warm up, time K steps of one form (prec 0: FP64, 1/2: mixed) with CUDA
    events, then optionally the end-to-end loop through the public API."""
    import torch
    from loma_phd_b200.lomacte import KERNEL_NAMES

    p, y, st, z0, g = make_case(a, w, prec, dev, rank)
    g_launches = g.launches_per_step
    y_family = g.y_family
    stream = torch.cuda.ExternalStream(g.stream, device=dev)

    def barrier():
        if dist is not None:
            dist.barrier()

    for _ in range(warmup):
        g.step(1)
    g.sync()
    clocks = ClockSampler(dev)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    g.profile_start()
    e0.record(stream)
    g.step(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    prof = g.profile_read()
    ck = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), dist, f"cuda:{dev}")
    value = job_throughput(mpts(w), steps, world, ms / 1e3)
    diag = g.diag()
    if not np.isfinite(diag["dm"]) or diag["status"] != 0:
        raise RuntimeError(f"bad diagnostics after the timed steps: {diag}")
    state = g.get_state()
    zf = g.get_scalar() if a.scalar else None

    # end-to-end through the public API with host buffers: every step loads
    # the state (and the scalar) from pinned host memory, advances one RK3
    # step and reads the state back.
    e2e = None
    S, Z, P = sizes(p)
    if want_e2e:
        host = {k: torch.from_numpy(np.ascontiguousarray(st[k]).view(np.float64).copy()).pin_memory()
                for k in ("vor", "phi", "psi", "scal")}
        h00 = {k: torch.from_numpy(np.ascontiguousarray(st[k], dtype=np.float64).copy()).pin_memory()
               for k in ("u00", "v00", "w00")}
        ptrs = [host[k].data_ptr() for k in ("vor", "phi", "psi", "scal")] + \
               [h00[k].data_ptr() for k in ("u00", "v00", "w00")]
        zh = torch.from_numpy(np.ascontiguousarray(z0).view(np.float64).copy()).pin_memory() \
            if a.scalar else None

        def e2e_step():
            g.load_state_ptrs(*ptrs)
            if zh is not None:
                g.load_scalar_ptr(zh.data_ptr())
            g.step(1)
            g.get_state_ptrs(*ptrs)
            if zh is not None:
                g.get_scalar_ptr(zh.data_ptr())

        ne = max(1, min(steps, 3))
        e2e_step()
        barrier()
        t0 = time.perf_counter()
        for _ in range(ne):
            e2e_step()
        el = max_over_ranks(time.perf_counter() - t0, dist, f"cuda:{dev}")
        nbytes = (5 if a.scalar else 4) * S * 16 + 3 * p.my * 8
        e2e = {"value": mpts(w) * ne * world / el, "unit": "Mpts*RK3-steps/s",
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes, "steps": ne}
        del host, h00, zh

    # cost of a statistics step (addstats1/2 and the phys2 sums at the first
    # substep, lmc_stats_step) beside a plain step, CUDA events on the
    # library's stream, best of three each; plain steps replay a CUDA graph,
    # statistics steps enqueue their kernels directly
    # the y operators: banded solves against dense GEMMs on the tensor cores
    # (lmc_yop_tune), on this grid and state
    yop = {f"op{op}": g.yop_tune(op) for op in (1, 2)} if stats_cost else None
    stats_step = None
    if stats_cost:
        def one(fn):
            g.sync()
            s0 = torch.cuda.Event(enable_timing=True)
            s1 = torch.cuda.Event(enable_timing=True)
            s0.record(stream)
            fn(1)
            s1.record(stream)
            torch.cuda.synchronize()
            return s0.elapsed_time(s1)
        g.stats_reset([(p.my + 1) // 2])
        t_plain = min(one(g.step) for _ in range(3))
        t_stats = min(one(g.stats_step) for _ in range(3))
        stats_step = {"plain_step_ms": t_plain, "stats_step_ms": t_stats, "spectra_planes": 1}
    g.close()

    # roofline of the dominant kernel, live CUDA-event times of the timed region
    wb = 16 if prec == 0 else 8
    top = max((k for k in KERNEL_NAMES if k in ALGO), key=lambda k: prof[k][0])
    tot_ms, cnt = prof[top]
    avg_s = tot_ms / max(cnt, 1) / 1e3
    sc, vs = int(a.scalar), int(a.sigma is not None)
    algo = ALGO[top](S, Z, P, wb, sc, vs)
    peak, kind = peaks()
    achieved = algo / avg_s / 1e9
    # fraction of the timed region during which each kernel group runs; the
    # T derivatives and the psi solve run on a second stream beside the main
    # chain, so the fractions can sum above 1
    share = {k: round(prof[k][0] / max(ms, 1e-9), 4) for k in KERNEL_NAMES if prof[k][1]}
    # the same by stage: the plane/line transposes are fused into the
    # transform kernels and the RK3 update into post2 (normalised to the
    # sum of the groups, as the two streams overlap)
    stages = {"fft_and_transposes": ("zinv", "xphys", "zfwd"),
              "y_solves": ("lapv", "assemble", "tder", "post1", "psi"),
              "rhs_and_rk3_update": ("post2",)}
    tot = sum(share.get(k, 0.0) for ks in stages.values() for k in ks)
    stage_share = {n: round(sum(share.get(k, 0.0) for k in ks) / max(tot, 1e-12), 4) for n, ks in stages.items()}
    tr = NCU_TRAFFIC.get((w["name"], prec == 0, sc, vs), {}).get(top)
    traffic = tr[0] * p.my / tr[1] if tr else None
    roofline = {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": kind, "traffic": traffic,
                "traffic_source": f"ncu dram__bytes_read.sum + dram__bytes_write.sum per launch at ny={tr[1]}, "
                                  f"scaled by ny" if tr else None,
                "algo_bytes_per_launch": algo, "avg_launch_ms": avg_s * 1e3}
    step_bytes = 3 * sum(f(S, Z, P, wb, sc, vs) for f in ALGO.values())
    return {"p": p, "ms": ms, "value": value, "clocks": ck, "roofline": roofline,
            "kernel_share": share, "stage_share": stage_share, "e2e": e2e, "state": state, "Z": zf, "diag": diag,
            "step_bytes": step_bytes, "stats_step": stats_step, "yop_autotune": yop,
            "launches_per_step": g_launches, "y_family": y_family,
            "step_roofline_frac": (step_bytes * steps / (ms / 1e3) / 1e9) / peak}


def state_errors(m, r):
    """Relative L2 difference per field of two final states (v00 and w00,
    second-order small, against the size of u00)."""
    out = {}
    for k in ("vor", "phi", "psi", "scal", "u00", "v00", "w00"):
        den = np.linalg.norm(r["state"][k])
        if k in ("v00", "w00"):
            den = max(den, np.linalg.norm(r["state"]["u00"]))
        out[k] = float(np.linalg.norm(np.asarray(m["state"][k]) - np.asarray(r["state"][k])) / den)
    if m.get("Z") is not None and r.get("Z") is not None:
        out["Z"] = float(np.linalg.norm(m["Z"] - r["Z"]) / np.linalg.norm(r["Z"]))
    return out


def error_run(a, dev, nsteps):
    """Both forms advanced nsteps from the same seeded state of the error
    workload: relative L2 per field, the largest relative difference of the
    momentum-thickness history (every 10 steps), the Deltat sequences (CFL
    mode), the simulated time reached and the time per step of each form."""
    import torch
    w = wl(a, a.error_workload)
    res = {}
    every = 10
    for prec in (0, a.mixed_form):
        p, y, st, z0, g = make_case(a, w, prec, dev, 0)
        dm, dts = [], []
        s = torch.cuda.ExternalStream(g.stream, device=dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for n in range(nsteps // every):
            g.step(every)
            dg = g.diag()
            dm.append(dg["dm"])
            dts.append(dg["Deltat"])
        e1.record(s)
        torch.cuda.synchronize()
        res[prec] = {"state": g.get_state(), "Z": g.get_scalar() if a.scalar else None, "dm": np.array(dm),
                     "dt": np.array(dts), "time": g.diag()["time"] + g.diag()["Deltat"],
                     "ms": e0.elapsed_time(e1) / max(1, nsteps // every * every)}
        g.close()
        gc.collect()
    m, r = res[a.mixed_form], res[0]
    dmerr = float(np.abs(m["dm"] - r["dm"]).max() / np.abs(r["dm"]).max()) if len(r["dm"]) else None
    dterr = float(np.abs(m["dt"] - r["dt"]).max() / np.abs(r["dt"]).max()) if len(r["dt"]) else None
    return {"steps": nsteps // every * every, "grid": f"{w['nx']}x{w['ny']}x{w['nz']}", "form": a.mixed_form,
            "workload": w["desc"], "rel_l2": state_errors(m, r), "dm_history_max_rel": dmerr,
            "deltat_history_max_rel": dterr, "time_reached": {"mixed": m["time"], "fp64": r["time"]},
            "dm_final": {"mixed": float(m["dm"][-1]), "fp64": float(r["dm"][-1])} if len(r["dm"]) else None,
            "ms_per_step": {"mixed": m["ms"], "fp64": r["ms"]}, "note": "mixed vs FP64 GPU path, same seeded state"}


def run_serving(a, dev):
    """The synthetic serving stream (Poisson arrivals of 3-D runs of uneven
    sizes) served by continuous batching, once in the mixed form and once in
    FP64; p50/p99 completion latency and aggregate throughput of each."""
    import torch
    from loma_phd_b200.serve import Server, synthetic_stream
    free, _ = torch.cuda.mem_get_info(dev)
    cap = int(min(150e9, 0.8 * free))
    out = {"stream": f"{a.serve_requests} requests, Poisson arrivals at 4/s, half 2-D (nz=1, nx in "
                     f"{{256..1024}}, ny=257), half 3-D (nx=nz in {{64..256}}, ny in {{129,193,257}}), "
                     f"Re~U[100,1000], s~U[1,8], steps log-uniform [200,2000] x "
                     f"{a.serve_scale:g}, HBM cap {cap / 1e9:.0f} GB, 16 slots",
           "unit": "s (latency), Mpts*RK3-steps/s (aggregate)"}
    for name, prec in (("mixed", a.mixed_form), ("fp64", 0)):
        reqs = synthetic_stream(a.serve_requests, seed=7, rate=4.0, steps_scale=a.serve_scale,
                                nx_range=(64, 256), precision=prec, frac_2d=0.5)
        out[name] = Server(cap, max_active=16, chunk=8, device=dev).run(reqs)["stats"]
    return out


def run_ensemble(a, dev):
    """An ensemble of independent cases of uneven grids (nx in {64..192},
    ny in {97, 129, 193}, nz in {64, 96, 128}, seeds 0..n-1), all resident
    at once and advanced concurrently, in the mixed form and in FP64:
    makespan, aggregate throughput and per-case completion latency."""
    import torch
    from loma_phd_b200.serve import Server, ensemble_requests
    free, _ = torch.cuda.mem_get_info(dev)
    cap = int(min(150e9, 0.8 * free))
    out = {"ensemble": f"{a.ensemble} cases, {a.ensemble_steps} RK3 steps each, all at t=0, "
                       f"nx in {{64,96,128,192}} x ny in {{97,129,193}} x nz in {{64,96,128}}, "
                       f"Re~U[100,400], s~U[1,8], seeds 0..{a.ensemble - 1}, {a.ensemble} slots",
           "unit": "s (latency, makespan, set-up), Mpts*RK3-steps/s (aggregate)"}
    for name, prec in (("mixed", a.mixed_form), ("fp64", 0)):
        reqs = ensemble_requests(a.ensemble, a.ensemble_steps, precision=prec)
        st = Server(cap, max_active=a.ensemble, chunk=10, device=dev).run(reqs)["stats"]
        out[name] = {k: st[k] for k in ("makespan_s", "aggregate_mpts_steps_per_s", "p50_latency_s",
                                        "p99_latency_s", "max_concurrent", "peak_device_bytes", "mean_setup_s")}
    return out


def medium_line(a, dev):
    """The medium grid (256^2 x 257) beside the headline: both forms, short."""
    w = wl(a, "medium")
    arms = {prec: run_arm(a, w, prec, dev, 0, 1, None, False, 10, 3, stats_cost=False)
            for prec in (0, a.mixed_form)}
    m, r = arms[a.mixed_form], arms[0]
    out = {"config": config(a, w, MIXED_NAMES[a.mixed_form]), "value": m["value"], "ms_per_step": m["ms"] / 10,
           "fp64": {"value": r["value"], "ms_per_step": r["ms"] / 10, "roofline": r["roofline"]},
           "mixed_over_fp64": m["value"] / r["value"], "roofline": m["roofline"], "clocks": m["clocks"],
           "stage_share": m["stage_share"], "steps": 10, "warmup": 3}
    return out


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
        return
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)
    w = wl(a)

    forms = {"mixed": [a.mixed_form], "fp64": [0], "both": [0, a.mixed_form]}[a.precision]
    arms = {}
    for prec in forms:  # one case on the device at a time
        arms[prec] = run_arm(a, w, prec, dev, rank, world, dist, not a.no_e2e, a.steps, a.warmup)
        gc.collect()
    mixed = a.mixed_form in arms
    head = arms[a.mixed_form] if mixed else arms[0]
    errs = state_errors(arms[a.mixed_form], arms[0]) if (mixed and 0 in arms) else None
    for r in arms.values():
        r.pop("state", None)
        r.pop("Z", None)
    gc.collect()
    medium = None
    if world == 1 and a.workload != "medium" and not a.no_medium:
        medium = medium_line(a, dev)
    err_long = None
    if world == 1 and a.error_steps > 0:
        err_long = error_run(a, dev, a.error_steps)
    serving = None
    if world == 1 and a.serve_requests > 0:
        serving = run_serving(a, dev)
    ensemble = None
    if world == 1 and a.ensemble > 0:
        ensemble = run_ensemble(a, dev)
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        nth = os.cpu_count() or 1
        val, per, desc = cpu_sample(a, w, w["cpu_stride"], nth, 0, 1)
        cpu = {"value": val, "unit": "Mpts*RK3-steps/s", "cores": nth, "kind": "port", "sample": desc}
    if rank == 0:
        p = head["p"]
        form = MIXED_NAMES[a.mixed_form] if mixed else "FP64 plain path"
        line = {
            "metric": "Mpts*RK3-steps/s", "value": head["value"], "unit": "Mpts*RK3-steps/s",
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": head["ms"] / a.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "mixed f32/f64" if mixed else "f64",
            "precision_form": a.mixed_form if mixed else 0,
            "data": "synthetic (seeded initial condition)",
            "config": dict(config(a, w, form), parallelism=f"replicas{world}",
                           l2="inputs larger than L2 (~%.0f GB touched per step)" % (head["step_bytes"] / 1e9),
                           mgal=f"{p.mgalx}x{p.mgalz}"),
            "gpu_launches": head["launches_per_step"] * a.steps,
            "y_kernels": head["y_family"],
            "clocks": head["clocks"], "roofline": head["roofline"], "kernel_share": head["kernel_share"],
            "stage_share": head["stage_share"],
            "step_roofline_frac": head["step_roofline_frac"],
            "e2e": head["e2e"], "cpu_baseline": cpu, "serving": serving, "stats_step": head["stats_step"],
            "yop_autotune": head["yop_autotune"],
            "ensemble": ensemble, "medium_grid": medium, "error_long": err_long,
        }
        if mixed and 0 in arms:
            f64 = arms[0]
            line["fp64"] = {"value": f64["value"], "ms_per_step": f64["ms"] / a.steps, "roofline": f64["roofline"],
                            "kernel_share": f64["kernel_share"], "stage_share": f64["stage_share"],
                            "e2e": f64["e2e"], "clocks": f64["clocks"],
                            "stats_step": f64["stats_step"], "yop_autotune": f64["yop_autotune"]}
            line["mixed_over_fp64"] = head["value"] / f64["value"]
            line["error_vs_fp64"] = {"rel_l2": errs, "steps": a.warmup + a.steps,
                                     "note": "mixed vs FP64 GPU path from the same seeded state (e2e steps "
                                             "restart from it)"}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
