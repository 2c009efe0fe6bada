"""Continuous batching of independent lomacte runs on one GPU.

Runs arrive as requests (grid, Re, density ratio, perturbation amplitude,
seed, steps, precision).  The server admits them while device memory
allows (each case's lmc_footprint against an HBM cap) and a slot is free,
keeps every admitted case resident (one handle, one CUDA stream, one CUDA
graph per RK3 step), and advances all of them concurrently in chunks of
steps, so the kernels of different cases overlap on the GPU.  A finished
case frees its slot and memory at once, and the next waiting request is
admitted while the others keep running.  The host set-up of a case
(initial condition, operator tables, uploads) runs in a worker thread so
that it overlaps the GPU work of the running cases.

The reference runs one case per MPI job and has no counterpart; this layer
sits on the C ABI only (lmc_create / lmc_load_state / lmc_step /
lmc_query / lmc_get_state / lmc_destroy).
"""
from __future__ import annotations

import collections
import dataclasses
import math
import time
from concurrent.futures import ThreadPoolExecutor
from typing import Callable, Dict, List, Optional

import numpy as np

from .lomacte import LMC_ENAN, ICParams, Lomacte, LomacteError, Params, footprint, make_ic, stretched_mesh


@dataclasses.dataclass
class RunRequest:
    rid: int
    nx: int
    nz: int
    ny: int
    steps: int
    Re: float = 160.0
    s: float = 4.0          # density (temperature) ratio T2/T1
    amp: float = 1e-2       # perturbation amplitude
    seed: int = 0
    precision: int = 1
    dt: float = 1e-4        # the initial Deltat of the reference's CFL mode (main.f:559)
    arrival: float = 0.0    # seconds after the start of the stream

    def params(self, device: int = 0) -> Params:
        """Deltat from CFL = 0.5 every 10 steps (the reference's run mode,
        hre.dat CFL / ncfl), so every request is stable whatever its grid and
        Reynolds number."""
        return Params.from_modes(self.nx, self.nz, self.ny, Re=self.Re, dt_mode=0, dt=self.dt, cfl=0.5, ncfl=10,
                                 precision=self.precision, device=device)

    @property
    def mpts(self) -> float:
        return self.nx * self.ny * self.nz / 1e6


@dataclasses.dataclass
class RunResult:
    rid: int
    arrival: float
    admitted: float
    finished: float
    steps: int
    mpts: float
    diag: Dict[str, float]
    state: Optional[dict] = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


@dataclasses.dataclass
class _Active:
    req: RunRequest
    case: Lomacte
    admitted: float
    remaining: int
    bytes: int
    inflight: int = 0
    started: float = 0.0   # set-up done, first steps enqueued


def _prepare(req: RunRequest, device: int) -> Lomacte:
    p = req.params(device)
    y = stretched_mesh(p.my)
    st = make_ic(p, y, ICParams(s=req.s, amp=req.amp, seed=req.seed))
    case = Lomacte(p, y)
    case.load_state(st)
    return case


class Server:
    """One GPU, many resident cases.

    hbm_cap   bytes of device memory the admitted cases may hold together
    max_active  number of cases (slots) resident at once
    chunk     steps enqueued per case between progress checks
    """

    def __init__(self, hbm_cap: int, max_active: int = 16, chunk: int = 8, device: int = 0,
                 keep_state: bool = False, prep_workers: int = 4):
        self.cap = int(hbm_cap)
        self.max_active = max_active
        self.chunk = max(1, chunk)
        self.device = device
        self.keep_state = keep_state
        self.prep_workers = prep_workers

    def run(self, requests: List[RunRequest], clock: Callable[[], float] = time.perf_counter) -> Dict[str, object]:
        for r in requests:
            fp = footprint(r.params(self.device))
            if fp == 0:
                raise ValueError(f"request {r.rid}: unsupported grid {r.nx}x{r.ny}x{r.nz}")
            if fp > self.cap:
                raise ValueError(f"request {r.rid} needs {fp} bytes, more than the cap {self.cap}")
        pending = collections.deque(sorted(requests, key=lambda r: (r.arrival, r.rid)))
        waiting: collections.deque = collections.deque()
        preparing: Dict[int, tuple] = {}
        active: Dict[int, _Active] = {}
        results: List[RunResult] = []
        used = 0
        peak_used = 0
        max_conc = 0
        diverged = 0
        setup: List[float] = []
        pool = ThreadPoolExecutor(max_workers=self.prep_workers)
        t0 = clock()
        try:
            while pending or waiting or preparing or active:
                now = clock() - t0
                while pending and pending[0].arrival <= now:
                    waiting.append(pending.popleft())
                # admission: first come first served, by memory and slots
                while waiting and len(active) + len(preparing) < self.max_active:
                    r = waiting[0]
                    fp = footprint(r.params(self.device))
                    if used + fp > self.cap:
                        break
                    waiting.popleft()
                    used += fp
                    peak_used = max(peak_used, used)
                    preparing[r.rid] = (r, fp, now, pool.submit(_prepare, r, self.device))
                progressed = False
                for rid in list(preparing):
                    r, fp, t_adm, fut = preparing[rid]
                    if fut.done():
                        case = fut.result()
                        del preparing[rid]
                        a = _Active(r, case, t_adm, r.steps, fp, started=clock() - t0)
                        setup.append(a.started - t_adm)
                        active[rid] = a
                        self._enqueue(a)
                        progressed = True
                max_conc = max(max_conc, len(active))
                for rid in list(active):
                    a = active[rid]
                    if not a.case.done():
                        continue
                    progressed = True
                    a.remaining -= a.inflight
                    a.inflight = 0
                    if a.remaining > 0:
                        self._enqueue(a)
                        continue
                    try:
                        d = a.case.diag()
                    except LomacteError as e:  # a run that went non-finite ends, reported
                        if e.code != LMC_ENAN:
                            raise
                        d = {"status": e.code}
                        diverged += 1
                    st = a.case.get_state() if self.keep_state else None
                    fin = clock() - t0
                    results.append(RunResult(rid, a.req.arrival, a.admitted, fin, a.req.steps, a.req.mpts, d, st))
                    used -= a.bytes
                    a.case.close()
                    del active[rid]
                if not progressed:
                    time.sleep(2e-4)
        finally:
            for a in active.values():
                a.case.close()
            pool.shutdown(wait=True)
        makespan = clock() - t0
        lat = np.array([r.latency for r in results])
        work = sum(r.mpts * r.steps for r in results)
        stats = {
            "requests": len(results),
            "makespan_s": makespan,
            "p50_latency_s": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_latency_s": float(np.percentile(lat, 99)) if len(lat) else None,
            "mean_latency_s": float(lat.mean()) if len(lat) else None,
            "aggregate_mpts_steps_per_s": work / makespan if makespan > 0 else None,
            "peak_device_bytes": peak_used,
            "max_concurrent": max_conc,
            "mean_setup_s": float(np.mean(setup)) if setup else None,
            "diverged": diverged,
        }
        return {"results": sorted(results, key=lambda r: r.rid), "stats": stats}

    def _enqueue(self, a: _Active) -> None:
        n = min(self.chunk, a.remaining)
        a.case.step(n)
        a.inflight = n


# supported grid sizes of the stream generator: nx = 2/3 mgal with mgal a
# transform length of the library
_MODES = (64, 96, 128, 192, 256, 384)


# x mode counts of 2-D requests (nx = 2/3 mgalx, mgalx from 384 to 1536)
_MODES_2D = (256, 384, 512, 768, 1024)


def synthetic_stream(n: int, seed: int = 0, rate: float = 2.0, steps_range=(200, 2000), steps_scale: float = 1.0,
                     nx_range=(64, 384), ny_choices=(129, 193, 257), precision: int = 1,
                     frac_2d: float = 0.0, nx2d_range=(256, 1024)) -> List[RunRequest]:
    """Poisson arrivals of runs: 3-D with nx = nz drawn from the supported
    sizes in nx_range and ny from ny_choices, or, with probability frac_2d,
    2-D (nz = 1) with nx from nx2d_range and ny = 257; Re ~ U[100, 1000],
    s ~ U[1, 8], steps log-uniform in steps_range (times steps_scale),
    amplitude ~ U[5e-3, 2e-2]."""
    rng = np.random.default_rng(seed)
    modes = [m for m in _MODES if nx_range[0] <= m <= nx_range[1]]
    modes2 = [m for m in _MODES_2D if nx2d_range[0] <= m <= nx2d_range[1]]
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        two_d = frac_2d > 0 and rng.uniform() < frac_2d
        if two_d:
            nx, nz, ny = int(rng.choice(modes2)), 1, 257
        else:
            nx = int(rng.choice(modes))
            nz, ny = nx, int(rng.choice(ny_choices))
        lo, hi = math.log(steps_range[0]), math.log(steps_range[1])
        steps = max(1, int(round(math.exp(rng.uniform(lo, hi)) * steps_scale)))
        out.append(RunRequest(rid=i, nx=nx, nz=nz, ny=ny, steps=steps, Re=float(rng.uniform(100, 1000)),
                              s=float(rng.uniform(1.0, 8.0)), amp=float(rng.uniform(5e-3, 2e-2)),
                              seed=int(rng.integers(0, 2**31 - 1)), precision=precision, arrival=t))
    return out


def ensemble_requests(n: int = 48, steps: int = 500, precision: int = 1, seed: int = 0) -> List[RunRequest]:
    """An ensemble of n independent cases, all present at t = 0, seeds 0 ..
    n-1: grids drawn uniformly from nx in {64, 96, 128, 192}, ny in {97,
    129, 193}, nz in {64, 96, 128}; Re ~ U[100, 400], s ~ U[1, 8],
    amplitude ~ U[5e-3, 2e-2]; the same number of steps each."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        nx = int(rng.choice((64, 96, 128, 192)))
        ny = int(rng.choice((97, 129, 193)))
        nz = int(rng.choice((64, 96, 128)))
        out.append(RunRequest(rid=i, nx=nx, nz=nz, ny=ny, steps=steps, Re=float(rng.uniform(100, 400)),
                              s=float(rng.uniform(1.0, 8.0)), amp=float(rng.uniform(5e-3, 2e-2)), seed=i,
                              precision=precision, arrival=0.0))
    return out
