"""Continuous batching (loma_phd_b200.serve) and the serving helpers of the
C ABI: CUDA-graph step replay, lmc_query, lmc_footprint.

Bars:
  * graph replay of a step gives the same state as enqueueing its kernels
    (bit-identical in FP64; mixed form within 1e-12: its FP64 plane sums
    use atomics whose order may change)
  * a run gives the same result alone and in the mix of concurrent runs
    (FP64: bit-identical; mixed: relative L2 <= 1e-10)
  * admission never lets the resident cases exceed the HBM cap
"""
import numpy as np
import pytest

from loma_phd_b200 import Lomacte, footprint
from loma_phd_b200.serve import RunRequest, Server, ensemble_requests, synthetic_stream
from tests.helpers import FIELDS, case, rel_l2


def test_stream_with_2d_requests():
    a = synthetic_stream(40, seed=5, frac_2d=0.5)
    two = [r for r in a if r.nz == 1]
    assert 5 < len(two) < 35
    assert all(r.ny == 257 and r.nx in (256, 384, 512, 768, 1024) for r in two)
    assert all(footprint(r.params()) > 0 for r in a)
    assert all(r.params().mgalz == 3 for r in two)


def test_ensemble_requests():
    e = ensemble_requests(48, 500, precision=0)
    assert [r.seed for r in e] == list(range(48)) and all(r.arrival == 0.0 and r.steps == 500 for r in e)
    assert all(r.nx in (64, 96, 128, 192) and r.ny in (97, 129, 193) and r.nz in (64, 96, 128) for r in e)
    assert len({(r.nx, r.ny, r.nz) for r in e}) > 10  # uneven grids
    assert all(footprint(r.params()) > 0 for r in e)


def test_stream_generator_and_footprint():
    a = synthetic_stream(12, seed=3, steps_scale=0.05)
    b = synthetic_stream(12, seed=3, steps_scale=0.05)
    assert [(r.nx, r.ny, r.steps, r.seed) for r in a] == [(r.nx, r.ny, r.steps, r.seed) for r in b]
    assert all(x.arrival < y.arrival for x, y in zip(a, a[1:]))
    for r in a:
        assert r.nx == r.nz and r.ny in (129, 193, 257) and 10 <= r.steps <= 100
        assert footprint(r.params()) > 0
    small = footprint(RunRequest(0, 64, 64, 129, 1).params())
    big = footprint(RunRequest(0, 128, 128, 129, 1).params())
    f64 = footprint(RunRequest(0, 128, 128, 129, 1, precision=0).params())
    assert 3 * small < big < f64
    assert footprint(RunRequest(0, 50, 50, 129, 1).params()) == 0  # no transform of that length


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [0, 1])
def test_graph_replay_matches_direct(gpu, prec):
    p, y, st = case(32, 32, 65, precision=prec)
    out = []
    for graphs in (False, True):
        g = Lomacte(p, y)
        g.use_graphs(graphs)
        g.load_state(st)
        g.step(7)
        out.append((g.get_state(), g.diag()))
        assert abs(g.device_bytes - footprint(p)) <= 0.02 * footprint(p)
        g.close()
    for k in FIELDS:
        if prec == 0:
            assert np.array_equal(out[0][0][k], out[1][0][k]), k
        else:
            assert rel_l2(out[1][0][k], out[0][0][k]) < 1e-12, k
    assert out[0][1]["time"] == out[1][1]["time"]


def _requests(prec):
    grids = [(64, 129), (96, 97), (64, 65), (128, 129)]
    # long enough (>= 150 steps) that a case is still running when the
    # next one has been prepared, so the mix really overlaps
    return [RunRequest(rid=i, nx=nx, nz=nx, ny=ny, steps=150 + 30 * i, Re=150.0 + 50 * i, s=2.0 + i,
                       seed=100 + i, precision=prec, arrival=0.0) for i, (nx, ny) in enumerate(grids)]


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [0, 1])
def test_same_result_alone_and_in_the_mix(gpu, prec):
    reqs = _requests(prec)
    cap = 8 * max(footprint(r.params()) for r in reqs)
    alone = {}
    for r in reqs:
        res = Server(cap, max_active=1, chunk=5, keep_state=True).run([r])
        alone[r.rid] = res["results"][0]
    mix = Server(cap, max_active=4, chunk=5, keep_state=True).run(reqs)
    assert mix["stats"]["max_concurrent"] >= 2
    for m in mix["results"]:
        a = alone[m.rid]
        assert m.diag["time"] == a.diag["time"]
        for k in FIELDS:
            if prec == 0:
                assert np.array_equal(m.state[k], a.state[k]), (m.rid, k)
            else:
                assert rel_l2(m.state[k], a.state[k]) <= 1e-10, (m.rid, k)


@pytest.mark.gpu
def test_admission_respects_the_cap(gpu):
    reqs = synthetic_stream(8, seed=1, rate=50.0, steps_scale=0.02, nx_range=(64, 128), ny_choices=(129,))
    cap = 2 * max(footprint(r.params()) for r in reqs)
    out = Server(cap, max_active=8, chunk=4).run(reqs)
    st = out["stats"]
    assert st["requests"] == len(reqs)
    assert st["peak_device_bytes"] <= cap
    assert st["p99_latency_s"] >= st["p50_latency_s"] > 0
    assert all(np.isfinite(r.diag["dm"]) for r in out["results"])
