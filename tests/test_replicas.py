"""The N>1 bench path on the CPU: two gloo ranks, each with its own case
seed, reduce their timed lengths to the maximum over ranks and report the
whole job's throughput (loma_phd_b200/replicas.py, used by bench.py)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from loma_phd_b200.replicas import case_seed, job_throughput, max_over_ranks


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = [12.5, 17.25][rank]  # rank 1 is the slower replica
    t = max_over_ranks(ms, dist, "cpu")
    dist.barrier()
    q.put((rank, case_seed(rank), t, job_throughput(16.0, 10, world, t / 1e3)))
    dist.destroy_process_group()


def test_two_replicas_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [0, 1]                  # independent cases
    assert all(o[2] == 17.25 for o in out)                # max over ranks on every rank
    assert out[0][3] == pytest.approx(16.0 * 10 * 2 / 0.01725)


def test_single_rank_without_group():
    assert max_over_ranks(3.5) == 3.5
    assert job_throughput(2.0, 5, 1, 0.5) == 20.0
