"""Slab decomposition plumbing on the CPU (loma_phd_b200/slab.py): the
blocks of pointers_calc (trunk/lomacte3/src/change.f:145-211) and the
plane <-> line exchanges of chpl2ln / chln2pl (change.f:1-143) as one
all-to-all each, run as 2 and 3 gloo ranks: every rank's line block equals
the same lines of the whole field, and the way back restores its plane
block bit for bit.  The device substep does not split over ranks (the
graded cases fit one GPU)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from loma_phd_b200.slab import SlabPlan, split


def test_blocks_of_pointers_calc():
    assert split(10, 4) == [(0, 3), (3, 6), (6, 8), (8, 10)]
    assert split(8, 4) == [(0, 2), (2, 4), (4, 6), (6, 8)]
    p = SlabPlan(nplanes=128, mgalz=384, my=257, nranks=8, strict=True)
    assert p.planes(7) == (112, 128) and p.lines(0) == (0, 12336)
    assert sum(e - b for b, e in (p.lines(r) for r in range(8))) == 384 * 257
    assert p.exchange_bytes(0) == (384 * 257 - 12336) * 16 * 16
    with pytest.raises(ValueError):
        SlabPlan(nplanes=12, mgalz=36, my=33, nranks=5, strict=True)
    with pytest.raises(ValueError):
        split(3, 4)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q, nplanes, mgalz, my):
    import torch
    import torch.distributed as dist

    from loma_phd_b200.slab import SlabPlan, lines_to_planes, planes_to_lines
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    plan = SlabPlan(nplanes=nplanes, mgalz=mgalz, my=my, nranks=world)
    rng = np.random.default_rng(5)
    whole = rng.standard_normal((mgalz * my, nplanes)) + 1j * rng.standard_normal((mgalz * my, nplanes))
    pb, pe = plan.planes(rank)
    lb, le = plan.lines(rank)
    mine = torch.from_numpy(np.ascontiguousarray(whole[:, pb:pe]))
    lines = planes_to_lines(mine, plan, rank)
    ok_lines = bool(np.array_equal(lines.numpy(), whole[lb:le, :]))
    back = lines_to_planes(lines, plan, rank)
    ok_back = bool(np.array_equal(back.numpy(), whole[:, pb:pe]))
    dist.barrier()
    q.put((rank, ok_lines, ok_back))
    dist.destroy_process_group()


@pytest.mark.parametrize("world,nplanes", [(2, 12), (3, 10)])
def test_exchange_gloo(world, nplanes):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q, nplanes, 36, 33)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[0] for o in out] == list(range(world))
    assert all(o[1] and o[2] for o in out), out


def _transform_rank(rank, world, port, q):
    """One rank of a slab-split inverse transform of T: z transforms of its
    kx planes, the plane -> line exchange, x transforms of its lines (numpy
    stands in for the device transforms); its lines of T against the
    oracle's physical T of the whole state."""
    import torch
    import torch.distributed as dist

    from loma_phd_b200.slab import SlabPlan, planes_to_lines
    from tests.helpers import case, oracle_for
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    p, y, st = case(24, 24, 33)
    o = oracle_for(p, y, st, nthreads=1)
    T = o.get_state()["scal"]                                   # [kx][kz][y]
    nkx, mz, my = T.shape
    plan = SlabPlan(nplanes=nkx, mgalz=p.mgalz, my=my, nranks=world)
    pb, pe = plan.planes(rank)
    nz1 = (mz - 1) // 2
    pad = np.zeros((pe - pb, p.mgalz, my), dtype=complex)       # kz padded (localyz2zy)
    for k in range(mz):
        pad[:, k if k <= nz1 else k + p.mgalz - mz, :] = T[pb:pe, k, :]
    zphys = np.fft.ifft(pad, axis=1) * p.mgalz                  # e^{+i kz z}
    block = np.ascontiguousarray(zphys.transpose(2, 1, 0).reshape(my * p.mgalz, pe - pb))  # [line][kx]
    lines = planes_to_lines(torch.from_numpy(block), plan, rank).numpy()
    lines[:, 0] = lines[:, 0].real                              # Im of mode 0 dropped (rftsingle.f:85-88)
    full = np.zeros((lines.shape[0], p.mgalx), dtype=complex)
    full[:, :nkx] = lines
    full[:, p.mgalx - nkx + 1:] = np.conj(lines[:, 1:][:, ::-1])
    phys = np.real(np.fft.ifft(full, axis=1)) * p.mgalx
    lb, le = plan.lines(rank)
    ref = o.physical(list(range(1, my + 1)))[:, 3]              # T [y][z][x]
    want = ref.reshape(my * p.mgalz, p.mgalx)[lb:le]
    err = float(np.abs(phys - want).max() / np.abs(want).max())
    dist.barrier()
    q.put((rank, err))
    dist.destroy_process_group()


def test_split_inverse_transform_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_transform_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(e < 1e-13 for _, e in out), out
