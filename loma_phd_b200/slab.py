"""Slab decomposition of one case over several ranks: the host plumbing of
the reference's only parallel strategy (trunk/lomacte3/src/change.f,
main.f:76-118).

In the spectral phase each rank owns a contiguous block of kx planes (all
y, all kz); in the physical phase a contiguous block of lines (z, y) with
all kx.  Between the two, every field crosses the ranks once: the
plane -> line exchange after the inverse z transforms (chpl2ln,
change.f:1-72) and the line -> plane exchange before the direct ones
(chln2pl, change.f:74-143).  The reference pairs ranks by XOR and sends one
plane at a time; here each exchange is one all-to-all over the process
group (NCCL over NVLink for device tensors, gloo on the CPU) with the
blocks of pointers_calc (change.f:145-211).

Layout of a z-padded field, as the library stores it on one device:
[line][kx] with line = y * mgalz + z and kx fastest.  A rank's plane block
is [nlines][pe - pb] (its kx planes, kx fastest); its line block is
[le - lb][nplanes].
"""
from __future__ import annotations

import dataclasses
from typing import List, Tuple


def split(n: int, k: int) -> List[Tuple[int, int]]:
    """Contiguous blocks [b, e) of n items over k ranks, the first n mod k
    ranks one item longer (pointers_calc, change.f:158-169, 0-based)."""
    if k < 1 or n < k:
        raise ValueError(f"cannot split {n} items over {k} ranks")
    n1, n2 = divmod(n, k)
    out, b = [], 0
    for r in range(k):
        e = b + n1 + (1 if r < n2 else 0)
        out.append((b, e))
        b = e
    return out


@dataclasses.dataclass(frozen=True)
class SlabPlan:
    """Plane and line blocks of nranks compute ranks.  strict = True keeps
    the reference's rule that the planes divide evenly (main.f:114-118)."""
    nplanes: int
    mgalz: int
    my: int
    nranks: int
    strict: bool = False

    def __post_init__(self):
        if self.strict and self.nplanes % self.nranks:
            raise ValueError(f"the number of planes {self.nplanes} must be a multiple of the ranks {self.nranks}")
        split(self.nplanes, self.nranks)
        split(self.nlines, self.nranks)

    @property
    def nlines(self) -> int:
        return self.mgalz * self.my

    def planes(self, rank: int) -> Tuple[int, int]:
        return split(self.nplanes, self.nranks)[rank]

    def lines(self, rank: int) -> Tuple[int, int]:
        return split(self.nlines, self.nranks)[rank]

    def exchange_bytes(self, rank: int, itemsize: int = 16) -> int:
        """Bytes rank sends in one exchange of one field (to the other ranks)."""
        pb, pe = self.planes(rank)
        lb, le = self.lines(rank)
        return (self.nlines - (le - lb)) * (pe - pb) * itemsize


def _real(t):
    import torch
    return torch.view_as_real(t) if t.is_complex() else t


def planes_to_lines(block, plan: SlabPlan, rank: int, group=None):
    """chpl2ln: this rank's plane block [nlines][np] -> its line block
    [nl][nplanes], by one all-to-all."""
    import torch
    import torch.distributed as dist
    pb, pe = plan.planes(rank)
    lb, le = plan.lines(rank)
    if tuple(block.shape) != (plan.nlines, pe - pb):
        raise ValueError("plane block of the wrong shape")
    lines = [plan.lines(s) for s in range(plan.nranks)]
    planes = [plan.planes(s) for s in range(plan.nranks)]
    # rows of the plane block are lines: the chunk for rank s is its lines
    send = _real(block.contiguous())
    w = 2 if block.is_complex() else 1
    in_split = [(e - b) * (pe - pb) * w for b, e in lines]
    out_split = [(le - lb) * (e - b) * w for b, e in planes]
    recv = torch.empty(sum(out_split), dtype=send.dtype, device=send.device)
    dist.all_to_all_single(recv, send.reshape(-1), out_split, in_split, group=group)
    out = torch.empty((le - lb, plan.nplanes), dtype=block.dtype, device=block.device)
    o = 0
    for (b, e), n in zip(planes, out_split):
        chunk = recv[o:o + n]
        o += n
        if block.is_complex():
            chunk = torch.view_as_complex(chunk.reshape(-1, 2))
        out[:, b:e] = chunk.reshape(le - lb, e - b)
    return out


def lines_to_planes(block, plan: SlabPlan, rank: int, group=None):
    """chln2pl: this rank's line block [nl][nplanes] -> its plane block
    [nlines][np], by one all-to-all."""
    import torch
    import torch.distributed as dist
    pb, pe = plan.planes(rank)
    lb, le = plan.lines(rank)
    if tuple(block.shape) != (le - lb, plan.nplanes):
        raise ValueError("line block of the wrong shape")
    lines = [plan.lines(s) for s in range(plan.nranks)]
    planes = [plan.planes(s) for s in range(plan.nranks)]
    w = 2 if block.is_complex() else 1
    send = torch.cat([_real(block[:, b:e].contiguous()).reshape(-1) for b, e in planes])
    in_split = [(le - lb) * (e - b) * w for b, e in planes]
    out_split = [(e - b) * (pe - pb) * w for b, e in lines]
    recv = torch.empty(sum(out_split), dtype=send.dtype, device=send.device)
    dist.all_to_all_single(recv, send, out_split, in_split, group=group)
    if block.is_complex():
        recv = torch.view_as_complex(recv.reshape(-1, 2))
    return recv.reshape(plan.nlines, pe - pb)
