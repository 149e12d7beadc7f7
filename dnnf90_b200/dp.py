"""Data parallelism over collocation points.

Points are independent through the whole forward and adjoint
(lib/train_module.f90:198-204), so each rank (one process per GPU) carries
its own points; the one exchange of a step is the sum of dL/dw and of the
loss over ranks -- the reference's replicated-step sum
(app/parallel_module.f90:91-104).  The gradient and the loss share one
contiguous FP64 buffer, so a step issues a single all-reduce.
"""
from __future__ import annotations


def shard(npts: int, rank: int, world: int):
    """Contiguous point range [start, stop) of rank; the first npts % world
    ranks take one point more."""
    if world < 1 or not 0 <= rank < world or npts < 0:
        raise ValueError(f"bad shard request npts={npts} rank={rank} world={world}")
    base, extra = divmod(npts, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


class ReducedStep:
    """One buffer [nw + 1] of FP64: grad = buf[:nw], loss = buf[nw:].

    ``step(local)`` zeroes the buffer, lets ``local(grad, loss)`` add this
    rank's contribution, and sums the buffer over the process group (when
    there is more than one rank).  Every rank must call it the same number
    of times, in the same order.
    """

    def __init__(self, nw: int, device, group=None):
        import torch
        import torch.distributed as dist

        self.nw = int(nw)
        self.buf = torch.zeros(self.nw + 1, dtype=torch.float64, device=device)
        self.grad = self.buf[: self.nw]
        self.loss = self.buf[self.nw:]
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1

    def step(self, local):
        import torch.distributed as dist

        self.buf.zero_()
        local(self.grad, self.loss)
        if self.world > 1:
            dist.all_reduce(self.buf, group=self.group)
        return self.grad, self.loss
