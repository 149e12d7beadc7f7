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


class DeviceNGD:
    """The device halves of the natural-gradient step on torch CUDA
    tensors (dnnf90_ngd_gram_dev, dnnf90_ngd_solve_dev,
    dnnf90_ngd_step_dual_dev), on the current stream."""

    def __init__(self, prec: int = 0):
        self.prec = int(prec)

    @staticmethod
    def _st(t):
        import torch
        return torch.cuda.current_stream(t.device).cuda_stream

    def gram(self, rows, G):
        from . import api
        api.call("dnnf90_ngd_gram_dev", rows.shape[0], rows.shape[1], rows.data_ptr(),
                 self.prec, G.data_ptr(), self._st(rows))

    def solve(self, G, b, nb, mu, u):
        from . import api
        api.call("dnnf90_ngd_solve_dev", b.shape[0], G.data_ptr(), b.data_ptr(), int(nb),
                 float(mu), u.data_ptr(), self._st(b))

    def dual(self, rows, b, nb, mu, u):
        from . import api
        api.call("dnnf90_ngd_step_dual_dev", rows.shape[0], rows.shape[1], rows.data_ptr(),
                 b.data_ptr(), int(nb), float(mu), u.data_ptr(), self._st(b))


def ngd_step_sharded(rows, b, mu: float, nb: int | None = None, route: str = "primal",
                     ops=None, group=None):
    """Damped Gauss-Newton step u = (J^T J / nb + mu I)^{-1} (b / nb) when
    the residual rows J are spread over the ranks (app/optimizer_module.f90:
    299-321 with app/parallel_module.f90:89-152).

    rows: this rank's rows [nloc][nw]; b: this rank's share of the gradient
    sum [nw] (b is a sum over the batch, so it is summed over the ranks);
    nb: the normaliser (default: the total row count).  Every rank returns
    the same u.

    route "primal": each rank forms its own J^T J; one all-reduce sums the
    metrics and the gradients (one buffer), then every rank solves.
    route "dual": the rows are gathered from every rank in rank order (the
    shares may differ by any amount), b is summed, and every rank solves the
    nrow x nrow Gram system.
    ops: the device halves (default DeviceNGD()); any object with the same
    gram / solve / dual methods on the tensors' device.
    """
    import torch
    import torch.distributed as dist

    if route not in ("primal", "dual"):
        raise ValueError(f"route must be 'primal' or 'dual', not {route!r}")
    ops = ops or DeviceNGD()
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    dev = rows.device
    # the device entries read rows with stride nw: views are copied first
    rows = rows.contiguous()
    b = b.contiguous()
    nloc, nw = rows.shape
    if world > 1:
        cnt = torch.tensor([nloc], dtype=torch.int64, device=dev)
        counts = [torch.zeros_like(cnt) for _ in range(world)]
        dist.all_gather(counts, cnt, group=group)
        counts = [int(c.item()) for c in counts]
    else:
        counts = [nloc]
    ntot = sum(counts)
    nb = ntot if nb is None else int(nb)
    u = torch.empty(nw, dtype=torch.float64, device=dev)
    if route == "primal":
        buf = torch.zeros(nw * nw + nw, dtype=torch.float64, device=dev)
        G, bsum = buf[: nw * nw].view(nw, nw), buf[nw * nw:]
        if nloc:
            ops.gram(rows, G)
        bsum.copy_(b)
        if world > 1:
            dist.all_reduce(buf, group=group)
        ops.solve(G, bsum, nb, mu, u)
        return u
    bsum = b.clone()
    if world > 1:
        dist.all_reduce(bsum, group=group)
        mx = max(counts)
        pad = torch.zeros(mx, nw, dtype=torch.float64, device=dev)
        pad[:nloc] = rows
        parts = [torch.empty_like(pad) for _ in range(world)]
        dist.all_gather(parts, pad, group=group)
        allrows = torch.cat([p[:c] for p, c in zip(parts, counts)]).contiguous()
    else:
        allrows = rows.contiguous()
    ops.dual(allrows, bsum, nb, mu, u)
    return u
