"""The multi-rank step on CPU: two gloo ranks each carry half of the points
and sum dL/dw and the loss with one all-reduce; the result must equal the
single-process gradient over all points.  The per-rank gradient comes from
the oracle here (no GPU); on a B200 the same ReducedStep wraps the device
entry dnnf90_grad_rule_dev and the all-reduce runs over NCCL."""
import multiprocessing as mp
import os
import socket
import sys

import numpy as np
import pytest

from conftest import ROOT, rel_err, xavier_weights

from dnnf90_b200.dp import shard

D0, K, DIMS, NPTS = 4, 3, [4, 16, 16, 1], 301


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _terms(tab):
    return [(1.0, tab.slot((1, 0, 0, 0)), 0), (0.5, tab.slot((0, 2, 0, 0)), 0),
            (1.0, tab.slot((0, 1, 0, 0)), 1)]


def _rank_main(rank, world, port, X, w, out_q):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch
    import torch.distributed as dist
    import pyoracle as po
    from dnnf90_b200.dp import ReducedStep, shard

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        tab = po.Tables(D0, K)
        a, b = shard(len(X), rank, world)
        step = ReducedStep(po.weight_count(DIMS), "cpu")

        def local(grad, loss):
            g, _, L, _ = po.grad_batch(tab, DIMS, w, X[a:b], kind=po.SEED_PINN,
                                       terms=_terms(tab), want_t=False)
            grad += torch.from_numpy(g)
            loss += L

        for _ in range(2):  # the buffer is reused: a second step gives the same sums
            g, L = step.step(local)
        if rank == 0:
            out_q.put((g.numpy().copy(), float(L)))
    finally:
        dist.destroy_process_group()


def test_shard_covers_every_point_once():
    for n in (0, 1, 7, 301, 65536):
        for world in (1, 2, 3, 8):
            ranges = [shard(n, r, world) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == n
            for (a0, b0), (a1, b1) in zip(ranges, ranges[1:]):
                assert b0 == a1 and b0 >= a0
            sizes = [b - a for a, b in ranges]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard(10, 2, 2)


def test_two_gloo_ranks_sum_to_the_full_gradient():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po

    X = np.random.default_rng(1).uniform(-1, 1, (NPTS, D0))
    w = xavier_weights(DIMS, 4)
    tab = po.Tables(D0, K)
    gref, _, Lref, _ = po.grad_batch(tab, DIMS, w, X, kind=po.SEED_PINN, terms=_terms(tab),
                                     want_t=False)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, X, w, q)) for r in range(2)]
    for p in procs:
        p.start()
    g, L = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert rel_err(g, gref) < 1e-13
    assert abs(L - Lref) <= 1e-13 * abs(Lref)


# ------------------------------------------------ sharded natural gradient


class _CpuNGD:
    """The device halves restated in numpy (CPU ranks have no device)."""

    def gram(self, rows, G):
        J = rows.numpy()
        G.copy_(__import__("torch").from_numpy(np.tril(J.T @ J)))

    def solve(self, G, b, nb, mu, u):
        L = np.tril(G.numpy())
        A = L + np.tril(L, -1).T
        u.copy_(__import__("torch").from_numpy(
            np.linalg.solve(A / nb + mu * np.eye(len(b)), b.numpy() / nb)))

    def dual(self, rows, b, nb, mu, u):
        J, bb = rows.numpy(), b.numpy() / nb
        K = mu * np.eye(len(J)) + J @ J.T / nb
        y = np.linalg.solve(K, J @ bb)
        u.copy_(__import__("torch").from_numpy((bb - J.T @ y / nb) / mu))


def _ngd_rank(rank, world, port, J, B, splits, out_q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch
    import torch.distributed as dist
    from dnnf90_b200.dp import ngd_step_sharded

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        a, c = splits[rank], splits[rank + 1]
        rows = torch.from_numpy(J[a:c].copy())
        b = torch.from_numpy(B[rank].copy())
        out = {}
        for route in ("primal", "dual"):
            out[route] = ngd_step_sharded(rows, b, 1e-3, route=route, ops=_CpuNGD()).numpy()
        out_q.put((rank, out))
    finally:
        dist.destroy_process_group()


def test_sharded_natural_gradient_over_two_gloo_ranks():
    """Rows split 9 : 4 over two ranks (the shares need not be equal): both
    routes give the single-process step over all rows, on every rank."""
    rng = np.random.default_rng(3)
    nw, nrow = 20, 13
    J = rng.normal(size=(nrow, nw))
    B = rng.normal(size=(2, nw))
    mu = 1e-3
    G = J.T @ J / nrow + mu * np.eye(nw)
    uref = np.linalg.solve(G, B.sum(axis=0) / nrow)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_ngd_rank, args=(r, 2, port, J, B, [0, 9, 13], q))
             for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in (0, 1):
        for route in ("primal", "dual"):
            assert rel_err(res[r][route], uref) < 1e-10, (r, route)
