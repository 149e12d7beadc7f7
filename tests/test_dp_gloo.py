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
