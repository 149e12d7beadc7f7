"""A committee step: independent networks of uneven width, depth, carried
set and point count trained in one CUDA graph (dnnf90_committee_step), each
member's gradient and loss checked against the oracle, on the first call
(which builds and times the graphs), on a replay, and on a replay after one
member's weights changed."""
import numpy as np
import pytest

from conftest import rel_err, xavier_weights
from dnnf90_b200 import api
import pyoracle as po

pytestmark = pytest.mark.gpu

# (d0, K, dims, points, precision)
MEMBERS = [
    (2, 2, [2, 32, 1], 1000, api.PREC_SPLIT),
    (3, 4, [3, 64, 64, 1], 3000, api.PREC_SPLIT),
    (4, 7, [4, 32, 32, 32, 1], 400, api.PREC_SPLIT),
    (2, 5, [2, 128, 128, 1], 2000, api.PREC_SPLIT),
    (4, 3, [4, 256, 1], 1500, api.PREC_SPLIT),
    (3, 6, [3, 64, 64, 64, 1], 700, api.PREC_F64),
]


def test_committee_step_matches_the_oracle():
    import torch
    dev = torch.device("cuda", 0)
    rule = api.SeedRule(api.SEED_HALFSQ)
    nets, xs, ws, Xs, tabs = [], [], [], [], []
    for i, (d0, k, dims, npts, prec) in enumerate(MEMBERS):
        ts = api.TableSet(d0, k)
        w = xavier_weights(dims, 30 + i)
        w[np.arange(len(w)) % 5 == 0] += 0.02
        nets.append(api.Net(ts, dims, weights=w, precision=prec))
        X = np.random.default_rng(40 + i).uniform(-1, 1, (npts, d0))
        Xs.append(X)
        xs.append(torch.tensor(X, device=dev))
        ws.append(w)
        tabs.append(po.Tables(d0, k))
    grads = [torch.full((m.nw,), float("nan"), dtype=torch.float64, device=dev) for m in nets]
    loss = torch.full((len(nets),), float("nan"), dtype=torch.float64, device=dev)

    def check():
        for i, (d0, k, dims, npts, prec) in enumerate(MEMBERS):
            gref, _, lref, _ = po.grad_batch(tabs[i], dims, ws[i], Xs[i], kind=po.SEED_HALFSQ,
                                             want_t=False)
            tol = 1e-12 if prec == api.PREC_F64 else 1e-5
            g = grads[i].cpu().numpy()
            assert rel_err(g, gref) < tol, (i, rel_err(g, gref))
            assert abs(float(loss[i]) - lref) <= tol * abs(lref), (i, float(loss[i]), lref)

    pol, ms = api.committee_step(nets, [rule] * len(nets), xs, grads, loss)
    assert pol in (0, 1, 2) and ms > 0
    check()
    api.committee_step(nets, [rule] * len(nets), xs, grads, loss)  # replay
    check()
    ws[1] = ws[1] * 0.9 + 0.01
    nets[1].set_weights(ws[1])
    api.committee_step(nets, [rule] * len(nets), xs, grads, loss)  # replay, new weights
    check()
    for m in nets:
        m.free()
    rule.free()
