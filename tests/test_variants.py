"""Every variant of the Bell forward and adjoint kernels against the oracle.

The autotuner picks one variant per launch shape by timing, so the parity
tests elsewhere see only the variant that won on the machine at hand.  Here
each variant is pinned in turn (dnnf90_tune_force) and the whole gradient
step is checked: derivatives, loss and dL/dw, in both precisions, over dense
and seeded sets from K = 1 to K = 8."""
import numpy as np
import pytest

import pyoracle as po
from conftest import per_order_error, rel_err, xavier_weights
from dnnf90_b200 import api

CASES = [
    (4, 7, None, [4, 64, 48, 1], 5),
    (2, 3, [[0, 1], [1, 0], [3, 0]], [2, 64, 64, 64, 1], 200),
    (3, 5, None, [3, 32, 32, 1], 40),
    (2, 8, None, [2, 32, 32, 1], 30),
    (1, 1, None, [1, 32, 32, 1], 64),
    (1, 2, None, [1, 36, 20, 1], 64),
]


_TABLES = {}


def _tables(d0, k, seeds):
    # table sets have no free in the reference's API (64 handles): one per case
    key = (d0, k, str(seeds))
    if key not in _TABLES:
        _TABLES[key] = (api.TableSet(d0, k, seeds), po.Tables(d0, k, seeds))
    return _TABLES[key]


@pytest.fixture
def pinned():
    yield api.tune_force
    api.tune_force(0, -1)
    api.tune_force(1, -1)


@pytest.mark.gpu
@pytest.mark.parametrize("d0,k,seeds,dims,npts", CASES)
@pytest.mark.parametrize("prec", [api.PREC_F64, api.PREC_SPLIT])
@pytest.mark.parametrize("fwd,adj", [(0, 0), (1, 1), (2, 2)])
def test_pinned_variant(pinned, d0, k, seeds, dims, npts, prec, fwd, adj):
    pinned(0, fwd)
    pinned(1, adj)
    rng = np.random.default_rng(17)
    w = xavier_weights(dims, 23)
    w[np.arange(len(w)) % 6 == 0] += 0.04
    X = rng.uniform(-1, 1, (npts, d0))
    ts, ref = _tables(d0, k, seeds)
    net = api.Net(ts, dims, weights=w, precision=prec)
    g = net.grad()
    r = api.SeedRule(api.SEED_HALFSQ)
    loss, T = g.rule_batch(X, r, want_t=True)
    gd = g.read()
    gref, Tref, lref, _ = po.grad_batch(ref, dims, w, X)
    tol = 1e-12 if prec == api.PREC_F64 else 1e-5
    assert max(per_order_error(T, Tref, ref.deg).values()) < tol
    assert rel_err(gd, gref) < tol, rel_err(gd, gref)
    assert abs(loss - lref) <= tol * abs(lref)
    r.free(); g.free(); net.free()


@pytest.mark.gpu
def test_force_rejects_bad_arguments():
    with pytest.raises(api.Dnnf90Error):
        api.tune_force(2, 0)
    with pytest.raises(api.Dnnf90Error):
        api.tune_force(0, -2)
