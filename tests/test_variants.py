"""Every variant of the Bell forward and adjoint kernels against the oracle.

The autotuner picks one variant per launch shape by timing, so the parity
tests elsewhere see only the variant that won on the machine at hand.  Here
each variant is pinned in turn (dnnf90_tune_force) and the whole gradient
step is checked: derivatives, loss and dL/dw, in both precisions, over dense
and seeded sets from K = 1 to K = 8.  The tanh series forward (v9, off by
default) is switched off for the Bell variants and on for its own case.
Variant 3 is the register-tiled Horner forward and tiled correlation
adjoint (dense sets, FP32; elsewhere the pin falls back to the default)."""
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
    (3, 7, None, [3, 100, 44, 1], 9),     # ragged neuron tiles (100 = 3 * 32 + 4)
    (4, 4, None, [4, 36, 36, 36, 1], 17),
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
    api.tune_force(2, -1)


@pytest.mark.gpu
@pytest.mark.parametrize("d0,k,seeds,dims,npts", CASES)
@pytest.mark.parametrize("prec", [api.PREC_F64, api.PREC_SPLIT])
@pytest.mark.parametrize("fwd,adj,series", [(0, 0, 0), (1, 1, 0), (2, 2, 0), (2, 2, 1), (3, 3, 0)])
def test_pinned_variant(pinned, d0, k, seeds, dims, npts, prec, fwd, adj, series):
    pinned(0, fwd)
    pinned(1, adj)
    pinned(2, series)
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
        api.tune_force(4, 0)
    with pytest.raises(api.Dnnf90Error):
        api.tune_force(2, 2)
    with pytest.raises(api.Dnnf90Error):
        api.tune_force(3, 2)
    with pytest.raises(api.Dnnf90Error):
        api.tune_force(0, -2)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [api.PREC_F64, api.PREC_SPLIT])
def test_series_forward_agrees_with_the_bell_recurrence(pinned, prec):
    """The tanh series forward and the Bell recurrence compute the same
    planes to rounding (T and dL/dw through the whole step)."""
    d0, k, seeds, dims, npts = 4, 7, None, [4, 64, 48, 1], 6
    rng = np.random.default_rng(5)
    w = xavier_weights(dims, 29)
    X = rng.uniform(-1, 1, (npts, d0))
    ts, _ = _tables(d0, k, seeds)
    out = []
    for series in (0, 1):
        pinned(2, series)
        net = api.Net(ts, dims, weights=w, precision=prec)
        g = net.grad()
        r = api.SeedRule(api.SEED_HALFSQ)
        loss, T = g.rule_batch(X, r, want_t=True)
        out.append((T, g.read(), loss))
        r.free(); g.free(); net.free()
    tol = 1e-13 if prec == api.PREC_F64 else 1e-5
    assert rel_err(out[1][0], out[0][0]) < tol and rel_err(out[1][1], out[0][1]) < tol


@pytest.mark.gpu
def test_autotuner_report_names_the_launch_shape():
    """Unpinned, a launch with several waves of work (2048 points x 4 neuron
    tiles) is tuned once: the report names its kernel, table set (D0, K,
    |A|), width and precision, the chosen variant is one of the variants'
    ids, and every trial was timed."""
    ts = api.TableSet(4, 7)
    dims = [4, 128, 128, 1]
    w = xavier_weights(dims, 3)
    X = np.random.default_rng(3).uniform(-1, 1, (2048, 4))
    net = api.Net(ts, dims, weights=w, precision=api.PREC_SPLIT)
    g = net.grad()
    rule = api.SeedRule(api.SEED_HALFSQ)
    g.rule_batch(X, rule)
    rows = [r for r in api.tune_report() if r[1:6] == (4, 7, 330, 128, "f32")]
    assert {"bell_fwd_train", "bell_adj"} <= {r[0] for r in rows}, rows
    for kern, _, _, _, _, _, chosen, trials in rows:
        names = api.ADJ_VARIANTS if kern == "bell_adj" else api.FWD_VARIANTS
        assert chosen in names
        assert len(trials) >= 2 and all(t > 0 for t in trials)
    rule.free()
    g.free()
    net.free()
