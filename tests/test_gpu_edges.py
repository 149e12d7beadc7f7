"""Edge cases of the device path against the oracle, through the C ABI:
the sin, erf and Bessel J0 / J1 activations, first-order tables (K = 1), a single input
(D0 = 1), one point, several outputs, and a closure set whose top degree
is below K."""
import numpy as np
import pytest

import pyoracle as po
from conftest import per_order_error, rel_err, xavier_weights
from dnnf90_b200 import api

pytestmark = pytest.mark.gpu

TOL = {api.PREC_F64: 1e-12, api.PREC_SPLIT: 1e-5}


def _check(d0, k, seeds, dims, npts, prec, activation=0, seed=0):
    rng = np.random.default_rng(seed)
    w = xavier_weights(dims, 7 + seed)
    w[np.arange(len(w)) % 6 == 0] += 0.05
    X = rng.uniform(-1, 1, (npts, d0))
    ts = api.TableSet(d0, k, seeds, activation=activation)
    ref = po.Tables(d0, k, seeds, activation=activation)
    net = api.Net(ts, dims, weights=w, precision=prec)
    tol = TOL[prec]
    T = net.eval(X)
    Tref = po.eval_batch(ref, dims, w, X)
    assert max(per_order_error(T, Tref, ref.deg).values()) < tol
    g = net.grad()
    r = api.SeedRule(api.SEED_HALFSQ)
    loss = g.rule_batch(X, r)
    gd = g.read()
    gref, _, lref, _ = po.grad_batch(ref, dims, w, X, kind=po.SEED_HALFSQ, want_t=False)
    assert rel_err(gd, gref) < tol, rel_err(gd, gref)
    assert abs(loss - lref) <= tol * abs(lref)
    r.free(); g.free(); net.free()


@pytest.mark.parametrize("prec", [api.PREC_F64, api.PREC_SPLIT])
@pytest.mark.parametrize("activation", [1, 2])
def test_sin_and_erf_activations(activation, prec):
    _check(3, 4, None, [3, 32, 32, 1], 64, prec, activation, seed=activation)


@pytest.mark.parametrize("prec", [api.PREC_F64, api.PREC_SPLIT])
def test_first_order_tables(prec):
    _check(3, 1, None, [3, 16, 16, 16, 1], 50, prec, seed=3)


@pytest.mark.parametrize("prec", [api.PREC_F64, api.PREC_SPLIT])
def test_single_input(prec):
    _check(1, 6, None, [1, 32, 32, 1], 40, prec, seed=4)


@pytest.mark.parametrize("prec", [api.PREC_F64, api.PREC_SPLIT])
def test_one_point_two_outputs(prec):
    _check(2, 3, None, [2, 16, 16, 2], 1, prec, seed=5)


def test_closure_below_k():
    # the closure of {(2, 0), (0, 1)} with K = 4 carries nothing above degree 2
    _check(2, 4, [[2, 0], [0, 1]], [2, 32, 32, 1], 33, api.PREC_F64, seed=6)


@pytest.mark.parametrize("prec", [api.PREC_F64, api.PREC_SPLIT])
@pytest.mark.parametrize("activation", [3, 4])
def test_bessel_activations(activation, prec):
    # J0 / J1 with their derivatives from J_0 .. J_{K+2}, K = 7 (nine orders)
    _check(2, 7, None, [2, 32, 32, 1], 48, prec, activation, seed=activation)
    _check(3, 4, None, [3, 32, 32, 1], 64, prec, activation, seed=10 + activation)
