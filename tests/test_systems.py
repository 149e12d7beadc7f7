"""System seed rules: several residuals over several output components
(calc_sys_residual / set_sys_seed, app/pinn_module.f90:86-162).

The oracle's restatement is pinned two ways on the CPU: against central
differences of its own loss, and against the scalar PINN rule, which is the
one-component special case.  On the GPU the device rule (forward -> seed on
the device -> adjoint) is checked against the oracle on a steady 2-D
Navier-Stokes system with outputs (u, v, p): two momentum residuals with
products of one component and another's derivative, and continuity.  The
value-only batched fit (net_grad_batch) is checked against a numpy
restatement of the reference's batched backpropagation.
"""
import numpy as np
import pytest

import pyoracle as po
from conftest import rel_err, xavier_weights

NU = 0.05


def _ns_terms(slot):
    """x- and y-momentum and continuity of steady incompressible flow."""
    s = {k: slot(v) for k, v in dict(v0=(0, 0), x=(1, 0), y=(0, 1), xx=(2, 0), yy=(0, 2)).items()}
    U, V, P = 1, 2, 3
    return [
        (1, 1.0, [(U, s["v0"]), (U, s["x"])]), (1, 1.0, [(V, s["v0"]), (U, s["y"])]),
        (1, 1.0, [(P, s["x"])]), (1, -NU, [(U, s["xx"])]), (1, -NU, [(U, s["yy"])]),
        (2, 1.0, [(U, s["v0"]), (V, s["x"])]), (2, 1.0, [(V, s["v0"]), (V, s["y"])]),
        (2, 1.0, [(P, s["y"])]), (2, -NU, [(V, s["xx"])]), (2, -NU, [(V, s["yy"])]),
        (3, 1.0, [(U, s["x"])]), (3, 1.0, [(V, s["y"])]),
    ]


def _oracle_slot(tab):
    alpha = [tuple(a) for a in tab.alpha]
    return lambda a: alpha.index(tuple(a)) + 1


def test_oracle_system_rule_against_finite_differences():
    tab = po.Tables(2, 2)
    dims = [2, 12, 12, 3]
    w = xavier_weights(dims, 3)
    X = np.random.default_rng(1).uniform(-1, 1, (9, 2))
    terms = _ns_terms(_oracle_slot(tab)) + [(2, 0.5, [(1, 2), (1, 2), (2, 3)])]  # a repeated factor
    src = np.random.default_rng(2).normal(size=(9, 3))
    args = dict(wres=[1.0, 2.0, 0.5], fac=1.5, src=src)
    g, _, _ = po.grad_sys_batch(tab, dims, w, X, 3, terms, **args)
    rng = np.random.default_rng(3)
    for _ in range(4):
        v = rng.normal(size=w.size)
        v /= np.linalg.norm(v)
        h = 1e-5
        lp = po.grad_sys_batch(tab, dims, w + h * v, X, 3, terms, want_t=False, **args)[2]
        lm = po.grad_sys_batch(tab, dims, w - h * v, X, 3, terms, want_t=False, **args)[2]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g @ v) <= 1e-7 * max(1.0, abs(fd)), (fd, g @ v)


def test_oracle_one_component_system_is_the_pinn_rule():
    tab = po.Tables(2, 3, [[0, 1], [1, 0], [3, 0]])
    slot = _oracle_slot(tab)
    dims = [2, 16, 16, 1]
    w = xavier_weights(dims, 4)
    X = np.random.default_rng(5).uniform(-1, 1, (20, 2))
    pinn = [(1.0, slot((0, 1)), 0), (6.0, slot((1, 0)), 1), (1.0, slot((3, 0)), 0)]
    sys_terms = [(1, c, [(1, 1), (1, s)] if nl else [(1, s)]) for c, s, nl in pinn]
    g1, T1, l1, _ = po.grad_batch(tab, dims, w, X, kind=po.SEED_PINN, terms=pinn, fac=0.7)
    g2, T2, l2 = po.grad_sys_batch(tab, dims, w, X, 1, sys_terms, fac=0.7)
    assert rel_err(g2, g1) < 1e-14 and abs(l2 - l1) <= 1e-14 * abs(l1)
    assert np.array_equal(T2[:, 0, :], T1)


# ---------------------------------------------------------------- device


def _device_case(prec, with_src):
    from dnnf90_b200 import api
    dims = [2, 48, 48, 3]
    ts = api.TableSet(2, 2)
    tab = po.Tables(2, 2)
    terms = _ns_terms(ts.slot)
    w = xavier_weights(dims, 8)
    w[np.arange(len(w)) % 5 == 0] += 0.03
    X = np.random.default_rng(6).uniform(-1, 1, (300, 2))
    src = np.random.default_rng(7).normal(size=(300, 3)) if with_src else None
    wres = [1.0, 1.0, 4.0]
    net = api.Net(ts, dims, weights=w, precision=prec)
    rule = api.SeedRule.system(3, terms, wres=wres, fac=0.5)
    g = net.grad()
    loss, tm = g.sys_batch(X, rule, src=src, want_t=True)
    gd = g.read()
    gref, Tref, lref = po.grad_sys_batch(tab, dims, w, X, 3, terms, wres=wres, fac=0.5, src=src)
    return (loss, tm, gd), (lref, Tref, gref), (net, rule, g, ts)


@pytest.mark.gpu
@pytest.mark.parametrize("with_src", [False, True])
@pytest.mark.parametrize("prec", [0, 1])
def test_device_system_rule_matches_the_oracle(prec, with_src):
    (loss, tm, gd), (lref, Tref, gref), (net, rule, g, ts) = _device_case(prec, with_src)
    tol = 1e-12 if prec == 0 else 1e-5
    assert rel_err(tm, Tref) < tol
    assert rel_err(gd, gref) < tol, rel_err(gd, gref)
    assert abs(loss - lref) <= tol * abs(lref)
    rule.free(); g.free(); net.free()


@pytest.mark.gpu
def test_system_rule_through_the_generic_entries():
    """With zero sources the rule also runs through dnnf90_grad_rule_batch
    and the device-pointer entry, with the same gradient."""
    import torch
    from dnnf90_b200 import api
    (loss, _, gd), _, (net, rule, g, ts) = _device_case(0, False)
    X = np.random.default_rng(6).uniform(-1, 1, (300, 2))
    g2 = net.grad()
    l2 = g2.rule_batch(X, rule)
    assert rel_err(g2.read(), gd) < 1e-14 and abs(l2 - loss) <= 1e-14 * abs(loss)
    dev = torch.device("cuda", 0)
    xd = torch.tensor(X, device=dev)
    gdev = torch.zeros(net.nw, dtype=torch.float64, device=dev)
    ldev = torch.zeros(1, dtype=torch.float64, device=dev)
    api.call("dnnf90_grad_rule_dev", net.nid, net.tid, X.shape[0], xd.data_ptr(), rule.rid,
             gdev.data_ptr(), ldev.data_ptr(), None, torch.cuda.current_stream(dev).cuda_stream)
    torch.cuda.synchronize(dev)
    assert rel_err(gdev.cpu().numpy(), gd) < 1e-14
    g2.free(); rule.free(); g.free(); net.free()


@pytest.mark.gpu
def test_system_rule_argument_checks():
    from dnnf90_b200 import api
    with pytest.raises(api.Dnnf90Error):
        api.SeedRule.system(2, [(3, 1.0, [(1, 1)])])            # residual outside 1..nres
    with pytest.raises(api.Dnnf90Error):
        api.SeedRule.system(1, [(1, 1.0, [(1, 1)] * 5)])        # five factors
    ts = api.TableSet(2, 2)
    net = api.Net(ts, [2, 16, 2], weights=xavier_weights([2, 16, 2], 1))
    rule = api.SeedRule.system(1, [(1, 1.0, [(3, 1)])])          # component 3 of 2
    g = net.grad()
    with pytest.raises(api.Dnnf90Error):
        g.sys_batch(np.zeros((4, 2)), rule)
    jr = api.SeedRule.system(1, [(1, 1.0, [(1, 2)])])
    with pytest.raises(api.Dnnf90Error):
        api.jacobian_rows(net, np.zeros((4, 2)), jr)
    rule.free(); jr.free(); g.free(); net.free(); ts.free()


# ------------------------------------------------------ value-only fit


def _value_fit_reference(dims, w, X, y, coef):
    """net_grad_batch (lib/train_module.f90:525-631) restated in numpy, FP64:
    forward with the bias channel, output deltas coef (N - y), deltas
    back through W_{l+1}^T times tanh', gradient blocks D_l [1, Z_{l-1}]^T.
    Weights in the flat layer layout (bias first)."""
    Ws, off = [], 0
    for l in range(1, len(dims)):
        n, m = dims[l], dims[l - 1]
        Ws.append(w[off:off + n * (m + 1)].reshape(n, m + 1))
        off += n * (m + 1)
    Z = [X]
    for l, W in enumerate(Ws):
        a = Z[-1] @ W[:, 1:].T + W[:, 0]
        Z.append(np.tanh(a) if l < len(Ws) - 1 else a)
    D = coef * (Z[-1] - y[:, None])
    loss = 0.5 * coef * float(((Z[-1][:, 0] - y) ** 2).sum())
    grads = [None] * len(Ws)
    for l in range(len(Ws) - 1, -1, -1):
        grads[l] = D.T @ np.hstack([np.ones((X.shape[0], 1)), Z[l]])
        if l > 0:
            D = (D @ Ws[l][:, 1:]) * (1.0 - Z[l] ** 2)
    return np.concatenate([g.reshape(-1) for g in grads]), loss


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [0, 1])
def test_value_fit_matches_the_batched_reference(prec):
    from dnnf90_b200 import api
    dims = [3, 64, 64, 1]
    w = xavier_weights(dims, 12)
    w[np.arange(len(w)) % 7 == 0] += 0.05
    rng = np.random.default_rng(13)
    X = rng.uniform(-1, 1, (5000, 3))
    y = np.sin(X.sum(axis=1))
    gref, lref = _value_fit_reference(dims, w, X, y, 0.8)
    tol = 1e-12 if prec == 0 else 1e-5
    # the value alone (closure of {0}), then a full K = 2 set: only the value slot enters
    for seeds, k in (([[0, 0, 0]], 1), (None, 2)):
        ts = api.TableSet(3, k, seeds)
        net = api.Net(ts, dims, weights=w, precision=prec)
        g = net.grad()
        for rep in range(2):            # two calls add up
            loss = g.value_batch(X, y, 0.8)
            assert abs(loss - lref) <= tol * lref
        assert rel_err(g.read(), 2 * gref) < tol, rel_err(g.read(), 2 * gref)
        g.free(); net.free(); ts.free()
    with pytest.raises(api.Dnnf90Error):               # a single output only
        ts = api.TableSet(3, 1, [[0, 0, 0]])
        net2 = api.Net(ts, [3, 8, 2], weights=xavier_weights([3, 8, 2], 1))
        g2 = net2.grad()
        g2.value_batch(X[:4], y[:4])
