"""Parity of the CUDA path with the CPU oracle (and through it with the
reference), called through the C ABI.

Tolerances: the plain FP64 path agrees with the reference to 1e-12
normwise per derivative order; the split path (FP32 planes, 3-term
split-BF16 GEMMs) to 1e-5 per order and on the weight gradient."""
import numpy as np
import pytest

import pyoracle as po
from conftest import per_order_error, rel_err, xavier_weights
from dnnf90_b200 import api

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOLSPLIT = 1e-5


def _net(ts, dims, w, prec=api.PREC_F64):
    return api.Net(ts, dims, weights=w, precision=prec)


def test_golden_cases_through_the_device(golden):
    for case in golden["hod_cases"] + golden["jet_cases"]:
        d0 = case["dims"][0]
        ts = api.TableSet(d0, case["k"], case["seeds"])
        net = _net(ts, case["dims"], po.check_weights(case["dims"]))
        t = net.eval(np.array(case["x"]))          # dnnf90_eval, one point
        ref = po.Tables(d0, case["k"], case["seeds"])
        errs = per_order_error(t, case["t"], ref.deg)
        assert max(errs.values()) < TOL64, (case["dims"], errs)
        net.free()


@pytest.mark.parametrize("d0,k,seeds,dims", [
    (4, 3, None, [4, 32, 32, 1]),
    (2, 3, [[0, 1], [1, 0], [3, 0]], [2, 64, 64, 64, 1]),
    (3, 2, [[1, 0, 0], [0, 2, 0], [0, 0, 2]], [3, 64, 64, 1]),
    (4, 7, None, [4, 48, 40, 1]),
    (3, 4, None, [3, 16, 16, 16, 16, 2]),
])
@pytest.mark.parametrize("prec", [api.PREC_F64, api.PREC_SPLIT])
def test_eval_batch(d0, k, seeds, dims, prec):
    rng = np.random.default_rng(11)
    w = xavier_weights(dims, 5)
    w[np.arange(len(w)) % 7 == 0] += 0.1     # nonzero biases
    X = rng.uniform(-1, 1, (37, d0))
    ts = api.TableSet(d0, k, seeds)
    ref = po.Tables(d0, k, seeds)
    net = _net(ts, dims, w, prec)
    T = net.eval(X)
    Tref = po.eval_batch(ref, dims, w, X)
    errs = per_order_error(T, Tref, ref.deg)
    assert max(errs.values()) < (TOL64 if prec == api.PREC_F64 else TOLSPLIT), errs
    if dims[-1] > 1:
        Tm = net.eval_multi(X)
        for p in range(3):
            _, tall = po.eval_point(ref, dims, w, X[p])
            assert rel_err(Tm[p], tall) < (TOL64 if prec == api.PREC_F64 else TOLSPLIT)
    net.free()


def _rule_terms(ts, name):
    if name == "halfsq":
        return po.SEED_HALFSQ, [], 1.0
    if name == "kdv":   # u_t + 6 u u_x + u_xxx with (x, t)
        return po.SEED_PINN, [(1.0, ts.slot((0, 1)), 0), (6.0, ts.slot((1, 0)), 1),
                              (1.0, ts.slot((3, 0)), 0)], 1.0
    if name == "zk7":   # all order-7 slots + u u_x (x = axis 2)
        terms = [(1.0, i + 1, 0) for i in range(ts.na) if ts.alpha[i].sum() == 7]
        return po.SEED_PINN, terms + [(1.0, ts.slot((0, 1, 0, 0)), 1)], 1.0
    raise ValueError(name)


@pytest.mark.parametrize("d0,k,seeds,dims,rule,npts", [
    (4, 3, None, [4, 32, 32, 1], "halfsq", 200),
    (2, 3, [[0, 1], [1, 0], [3, 0]], [2, 64, 64, 64, 1], "kdv", 300),
    (4, 7, None, [4, 64, 64, 64, 1], "zk7", 6),
    (4, 5, None, [4, 24, 20, 3], "halfsq", 40),
    (2, 3, None, [2, 256, 256, 256, 1], "halfsq", 64),   # K = 256 layer GEMMs (N tile 64)
])
@pytest.mark.parametrize("prec", [api.PREC_F64, api.PREC_SPLIT])
def test_grad_rule_batch(d0, k, seeds, dims, rule, npts, prec):
    rng = np.random.default_rng(3)
    w = xavier_weights(dims, 9)
    w[np.arange(len(w)) % 5 == 0] += 0.05
    X = rng.uniform(-1, 1, (npts, d0))
    ts = api.TableSet(d0, k, seeds)
    ref = po.Tables(d0, k, seeds)
    kind, terms, fac = _rule_terms(ts, rule)
    net = _net(ts, dims, w, prec)
    g = net.grad()
    r = api.SeedRule(kind, terms, fac)
    loss, T = g.rule_batch(X, r, want_t=True)
    gd = g.read()
    gref, Tref, lref, _ = po.grad_batch(ref, dims, w, X, kind=kind, terms=terms, fac=fac)
    tol = TOL64 if prec == api.PREC_F64 else TOLSPLIT
    assert max(per_order_error(T, Tref, ref.deg).values()) < tol
    assert rel_err(gd, gref) < tol, rel_err(gd, gref)
    assert abs(loss - lref) <= tol * abs(lref)
    r.free(); g.free(); net.free()


def test_grad_point_queue_equals_batch():
    dims = [4, 32, 32, 1]
    ts = api.TableSet(4, 3)
    ref = po.Tables(4, 3)
    w = xavier_weights(dims, 2)
    X = np.random.default_rng(4).uniform(-1, 1, (50, 4))
    S = np.random.default_rng(5).normal(size=(50, ts.na))
    net = _net(ts, dims, w)
    g1, g2 = net.grad(), net.grad()
    for i in range(50):
        g1.point(X[i], S[i])           # queued, flushed by read
    g2.batch(X, S)
    a, b = g1.read(), g2.read()
    gref, _, _, _ = po.grad_batch(ref, dims, w, X, kind=po.SEED_GIVEN, seeds=S)
    assert rel_err(a, gref) < TOL64 and rel_err(b, gref) < TOL64
    g1.zero()
    assert np.all(g1.read() == 0)
    g1.free(); g2.free(); net.free()


def test_adam_step_matches_the_oracle():
    dims = [4, 16, 16, 1]
    ts = api.TableSet(4, 3)
    ref = po.Tables(4, 3)
    w = xavier_weights(dims, 8)
    X = np.random.default_rng(1).uniform(-1, 1, (64, 4))
    net = _net(ts, dims, w)
    g = net.grad()
    m, v, wr = np.zeros_like(w), np.zeros_like(w), w.copy()
    for step in range(1, 4):
        g.zero()
        r = api.SeedRule(api.SEED_HALFSQ)
        g.rule_batch(X, r)
        g.adam(1e-3, 0.9, 0.999, 1e-8, 64, step)
        gref = po.grad_batch(ref, dims, wr, X)[0]
        po.adam_step(wr, gref, m, v, 1e-3, 0.9, 0.999, 1e-8, 64, step)
        r.free()
    assert rel_err(net.get_weights(), wr) < 1e-12
    g.free(); net.free()


def test_jacobian_rows_and_ngd_step():
    # config-5 shape: heat residual u_t - (u_xx + u_yy) on (t, x, y)
    dims = [3, 64, 64, 1]
    seeds = [[1, 0, 0], [0, 2, 0], [0, 0, 2]]
    ts = api.TableSet(3, 2, seeds)
    ref = po.Tables(3, 2, seeds)
    terms = [(1.0, ts.slot((1, 0, 0)), 0), (-1.0, ts.slot((0, 2, 0)), 0),
             (-1.0, ts.slot((0, 0, 2)), 0)]
    w = xavier_weights(dims, 12)
    X = np.random.default_rng(2).uniform(0, 1, (256, 3))
    for prec in (api.PREC_F64, api.PREC_SPLIT):
        net = _net(ts, dims, w, prec)
        r = api.SeedRule(api.SEED_JROW, terms)
        rows, resid, T = api.jacobian_rows(net, X, r)
        _, Tref, _, rref = po.grad_batch(ref, dims, w, X, kind=po.SEED_JROW, terms=terms)
        tol = TOL64 if prec == api.PREC_F64 else TOLSPLIT
        assert rel_err(rows, rref) < tol
        Rref = sum(c * Tref[:, s - 1] for c, s, _ in terms)
        assert rel_err(resid, Rref) < tol
        b = (resid[:, None] * rows).sum(axis=0)
        nb, mu = len(X), 1e-6
        u = api.ngd_step(net, rows, b, nb, mu, prec)
        # the damped metric is ill-conditioned (rank <= points + mu I), so
        # the solve is judged by its backward error on the oracle's system
        bref = (Rref[:, None] * rref).sum(axis=0) / nb
        G = rref.T @ rref / nb + mu * np.eye(rref.shape[1])
        berr = np.linalg.norm(G @ u - bref) / (np.linalg.norm(G, 2) * np.linalg.norm(u)
                                               + np.linalg.norm(bref))
        assert berr < (1e-12 if prec == api.PREC_F64 else 1e-6), berr
        r.free(); net.free()


def test_directional_known_answers_on_the_device(golden):
    dk = golden["dirkat"]
    d0, W = dk["d0"], dk["width"]
    w_ref, w, p = dk["w_ref"], [], 0
    for fan, n in [(d0, W), (W, W), (W, 1)]:
        for _ in range(n):
            w.append(w_ref[p + fan]); w.extend(w_ref[p:p + fan]); p += fan + 1
    X = np.array(dk["x"]).reshape(dk["npt"], d0)
    for ks, (lref, gref) in dk["table"].items():
        K = int(ks)
        ts = api.TableSet(4, K, [[K, 0, 0, 0]])
        net = _net(ts, [4, 8, 8, 1], np.array(w))
        g = net.grad()
        r = api.SeedRule(api.SEED_PINN, [(1.0, ts.slot((K, 0, 0, 0)), 0)], 2.0)
        loss = g.rule_batch(X, r)
        # rule loss is fac R^2 / 2 = R^2 summed: the table's loss
        assert abs(loss / lref - 1) < 1e-11, (K, loss, lref)
        assert abs(g.read()[1] / gref - 1) < 5e-9
        r.free(); g.free(); net.free()


def test_ngd_step_at_heat_scale():
    """Damped Gauss-Newton step on the heat residual at full size: 4096
    points, 3-64-64-1 (4481 weights).  The split path forms J^T J on the
    tensor cores (split-BF16 products, FP32 accumulation per 512 rows, FP64
    across them) and solves in FP64; both are judged by backward error on
    the FP64 system, the metric itself against numpy."""
    dims = [3, 64, 64, 1]
    seeds = [[1, 0, 0], [0, 2, 0], [0, 0, 2]]
    ts = api.TableSet(3, 2, seeds)
    terms = [(1.0, ts.slot((1, 0, 0)), 0), (-1.0, ts.slot((0, 2, 0)), 0),
             (-1.0, ts.slot((0, 0, 2)), 0)]
    w = xavier_weights(dims, 5)
    X = np.random.default_rng(8).uniform(0, 1, (4096, 3))
    net = _net(ts, dims, w, api.PREC_F64)
    r = api.SeedRule(api.SEED_JROW, terms)
    rows, resid, _ = api.jacobian_rows(net, X, r)
    assert rows.shape == (4096, 4481)
    nb, mu = len(X), 1e-6
    b = (resid[:, None] * rows).sum(axis=0)
    G = rows.T @ rows / nb + mu * np.eye(rows.shape[1])
    bn = b / nb
    v = np.random.default_rng(0).normal(size=G.shape[0])
    for _ in range(30):  # power iteration for ||G||_2
        v = G @ v
        v /= np.linalg.norm(v)
    g2 = float(v @ (G @ v))
    for prec, bound in ((api.PREC_F64, 1e-12), (api.PREC_SPLIT, 1e-6)):
        u = api.ngd_step(net, rows, b, nb, mu, prec)
        assert np.all(np.isfinite(u))
        berr = np.linalg.norm(G @ u - bn) / (g2 * np.linalg.norm(u) + np.linalg.norm(bn))
        assert berr < bound, (prec, berr)
    r.free(); net.free()


def test_ngd_dual_route_equals_the_primal_step():
    """The Gram-space route (app/optimizer_module.f90:408-446) on fewer rows
    than weights: 512 heat-residual rows, 4481 weights.  The step must be the
    primal one to roundoff, and both must meet the primal backward-error
    bound on the FP64 system."""
    dims = [3, 64, 64, 1]
    seeds = [[1, 0, 0], [0, 2, 0], [0, 0, 2]]
    ts = api.TableSet(3, 2, seeds)
    terms = [(1.0, ts.slot((1, 0, 0)), 0), (-1.0, ts.slot((0, 2, 0)), 0),
             (-1.0, ts.slot((0, 0, 2)), 0)]
    w = xavier_weights(dims, 6)
    X = np.random.default_rng(9).uniform(0, 1, (512, 3))
    net = _net(ts, dims, w, api.PREC_F64)
    r = api.SeedRule(api.SEED_JROW, terms)
    rows, resid, _ = api.jacobian_rows(net, X, r)
    nb, mu = len(X), 1e-3
    b = (resid[:, None] * rows).sum(axis=0)
    G = rows.T @ rows / nb + mu * np.eye(rows.shape[1])
    bn = b / nb
    g2 = np.linalg.norm(rows, 2) ** 2 / nb + mu
    # the routes agree to roundoff amplified by the conditioning (||G|| /
    # mu); the dual route forms its nrow x nrow Gram matrix in FP64 in both
    # precisions, so it meets the FP64 bound; the split primal metric is
    # judged by backward error
    up = api.ngd_step(net, rows, b, nb, mu, api.PREC_F64)
    ud = api.ngd_step(net, rows, b, nb, mu, api.PREC_F64, dual=True)
    uds = api.ngd_step(net, rows, b, nb, mu, api.PREC_SPLIT, dual=True)
    ups = api.ngd_step(net, rows, b, nb, mu, api.PREC_SPLIT)
    assert rel_err(ud, up) < 1e-9, rel_err(ud, up)
    assert rel_err(uds, ud) < 1e-9     # FP64 both; atomics order the sums differently
    for u, bound in ((up, 1e-12), (ud, 1e-12), (ups, 1e-6)):
        berr = np.linalg.norm(G @ u - bn) / (g2 * np.linalg.norm(u) + np.linalg.norm(bn))
        assert berr < bound, berr
    with pytest.raises(api.Dnnf90Error):
        api.ngd_step(net, rows, b, nb, 0.0, api.PREC_F64, dual=True)   # mu must be > 0
    r.free(); net.free(); ts.free()


@pytest.mark.gpu
def test_sharded_ngd_halves_on_the_device():
    """The step for rows spread over ranks (dp.ngd_step_sharded) on one
    device: the metric built in two row blocks and summed, then solved
    (dnnf90_ngd_gram_dev + dnnf90_ngd_solve_dev), and the device dual route,
    equal the host entry dnnf90_ngd_step on all rows."""
    import torch
    from dnnf90_b200.dp import DeviceNGD, ngd_step_sharded
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(21)
    ts = api.TableSet(2, 1)
    net = _net(ts, [2, 20, 20, 1], None, api.PREC_F64)   # the host entry takes nw from it
    nw, nrow, mu = net.nw, 300, 1e-3
    J = rng.normal(size=(nrow, nw)) / np.sqrt(nw)
    b = rng.normal(size=nw)
    up = api.ngd_step(net, J, b, nrow, mu, api.PREC_F64)
    Jd, bd = torch.tensor(J, device=dev), torch.tensor(b, device=dev)
    for prec, tol in ((0, 1e-10), (1, 1e-5)):
        ops = DeviceNGD(prec)
        u1 = ngd_step_sharded(Jd, bd, mu, ops=ops).cpu().numpy()
        # two row blocks, their metrics summed as the all-reduce would
        G = torch.zeros(nw, nw, dtype=torch.float64, device=dev)
        G2 = torch.zeros_like(G)
        ops.gram(Jd[:170].contiguous(), G)
        ops.gram(Jd[170:].contiguous(), G2)
        G += G2
        u2 = torch.empty(nw, dtype=torch.float64, device=dev)
        ops.solve(G, bd, nrow, mu, u2)
        assert rel_err(u1, up) < tol and rel_err(u2.cpu().numpy(), up) < tol, prec
    ud = ngd_step_sharded(Jd, bd, mu, route="dual").cpu().numpy()
    assert rel_err(ud, up) < 1e-9
    net.free(); ts.free()
