"""Extended Kalman filter (lib/kalman_module.f90): the rank-one update of
kf_update_grad (:353-490) on the dense and the node-wise decoupled
covariance, with the forgetting schedule, process noise and innovation gate.

The oracle restatement is pinned on the CPU by the reference's own known
answer (tools/example_libverify.f90:215-286: on a linear network, lambda = 1,
the filter reproduces the ridge normal-equation solution to 1e-9) and by
properties of the algebra: a decoupled filter with one block is the dense
one, and a gated update is the ungated update of the row and innovation
scaled by the gate's s.  On the GPU the device filter is checked against the
oracle observation by observation (weights, covariance, lambda, gate count),
through the ridge known answer, across call and staging boundaries, and on a
nonpositive denominator.
"""
import numpy as np
import pytest

import pyoracle as po
from conftest import rel_err

D0, NS, P0 = 3, 60, 50.0


def _ridge_samples():
    """The deterministic samples of the reference's check (1-based n, i)."""
    n = np.arange(1, NS + 1)[:, None]
    i = np.arange(1, D0 + 1)[None, :]
    x = np.sin(1.7 * n + 0.9 * i)
    y = 0.7 - 1.3 * x[:, 0] + 0.4 * x[:, 1] + 2.1 * x[:, 2]
    return x, y


def _ridge_solution(x, y):
    xe = np.hstack([np.ones((len(x), 1)), x])
    A = np.eye(D0 + 1) / P0 + xe.T @ xe
    return np.linalg.solve(A, xe.T @ y)


def test_oracle_kalman_is_the_ridge_solution_on_a_linear_net():
    x, y = _ridge_samples()
    kf = po.Kalman([D0, 1], P0, 1.0, 1.0)
    w = np.zeros(D0 + 1)                        # net_init zeroes the weights
    for n in range(NS):
        xe = np.concatenate([[1.0], x[n]])
        kf.update(w, xe, y[n] - w @ xe)
    b = _ridge_solution(x, y)
    assert np.abs(w - b).max() / np.abs(b).max() < 1e-9


def _random_sequence(nw, nobs, seed):
    rng = np.random.default_rng(seed)
    rows = rng.normal(size=(nobs, nw)) / np.sqrt(nw)
    xi = 2.0 * rng.normal(size=nobs)
    scale = rng.uniform(0.5, 2.0, nobs)
    return rows, xi, scale


def test_oracle_one_block_decoupled_is_dense():
    dims = [3, 1]                               # one neuron: one block of 4
    rows, xi, sc = _random_sequence(4, 25, 1)
    a, b = po.Kalman(dims, 3.0, 0.98, 0.99, q=1e-3), po.Kalman(dims, 3.0, 0.98, 0.99, True, q=1e-3)
    wa, wb = np.zeros(4), np.zeros(4)
    for r, e, s in zip(rows, xi, sc):
        a.update(wa, r, e, s)
        b.update(wb, r, e, s)
    assert np.array_equal(wa, wb) and np.array_equal(a.P, b.P) and a.lam == b.lam


def test_oracle_decoupled_first_update_is_the_dense_diagonal_blocks():
    """From P = p0 I (block diagonal) the first update gives both filters
    the same P j, the same global denominator and the same weight step; the
    decoupled covariance is then the dense one's diagonal blocks."""
    dims = [3, 5, 4, 1]
    nw = po.weight_count(dims)
    rows, xi, sc = _random_sequence(nw, 1, 9)
    d, b = po.Kalman(dims, 0.8, 0.97, 0.99, q=1e-3, gate=1.0), po.Kalman(dims, 0.8, 0.97, 0.99, True, q=1e-3, gate=1.0)
    wd, wb = np.zeros(nw), np.zeros(nw)
    d.update(wd, rows[0], xi[0], sc[0])
    b.update(wb, rows[0], xi[0], sc[0])
    assert np.array_equal(wd, wb) and d.lam == b.lam and d.ngated.value == b.ngated.value
    Pd = d.P.reshape(nw, nw)
    blocks = np.concatenate([Pd[o:o + n, o:o + n].reshape(-1) for o, n in zip(b.boff, b.bsz)])
    assert np.array_equal(blocks, b.P)


def test_oracle_gate_is_a_noise_scale():
    """A tripped gate applies the update of the row and innovation scaled
    by s, s^2 = gate^2 lambda / (xi^2 - gate^2 j.Pj), which leaves the
    normalised innovation at the gate."""
    dims = [2, 4, 1]
    nw = po.weight_count(dims)
    rows, _, _ = _random_sequence(nw, 1, 2)
    j, xi, gate = rows[0], 40.0, 2.0
    g = po.Kalman(dims, 2.0, 0.99, 0.995, gate=gate)
    wg = np.zeros(nw)
    jpj = j @ (g.P.reshape(nw, nw) @ j)
    lam = g.lam
    g.update(wg, j, xi)
    assert g.ngated.value == 1
    s = np.sqrt(gate ** 2 * lam / (xi ** 2 - gate ** 2 * jpj))
    assert abs((s * xi) ** 2 - gate ** 2 * (lam + s ** 2 * jpj)) < 1e-9 * xi ** 2
    u = po.Kalman(dims, 2.0, 0.99, 0.995)
    wu = np.zeros(nw)
    u.update(wu, j, xi, s)
    assert rel_err(wg, wu) < 1e-14 and rel_err(g.P, u.P) < 1e-14
    # an innovation inside the gate leaves the update alone
    h, k = po.Kalman(dims, 2.0, 0.99, 0.995, gate=gate), po.Kalman(dims, 2.0, 0.99, 0.995)
    wh, wk = np.zeros(nw), np.zeros(nw)
    h.update(wh, j, 0.1)
    k.update(wk, j, 0.1)
    assert h.ngated.value == 0 and np.array_equal(wh, wk) and np.array_equal(h.P, k.P)


# ---------------------------------------------------------------- device


def _net(dims, w=None):
    from dnnf90_b200 import api
    ts = api.TableSet(dims[0], 1)
    return api.Net(ts, dims, weights=w), ts


@pytest.mark.gpu
def test_device_kalman_is_the_ridge_solution_on_a_linear_net():
    from dnnf90_b200 import api
    x, y = _ridge_samples()
    net, ts = _net([D0, 1], np.zeros(D0 + 1))
    kf = api.Kalman(net, P0, 1.0, 1.0)
    for n in range(NS):                         # one observation per call
        xe = np.concatenate([[1.0], x[n]])
        w = net.get_weights()
        kf.update_rows(xe, y[n] - w @ xe)
    b = _ridge_solution(x, y)
    assert np.abs(net.get_weights() - b).max() / np.abs(b).max() < 1e-9
    kf.free(); net.free(); ts.free()


CASES = [  # dims, decoupled, q, gate, nobs
    ([3, 20, 20, 1], False, 0.0, 0.0, 40),
    ([3, 20, 20, 1], False, 1e-4, 1.5, 40),
    ([3, 20, 20, 1], True, 0.0, 0.0, 40),
    ([3, 20, 20, 1], True, 1e-4, 1.5, 40),
    ([2, 3, 1], False, 1e-3, 0.0, 30),          # nw = 13: one padded tile
    ([2, 3, 1], True, 0.0, 1.0, 30),
    ([4, 40, 33, 2], False, 0.0, 2.0, 12),      # nw = 1485, block edges off the tile grid
    ([4, 40, 33, 2], True, 1e-5, 0.0, 12),
]


def _run_both(dims, decoupled, q, gate, nobs, seed=3):
    from dnnf90_b200 import api
    nw = po.weight_count(dims)
    rows, xi, sc = _random_sequence(nw, nobs, seed)
    w0 = np.random.default_rng(seed + 1).normal(size=nw) * 0.1
    net, ts = _net(dims, w0)
    kf = api.Kalman(net, 0.7, 0.98, 0.9987, decoupled, q, gate)
    ref = po.Kalman(dims, 0.7, 0.98, 0.9987, decoupled, q, gate)
    wref = w0.copy()
    for r, e, s in zip(rows, xi, sc):
        ref.update(wref, r, e, s)
    return (kf, net, ts), ref, wref, (rows, xi, sc)


@pytest.mark.gpu
@pytest.mark.parametrize("dims,decoupled,q,gate,nobs", CASES)
def test_device_kalman_matches_the_oracle(dims, decoupled, q, gate, nobs):
    (kf, net, ts), ref, wref, (rows, xi, sc) = _run_both(dims, decoupled, q, gate, nobs)
    kf.update_rows(rows, xi, sc)
    lam, ng = kf.state()
    assert ng == ref.ngated.value
    if gate > 0 and len(dims) > 3:
        assert ng > 0                           # the gate was exercised
    assert abs(lam - ref.lam) <= 1e-15
    assert rel_err(net.get_weights(), wref) < 1e-11, rel_err(net.get_weights(), wref)
    P = kf.cov().reshape(-1)
    assert rel_err(P, ref.P) < 1e-11, rel_err(P, ref.P)
    if not decoupled:
        Pm = P.reshape(net.nw, net.nw)
        assert np.array_equal(Pm, Pm.T)         # exactly symmetric
    kf.free(); net.free(); ts.free()


@pytest.mark.gpu
@pytest.mark.parametrize("decoupled", [False, True])
def test_device_kalman_split_across_calls_and_stages(decoupled, monkeypatch):
    """The same sequence in one call, in several calls, and through a
    staging area of a few rows gives the same filter."""
    from dnnf90_b200 import api
    dims = [3, 20, 20, 1]
    (kf, net, ts), ref, wref, (rows, xi, sc) = _run_both(dims, decoupled, 1e-4, 1.5, 40)
    kf.update_rows(rows, xi, sc)
    w1, P1, s1 = net.get_weights(), kf.cov(), kf.state()
    for parts, stage_kb in (([7, 1, 20, 12], None), ([40], 9)):
        net2, ts2 = _net(dims, np.random.default_rng(4).normal(size=net.nw) * 0.1)
        kf2 = api.Kalman(net2, 0.7, 0.98, 0.9987, decoupled, 1e-4, 1.5)
        if stage_kb:                            # 9 KB: two rows of 521 weights per stage
            monkeypatch.setenv("DNNF90_KF_STAGE_KB", str(stage_kb))
        k0 = 0
        for m in parts:
            kf2.update_rows(rows[k0:k0 + m], xi[k0:k0 + m], sc[k0:k0 + m])
            k0 += m
        monkeypatch.delenv("DNNF90_KF_STAGE_KB", raising=False)
        assert np.array_equal(net2.get_weights(), w1)
        assert np.array_equal(kf2.cov(), P1) and kf2.state() == s1
        kf2.free(); net2.free(); ts2.free()
    kf.free(); net.free(); ts.free()


@pytest.mark.gpu
def test_device_kalman_stops_at_a_nonpositive_denominator():
    from dnnf90_b200 import api
    dims = [3, 20, 20, 1]
    nw = po.weight_count(dims)
    rows, xi, sc = _random_sequence(nw, 10, 5)
    rows[6, 17] = np.nan                        # j.Pj is NaN at observation 7
    net, ts = _net(dims, np.zeros(nw))
    kf = api.Kalman(net, 0.7, 0.98, 0.9987)
    with pytest.raises(api.Dnnf90Error):
        kf.update_rows(rows, xi, sc)
    assert "observation 7" in api.lib().dnnf90_last_error().decode()
    assert api.lib().dnnf90_kf_status(kf.kid) == 7
    ref = po.Kalman(dims, 0.7, 0.98, 0.9987)
    wref = np.zeros(nw)
    for k in range(6):
        ref.update(wref, rows[k], xi[k], sc[k])
    assert rel_err(net.get_weights(), wref) < 1e-11
    assert rel_err(kf.cov().reshape(-1), ref.P) < 1e-11 and abs(kf.state()[0] - ref.lam) < 1e-15
    kf.update_rows(rows[7:], xi[7:], sc[7:])    # the filter goes on from there
    assert api.lib().dnnf90_kf_status(kf.kid) == 0
    for k in range(7, 10):
        ref.update(wref, rows[k], xi[k], sc[k])
    assert rel_err(net.get_weights(), wref) < 1e-11
    kf.free(); net.free(); ts.free()


@pytest.mark.gpu
def test_device_kalman_device_entry():
    import torch
    from dnnf90_b200 import api
    dims = [3, 20, 20, 1]
    (kf, net, ts), ref, wref, (rows, xi, sc) = _run_both(dims, True, 1e-4, 1.5, 40)
    dev = torch.device("cuda", 0)
    w0 = net.get_weights()
    wd = torch.tensor(w0, device=dev)
    rd, xd, sd = (torch.tensor(a, device=dev) for a in (rows, xi, sc))
    api.call("dnnf90_kf_update_rows_dev", kf.kid, len(xi), rd.data_ptr(), xd.data_ptr(),
             sd.data_ptr(), wd.data_ptr(), torch.cuda.current_stream(dev).cuda_stream)
    assert rel_err(wd.cpu().numpy(), wref) < 1e-11
    assert np.array_equal(net.get_weights(), w0)   # the network's own weights untouched
    assert rel_err(kf.cov().reshape(-1), ref.P) < 1e-11
    kf.free(); net.free(); ts.free()


@pytest.mark.gpu
def test_kalman_argument_checks():
    from dnnf90_b200 import api
    net, ts = _net([3, 8, 1])
    for args in ((0.0, 0.98, 0.99), (1.0, 0.0, 0.99), (1.0, 0.98, 1.5), (1.0, 1.2, 0.9)):
        with pytest.raises(api.Dnnf90Error):
            api.Kalman(net, *args)
    with pytest.raises(api.Dnnf90Error):
        api.Kalman(net, 1.0, 0.98, 0.99, q=-1.0)
    kf = api.Kalman(net, 1.0, 0.98, 0.99)
    net.free()
    with pytest.raises(api.Dnnf90Error):        # the network is gone
        kf.update_rows(np.zeros(net.nw), [0.0])
    kid = kf.kid
    kf.free()
    assert api.lib().dnnf90_kf_free(kid) < 0      # freed twice
    ts.free()


# ------------------------------------------------- iterated EKF (kf_iekf_*)


def _obs(a, z):
    """A nonlinear scalar observation h(w) = sum a_i sin(w_i) with target z:
    R(w) = h(w) - z and dR/dw = a cos(w)."""
    return (lambda w: float(a @ np.sin(w)) - z), (lambda w: a * np.cos(w))


def test_oracle_one_final_iteration_is_the_plain_update():
    dims = [3, 6, 1]
    nw = po.weight_count(dims)
    rng = np.random.default_rng(8)
    w0 = rng.normal(size=nw)
    R, J = _obs(rng.normal(size=nw), 0.3)
    for dec in (False, True):
        a, b = po.Kalman(dims, 0.5, 0.98, 0.99, dec, 1e-3), po.Kalman(dims, 0.5, 0.98, 0.99, dec, 1e-3)
        wa, wb = w0.copy(), w0.copy()
        a.iekf_begin(wa)
        a.iekf_iter(wa, J(wa), R(wa), 0.25, True)
        b.update(wb, J(w0), -R(w0), 1.0 / np.sqrt(0.25))
        assert np.array_equal(wa, wb) and np.array_equal(a.P, b.P) and a.lam == b.lam


@pytest.mark.gpu
@pytest.mark.parametrize("decoupled", [False, True])
def test_device_iekf_matches_the_oracle(decoupled):
    from dnnf90_b200 import api
    dims = [3, 20, 20, 1]
    nw = po.weight_count(dims)
    rng = np.random.default_rng(9)
    w0 = rng.normal(size=nw) * 0.5
    net, ts = _net(dims, w0)
    kf = api.Kalman(net, 0.3, 0.98, 0.9987, decoupled, 1e-4, gate=0.5)  # the gate is ignored
    ref = po.Kalman(dims, 0.3, 0.98, 0.9987, decoupled, 1e-4, gate=0.5)
    wref = w0.copy()
    for obs in range(3):
        R, J = _obs(rng.normal(size=nw) / np.sqrt(nw), rng.normal())
        kf.iekf_begin()
        ref.iekf_begin(wref)
        for it in range(3):
            final = it == 2
            wd = net.get_weights()
            kf.iekf_iter(J(wd), R(wd), 0.5, final)
            ref.iekf_iter(wref, J(wref), R(wref), 0.5, final)
            assert rel_err(net.get_weights(), wref) < 1e-11
        assert abs(kf.state()[0] - ref.lam) <= 1e-15
    assert rel_err(kf.cov().reshape(-1), ref.P) < 1e-11
    assert kf.state()[1] == 0
    kf.free(); net.free(); ts.free()


@pytest.mark.gpu
def test_device_iekf_single_final_iteration_is_the_plain_update():
    from dnnf90_b200 import api
    dims = [3, 20, 20, 1]
    nw = po.weight_count(dims)
    rng = np.random.default_rng(10)
    w0 = rng.normal(size=nw) * 0.5
    R, J = _obs(rng.normal(size=nw) / np.sqrt(nw), 0.2)
    na, tsa = _net(dims, w0)
    nb, tsb = _net(dims, w0)
    a, b = api.Kalman(na, 0.3, 0.98, 0.9987), api.Kalman(nb, 0.3, 0.98, 0.9987)
    a.iekf_begin()
    a.iekf_iter(J(w0), R(w0), 0.5, True)
    b.update_rows(J(w0), -R(w0), 1.0 / np.sqrt(0.5))
    assert np.array_equal(na.get_weights(), nb.get_weights())
    assert np.array_equal(a.cov(), b.cov()) and a.state() == b.state()
    with pytest.raises(api.Dnnf90Error):
        a.iekf_iter(J(w0), R(w0), 0.0, True)       # rnoise must be positive
    c = api.Kalman(na, 0.3, 0.98, 0.9987)
    with pytest.raises(api.Dnnf90Error):
        c.iekf_iter(J(w0), R(w0), 0.5, True)       # no prior yet
    for k in (a, b, c):
        k.free()
    na.free(); nb.free(); tsa.free(); tsb.free()


@pytest.mark.gpu
@pytest.mark.parametrize("decoupled", [False, True])
def test_one_launch_and_two_launch_paths_are_bit_identical(decoupled, monkeypatch):
    """The one-launch sequence (cooperative, grid barriers) and the two
    launches per update share the tile code and every summation order, so
    they give the same bits: weights, covariance, lambda and gate count,
    also across staging chunks."""
    from dnnf90_b200 import api
    dims = [3, 20, 20, 1]
    out = []
    try:
        for path in (0, 1):
            api.tune_force(3, path)
            (kf, net, ts), ref, wref, (rows, xi, sc) = _run_both(dims, decoupled, 1e-4, 1.5, 40)
            kf.update_rows(rows[:25], xi[:25], sc[:25])
            monkeypatch.setenv("DNNF90_KF_STAGE_KB", "9")
            kf.update_rows(rows[25:], xi[25:], sc[25:])
            monkeypatch.delenv("DNNF90_KF_STAGE_KB")
            out.append((net.get_weights(), kf.cov(), kf.state()))
            assert rel_err(net.get_weights(), wref) < 1e-11
            kf.free(); net.free(); ts.free()
    finally:
        api.tune_force(3, -1)
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    assert out[0][2] == out[1][2]


# ------------------------------------------------ per-point pass on the device


@pytest.mark.gpu
@pytest.mark.parametrize("decoupled", [False, True])
def test_device_filter_pass_matches_the_oracle_loop(decoupled):
    """dnnf90_kf_pass: for each point its row dR/dw and R at the weights the
    previous update left, then the update with xi = -R; against the oracle
    running the same loop (its rows from the oracle's adjoint)."""
    from dnnf90_b200 import api
    dims = [2, 16, 16, 1]
    ts = api.TableSet(2, 3, [[0, 1], [1, 0], [3, 0]])
    tab = po.Tables(2, 3, [[0, 1], [1, 0], [3, 0]])
    terms = [(1.0, ts.slot((0, 1)), 0), (6.0, ts.slot((1, 0)), 1), (1.0, ts.slot((3, 0)), 0)]
    w0 = np.random.default_rng(31).normal(size=po.weight_count(dims)) * 0.4
    X = np.random.default_rng(32).uniform(-1, 1, (30, 2))
    net = api.Net(ts, dims, weights=w0)
    rule = api.SeedRule(api.SEED_JROW, terms)
    kf = api.Kalman(net, 0.5, 0.98, 0.9987, decoupled, 1e-4, gate=2.0)
    kf.pass_points(X, rule, rnoise=0.25)
    ref = po.Kalman(dims, 0.5, 0.98, 0.9987, decoupled, 1e-4, gate=2.0)
    w = w0.copy()
    for x in X:
        _, T, _, rows = po.grad_batch(tab, dims, w, x[None, :], kind=po.SEED_JROW, terms=terms)
        R = sum(c * (T[0, 0] * T[0, s - 1] if nl else T[0, s - 1]) for c, s, nl in terms)
        ref.update(w, rows[0], -R, 1.0 / np.sqrt(0.25))
    assert rel_err(net.get_weights(), w) < 1e-10, rel_err(net.get_weights(), w)
    assert rel_err(kf.cov().reshape(-1), ref.P) < 1e-10
    lam, ng = kf.state()
    assert abs(lam - ref.lam) <= 1e-15 and ng == ref.ngated.value
    with pytest.raises(api.Dnnf90Error):
        kf.pass_points(X[:2], rule, rnoise=0.0)
    net.set_precision(api.PREC_SPLIT)
    with pytest.raises(api.Dnnf90Error):                  # the pass runs in FP64 only
        kf.pass_points(X[:2], rule)
    kf.free(); rule.free(); net.free(); ts.free()


@pytest.mark.gpu
@pytest.mark.parametrize("niter", [1, 3])
def test_device_iterated_pass_matches_the_oracle(niter):
    """dnnf90_kf_pass_iekf against the oracle's kf_iekf_begin / kf_iekf_iter
    loop, each relinearisation from the oracle's row and residual at the
    current weights; one iteration is the plain pass."""
    from dnnf90_b200 import api
    dims = [2, 16, 16, 1]
    ts = api.TableSet(2, 3, [[0, 1], [1, 0], [3, 0]])
    tab = po.Tables(2, 3, [[0, 1], [1, 0], [3, 0]])
    terms = [(1.0, ts.slot((0, 1)), 0), (6.0, ts.slot((1, 0)), 1), (1.0, ts.slot((3, 0)), 0)]
    w0 = np.random.default_rng(41).normal(size=po.weight_count(dims)) * 0.4
    X = np.random.default_rng(42).uniform(-1, 1, (20, 2))
    net = api.Net(ts, dims, weights=w0)
    rule = api.SeedRule(api.SEED_JROW, terms)
    kf = api.Kalman(net, 0.5, 0.98, 0.9987, False, 1e-4)
    kf.pass_points(X, rule, rnoise=0.25, niter=niter)
    ref = po.Kalman(dims, 0.5, 0.98, 0.9987, False, 1e-4)
    w = w0.copy()
    for x in X:
        ref.iekf_begin(w)
        for it in range(niter):
            _, T, _, rows = po.grad_batch(tab, dims, w, x[None, :], kind=po.SEED_JROW,
                                          terms=terms)
            R = sum(c * (T[0, 0] * T[0, s - 1] if nl else T[0, s - 1]) for c, s, nl in terms)
            ref.iekf_iter(w, rows[0], R, 0.25, it == niter - 1)
    assert rel_err(net.get_weights(), w) < 1e-10, rel_err(net.get_weights(), w)
    assert rel_err(kf.cov().reshape(-1), ref.P) < 1e-10
    assert abs(kf.state()[0] - ref.lam) <= 1e-15
    if niter == 1:   # one iteration per point is the plain pass
        net2 = api.Net(ts, dims, weights=w0)
        kf2 = api.Kalman(net2, 0.5, 0.98, 0.9987, False, 1e-4)
        kf2.pass_points(X, rule, rnoise=0.25)
        assert rel_err(net2.get_weights(), net.get_weights()) < 1e-13
        kf2.free(); net2.free()
    with pytest.raises(api.Dnnf90Error):
        api.call("dnnf90_kf_pass_iekf", kf.kid, net.tid, 1, api._pd(X), rule.rid, 0.25, 0)
    kf.free(); rule.free(); net.free(); ts.free()


# ------------------------------------------------ systems of residuals


def _sys_terms(slot):
    """Two residuals over outputs (u, v): u u_x + v_y and u_y - v v_x + 0.3 u_xx."""
    s = {k: slot(v) for k, v in dict(v0=(0, 0), x=(1, 0), y=(0, 1), xx=(2, 0)).items()}
    U, V = 1, 2
    return [(1, 1.0, [(U, s["v0"]), (U, s["x"])]), (1, 1.0, [(V, s["y"])]),
            (2, 1.0, [(U, s["y"])]), (2, -1.0, [(V, s["v0"]), (V, s["x"])]),
            (2, 0.3, [(U, s["xx"])])]


def _oracle_sys_obs(tab, dims, w, x, terms, ir, src):
    """R_ir at the weights w, and the row dR_ir/dw by the oracle's adjoint
    seeded with dR_ir/dT (set_sys_seed with a one in slot ir, unweighted)."""
    _, tall = po.eval_point(tab, dims, w, x)
    T = lambda f: tall[f[0] - 1, f[1] - 1]
    R = -src[ir - 1] if src is not None else 0.0
    seed = np.zeros_like(tall)
    for r, c, fs in terms:
        if r != ir:
            continue
        R += c * np.prod([T(f) for f in fs])
        for m, f in enumerate(fs):
            seed[f[0] - 1, f[1] - 1] += c * np.prod([T(g) for mm, g in enumerate(fs) if mm != m])
    row, _ = po.grad_point(tab, dims, w, x, seed)
    return R, row


@pytest.mark.gpu
@pytest.mark.parametrize("niter", [0, 2])
def test_device_system_pass_matches_the_oracle_loop(niter):
    """dnnf90_kf_pass_sys: each point's residuals in turn, each re-evaluated
    at the weights the previous update left, with per-residual noise; the
    oracle runs the trainer's loop (app/sgd_batch_module.f90:497-545)."""
    from dnnf90_b200 import api
    dims = [2, 16, 16, 2]
    ts = api.TableSet(2, 2)
    tab = po.Tables(2, 2)
    terms = _sys_terms(ts.slot)
    w0 = np.random.default_rng(51).normal(size=po.weight_count(dims)) * 0.4
    X = np.random.default_rng(52).uniform(-1, 1, (12, 2))
    src = np.random.default_rng(53).normal(size=(12, 2)) * 0.1
    rnoise = np.array([0.5, 2.0])
    net = api.Net(ts, dims, weights=w0)
    rule = api.SeedRule.system(2, terms)
    kf = api.Kalman(net, 0.5, 0.98, 0.9987, False, 1e-4)
    kf.pass_system(X, rule, src=src, rnoise=rnoise, niter=niter)
    ref = po.Kalman(dims, 0.5, 0.98, 0.9987, False, 1e-4)
    w = w0.copy()
    for p, x in enumerate(X):
        for ir in (1, 2):
            if niter == 0:
                R, row = _oracle_sys_obs(tab, dims, w, x, terms, ir, src[p])
                ref.update(w, row, -R, 1.0 / np.sqrt(rnoise[ir - 1]))
                continue
            ref.iekf_begin(w)
            for it in range(niter):
                R, row = _oracle_sys_obs(tab, dims, w, x, terms, ir, src[p])
                ref.iekf_iter(w, row, R, rnoise[ir - 1], it == niter - 1)
    assert rel_err(net.get_weights(), w) < 1e-10, rel_err(net.get_weights(), w)
    assert rel_err(kf.cov().reshape(-1), ref.P) < 1e-10
    assert abs(kf.state()[0] - ref.lam) <= 1e-15
    with pytest.raises(api.Dnnf90Error):
        kf.pass_system(X[:1], rule, rnoise=[1.0, 0.0])
    jr = api.SeedRule(api.SEED_JROW, [(1.0, ts.slot((1, 0)), 0)])
    with pytest.raises(api.Dnnf90Error):                    # a system rule is needed
        kf.pass_system(X[:1], jr)
    kf.free(); jr.free(); rule.free(); net.free(); ts.free()


@pytest.mark.gpu
def test_device_entry_captured_in_a_cuda_graph():
    """Under stream capture the update takes the two-launch path and returns
    without waiting; one replay applies the same updates, to the bit, as a
    direct call (which takes the one-launch path at this size)."""
    import torch
    from dnnf90_b200 import api
    dims = [3, 20, 20, 1]
    (kfa, neta, tsa), _, _, (rows, xi, sc) = _run_both(dims, False, 1e-4, 1.5, 24)
    (kfb, netb, tsb), _, _, _ = _run_both(dims, False, 1e-4, 1.5, 24)
    dev = torch.device("cuda", 0)
    rd, xd, sd = (torch.tensor(a, device=dev) for a in (rows, xi, sc))
    wa = torch.tensor(neta.get_weights(), device=dev)
    wb = wa.clone()
    api.call("dnnf90_kf_update_rows_dev", kfa.kid, len(xi), rd.data_ptr(), xd.data_ptr(),
             sd.data_ptr(), wa.data_ptr(), torch.cuda.current_stream(dev).cuda_stream)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        api.call("dnnf90_kf_update_rows_dev", kfb.kid, len(xi), rd.data_ptr(), xd.data_ptr(),
                 sd.data_ptr(), wb.data_ptr(), torch.cuda.current_stream(dev).cuda_stream)
    g.replay()
    torch.cuda.synchronize(dev)
    assert api.lib().dnnf90_kf_status(kfb.kid) == 0
    assert torch.equal(wa, wb)
    assert np.array_equal(kfa.cov(), kfb.cov()) and kfa.state() == kfb.state()
    del g
    for kf, net, ts in ((kfa, neta, tsa), (kfb, netb, tsb)):
        kf.free(); net.free(); ts.free()
