"""The torch.autograd.Function over the device library (KdV-style PINN step).

Workload: D0=2 (x, t), K=3, carried set = downward closure of
{(0,1), (1,0), (3,0)}, MLP 2-64-64-64-1 tanh, 16384 points uniform on
[-10,10] x [0,1], residual R = u_t + 6 u u_x + u_xxx, L = sum R^2 / 2.

The adjoint gradient is checked three ways, as the reference checks its own
(app/hod_check_module.f90): against the oracle's gradient, against central
finite differences of the full loss along random directions, and against a
nested-autograd reference that differentiates a plain torch MLP three times.
"""
import numpy as np
import pytest

from conftest import per_order_error, rel_err, xavier_weights
from dnnf90_b200 import api
from dnnf90_b200.autograd import hod
import pyoracle as po

pytestmark = pytest.mark.gpu

D0, K = 2, 3
SEEDS = [[0, 1], [1, 0], [3, 0]]
DIMS = [2, 64, 64, 64, 1]
NPTS = 16384
TOL64 = 1e-12
TOLSPLIT = 1e-5


def _points(n, seed=11):
    rng = np.random.default_rng(seed)
    return np.stack([rng.uniform(-10, 10, n), rng.uniform(0, 1, n)], axis=1)


def _weights():
    w = xavier_weights(DIMS, 21)
    w[np.arange(len(w)) % 7 == 0] += 0.03  # non-zero biases
    return w


def _setup(prec):
    ts = api.TableSet(D0, K, SEEDS)
    net = api.Net(ts, DIMS, precision=prec)
    slots = dict(t=ts.slot([0, 1]) - 1, x=ts.slot([1, 0]) - 1, xxx=ts.slot([3, 0]) - 1)
    return ts, net, slots


def _residual(T, s):
    u = T[:, 0, 0]
    return T[:, 0, s["t"]] + 6.0 * u * T[:, 0, s["x"]] + T[:, 0, s["xxx"]]


def _loss_and_grad(net, slots, X, w, keep=True):
    import torch
    dev = torch.device("cuda", 0)
    x = torch.tensor(X, device=dev)
    wt = torch.tensor(w, device=dev, requires_grad=True)
    T = hod(x, wt, net, keep=keep)
    L = 0.5 * (_residual(T, slots) ** 2).sum()
    L.backward()
    return float(L.detach()), wt.grad.cpu().numpy(), T.detach().cpu().numpy()


def _oracle(X, w):
    ref = po.Tables(D0, K, SEEDS)
    terms = [(1.0, ref.slot([0, 1]), 0), (6.0, ref.slot([1, 0]), 1), (1.0, ref.slot([3, 0]), 0)]
    g, T, L, _ = po.grad_batch(ref, DIMS, w, X, kind=po.SEED_PINN, terms=terms, fac=1.0)
    return g, T, L, ref


@pytest.mark.parametrize("prec", [api.PREC_F64, api.PREC_SPLIT])
def test_autograd_gradient_matches_the_oracle(prec):
    X, w = _points(NPTS), _weights()
    ts, net, slots = _setup(prec)
    L, g, T = _loss_and_grad(net, slots, X, w)
    gref, Tref, Lref, ref = _oracle(X, w)
    tol = TOL64 if prec == api.PREC_F64 else TOLSPLIT
    assert max(per_order_error(T[:, 0, :], Tref, ref.deg).values()) < tol
    assert rel_err(g, gref) < tol, rel_err(g, gref)
    assert abs(L - Lref) <= tol * abs(Lref)
    net.free()


def test_keep_and_recompute_agree():
    X, w = _points(4096, 5), _weights()
    ts, net, slots = _setup(api.PREC_F64)
    L1, g1, _ = _loss_and_grad(net, slots, X, w, keep=True)
    L2, g2, _ = _loss_and_grad(net, slots, X, w, keep=False)
    assert L1 == L2
    assert rel_err(g2, g1) < 1e-14
    net.free()


def test_automatic_memory_mode():
    """keep=None keeps the planes when every layer's planes for the points
    fit the work space (here: 4096 points of this net, about 40 MB), and
    recomputes when they do not (a 1000-point chunk; 10^9 points); both give
    the store-mode gradient."""
    from dnnf90_b200.autograd import keep_fits
    X, w = _points(4096, 5), _weights()
    ts, net, slots = _setup(api.PREC_F64)
    assert keep_fits(net, 4096)
    assert not keep_fits(net, 10 ** 9)
    L1, g1, _ = _loss_and_grad(net, slots, X, w, keep=True)
    L2, g2, _ = _loss_and_grad(net, slots, X, w, keep=None)
    assert L1 == L2 and rel_err(g2, g1) < 1e-14
    api.call("dnnf90_twork_set_chunk", net.tid, 1000)
    assert not keep_fits(net, 4096)
    L3, g3, _ = _loss_and_grad(net, slots, X, w, keep=None)
    assert abs(L3 - L1) <= 1e-13 * abs(L1) and rel_err(g3, g1) < 1e-13
    net.free()


def test_finite_differences_of_the_full_loss():
    """Central differences of L along random unit directions (the
    directional form of the reference's Hod_check)."""
    import torch
    X, w = _points(2048, 7), _weights()
    ts, net, slots = _setup(api.PREC_F64)
    _, g, _ = _loss_and_grad(net, slots, X, w)
    dev = torch.device("cuda", 0)
    x = torch.tensor(X, device=dev)

    def loss(wv):
        with torch.no_grad():
            T = hod(x, torch.tensor(wv, device=dev), net)
            return float(0.5 * (_residual(T, slots) ** 2).sum())

    rng = np.random.default_rng(3)
    for _ in range(4):
        v = rng.normal(size=w.size)
        v /= np.linalg.norm(v)
        h = 1e-5
        fd = (loss(w + h * v) - loss(w - h * v)) / (2 * h)
        an = float(g @ v)
        assert abs(fd - an) <= 1e-6 * max(abs(an), np.linalg.norm(g) * 1e-3), (fd, an)
    net.free()


def _torch_mlp(x, wt):
    import torch
    h, off = x, 0
    for l in range(1, len(DIMS)):
        m, n = DIMS[l - 1], DIMS[l]
        W = wt[off:off + n * (m + 1)].view(n, m + 1)
        off += n * (m + 1)
        z = h @ W[:, 1:].T + W[:, 0]
        h = torch.tanh(z) if l < len(DIMS) - 1 else z
    return h[:, 0]


def test_nested_autograd_reference():
    """The derivatives and the gradient against torch's own nested autograd
    of the same MLP in FP64 (three levels of create_graph)."""
    import torch
    X, w = _points(NPTS, 13), _weights()
    ts, net, slots = _setup(api.PREC_F64)
    L, g, T = _loss_and_grad(net, slots, X, w)

    dev = torch.device("cuda", 0)
    x = torch.tensor(X, device=dev, requires_grad=True)
    wt = torch.tensor(w, device=dev, requires_grad=True)
    u = _torch_mlp(x, wt)
    (du,) = torch.autograd.grad(u.sum(), x, create_graph=True)
    u_x, u_t = du[:, 0], du[:, 1]
    (d2,) = torch.autograd.grad(u_x.sum(), x, create_graph=True)
    (d3,) = torch.autograd.grad(d2[:, 0].sum(), x, create_graph=True)
    u_xxx = d3[:, 0]
    R = u_t + 6.0 * u * u_x + u_xxx
    Lt = 0.5 * (R ** 2).sum()
    (gt,) = torch.autograd.grad(Lt, wt)

    Tt = np.stack([v.detach().cpu().numpy() for v in (u, u_t, u_x, u_xxx)], axis=1)
    Td = T[:, 0, [0, slots["t"], slots["x"], slots["xxx"]]]
    assert rel_err(Td, Tt) < 1e-11
    assert abs(L - float(Lt.detach())) <= 1e-11 * abs(float(Lt.detach()))
    assert rel_err(g, gt.cpu().numpy()) < 1e-10, rel_err(g, gt.cpu().numpy())
    net.free()
