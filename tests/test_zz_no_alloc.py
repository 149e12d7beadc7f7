"""The natural-gradient step through the entry point that allocates no
device memory (dnnf90_ngd_step_noalloc).  It serves hosts that cannot call
the device allocator while they run: a host that hands all device memory
out up front from its own pool, or one held to a fixed device budget.

Each call is checked against the allocating entry dnnf90_ngd_step on the
same system and against the oracle's FP64 step (app/optimizer_module.f90:
221-522), twice in a row, since the second call finds the first call's
leftovers in the shared scratch area; the device's free memory must not
move across a call.  The largest size the fixed area holds (nw = 1024) is
covered, and a larger one, a non-positive damping and a capturing stream
are refused.

Collected last, so a run that stops at its first failure has already run
every other test; it passes alone in a fresh process as well."""
import numpy as np
import pytest

import pyoracle as po
from dnnf90_b200 import api

pytestmark = pytest.mark.gpu


def _noalloc(nrow, nw, Jd, bd, nb, mu, ud, stream):
    return api.lib().dnnf90_ngd_step_noalloc(nrow, nw, Jd.data_ptr(), bd.data_ptr(), nb, mu,
                                             ud.data_ptr(), stream)


def _relerr(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def test_noalloc_ngd_matches_the_allocating_entry_and_the_oracle():
    import torch

    ts = api.TableSet(3, 2, [[1, 0, 0], [0, 2, 0], [0, 0, 2]])
    dims = [3, 16, 16, 1]
    net = api.Net(ts, dims)
    nw = net.nw
    rng = np.random.default_rng(17)
    nrow, nb, mu = 600, 600, 1e-2
    J = rng.normal(size=(nrow, nw))
    b = rng.normal(size=nw)
    u_ref = api.ngd_step(net, J, b, nb, mu, api.PREC_F64)
    u_orc = po.ngd_step(J, b, nb, mu)
    dev = torch.device("cuda", 0)
    Jd = torch.tensor(J, device=dev)
    bd = torch.tensor(b, device=dev)
    ud = torch.full((nw,), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):  # the second call sees the first call's leftovers
        ud.fill_(float("nan"))
        torch.cuda.synchronize(dev)
        free0 = torch.cuda.mem_get_info(dev)[0]
        assert _noalloc(nrow, nw, Jd, bd, nb, mu, ud, stream) == 0, api.lib().dnnf90_last_error()
        torch.cuda.synchronize(dev)
        free1 = torch.cuda.mem_get_info(dev)[0]
        if call == 1:  # the first call may load the module (and back the area)
            assert free1 == free0, (free0, free1)
        u = ud.cpu().numpy()
        assert np.all(np.isfinite(u))
        assert _relerr(u, u_ref) < 1e-10
        assert _relerr(u, u_orc) < 1e-10
    net.free()


def test_noalloc_ngd_at_the_largest_size():
    import torch

    nw, nrow, nb, mu = 1024, 700, 700, 1e-3
    rng = np.random.default_rng(23)
    J = rng.normal(size=(nrow, nw)) / np.sqrt(nw)
    b = rng.normal(size=nw)
    u_orc = po.ngd_step(J, b, nb, mu)
    dev = torch.device("cuda", 0)
    Jd, bd = torch.tensor(J, device=dev), torch.tensor(b, device=dev)
    ud = torch.empty(nw, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for _ in range(2):
        ud.fill_(float("nan"))
        assert _noalloc(nrow, nw, Jd, bd, nb, mu, ud, stream) == 0, api.lib().dnnf90_last_error()
        u = ud.cpu().numpy()
        assert _relerr(u, u_orc) < 1e-9, _relerr(u, u_orc)


def test_noalloc_ngd_refusals():
    import torch

    dev = torch.device("cuda", 0)
    nw, nrow = 40, 8
    Jd = torch.ones((nrow, 1025), dtype=torch.float64, device=dev)
    bd = torch.ones(1025, dtype=torch.float64, device=dev)
    ud = torch.zeros(1025, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    # a size beyond the fixed area
    assert _noalloc(1, 1025, Jd, bd, 1, 1e-3, ud, stream) == -1
    assert b"scratch" in api.lib().dnnf90_last_error()
    # a damping that is not positive
    assert _noalloc(nrow, nw, Jd, bd, nrow, 0.0, ud, stream) == -1
    assert b"mu" in api.lib().dnnf90_last_error()
    # a stream being captured: refused before anything is enqueued
    s = torch.cuda.Stream(dev)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        rc = _noalloc(nrow, nw, Jd, bd, nrow, 1e-3, ud, s.cuda_stream)
    assert rc == -5
    assert b"captured" in api.lib().dnnf90_last_error()
    del g
