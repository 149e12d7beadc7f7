"""The natural-gradient step through the entry point that allocates no
device memory (dnnf90_ngd_step_noalloc), for hosts that cannot allocate
while they run, checked against dnnf90_ngd_step on the same system.

Collected last, so a run that stops at its first failure has already run
every other test; it passes alone in a fresh process as well."""
import numpy as np
import pytest

from dnnf90_b200 import api

pytestmark = pytest.mark.gpu


def test_noalloc_ngd_matches_the_allocating_entry():
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
    dev = torch.device("cuda", 0)
    Jd = torch.tensor(J, device=dev)
    bd = torch.tensor(b, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for _ in range(2):  # the second call sees the first call's leftovers
        ud = torch.full((nw,), float("nan"), dtype=torch.float64, device=dev)
        api.call("dnnf90_ngd_step_noalloc", nrow, nw, Jd.data_ptr(), bd.data_ptr(), nb, mu,
                 ud.data_ptr(), stream)
        u = ud.cpu().numpy()
        assert np.all(np.isfinite(u))
        err = np.max(np.abs(u - u_ref)) / np.max(np.abs(u_ref))
        assert err < 1e-10, err
    # a size beyond the fixed scratch is refused with a message
    big = 1025
    rc = api.lib().dnnf90_ngd_step_noalloc(1, big, Jd.data_ptr(), bd.data_ptr(), 1, mu,
                                           ud.data_ptr(), stream)
    assert rc == -1
    assert b"scratch" in api.lib().dnnf90_last_error()
    net.free()
