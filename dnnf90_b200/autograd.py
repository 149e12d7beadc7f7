"""torch.autograd.Function over the device library's C ABI.

``HodFunction.apply(x, w)`` returns the carried derivatives
T[npts][nout][na] of the network at the points x, all computed by the
library's kernels on torch's current CUDA stream; its backward takes
dL/dT (any loss built from those derivatives in torch) and returns dL/dw
through the library's exact analytic adjoint (lib/train_module.f90:
360-450) -- the weights enter through the forward GEMMs and the Bell step,
so no torch op sees them.  dL/dx is not formed (None).

Two memory modes: ``keep=True`` keeps every plane of the forward on the
device for the backward (store mode); ``keep=False`` recomputes the forward
inside the backward, chunk by chunk (recompute mode).  ``keep=None`` (the
default) chooses: store mode when every layer's planes for all the points
fit the work space's budget (``dnnf90_keep_fits``: their size follows from
|A|, that is from D0 and K, the widths and the point count), recompute mode
otherwise -- the case of large K and carried sets.
"""
from __future__ import annotations

import ctypes

import torch

from . import api


def _ptr(t: torch.Tensor):
    return t.data_ptr() if t is not None else None


def _stream():
    return torch.cuda.current_stream().cuda_stream


def keep_fits(net: "api.Net", npts: int) -> bool:
    """Whether a store-mode forward of npts points fits net's work space."""
    fits = ctypes.c_int(0)
    api.call("dnnf90_keep_fits", net.nid, net.tid, npts, ctypes.byref(fits))
    return fits.value == 1


class HodFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x: torch.Tensor, w: torch.Tensor, net: "api.Net", keep):
        if not (x.is_cuda and w.is_cuda):
            raise ValueError("HodFunction runs on CUDA tensors only")
        x = x.detach().to(torch.float64).contiguous()
        w = w.detach().to(torch.float64).contiguous()
        api.call("dnnf90_set_weights_dev", net.nid, _ptr(w), _stream())
        npts = x.shape[0]
        if keep is None:
            keep = keep_fits(net, npts)
        ctx.keep = bool(keep)
        tm = torch.empty((npts, net.na, net.nout), dtype=torch.float64, device=x.device)
        api.call("dnnf90_forward_dev", net.nid, net.tid, npts, _ptr(x), _ptr(tm),
                 1 if keep else 0, _stream())
        ctx.net = net
        ctx.save_for_backward(x, w)
        # [npts][nout][na], the layout of dnnf90_eval_batch_multi
        return tm.permute(0, 2, 1).contiguous()

    @staticmethod
    def backward(ctx, gT: torch.Tensor):
        x, w = ctx.saved_tensors
        net = ctx.net
        seed = gT.detach().to(torch.float64).contiguous()  # [npts][nout][na]
        g = torch.zeros(net.nw, dtype=torch.float64, device=x.device)
        # the weights may have been reset by another forward in between
        api.call("dnnf90_set_weights_dev", net.nid, _ptr(w), _stream())
        api.call("dnnf90_backward_dev", net.nid, net.tid, x.shape[0], _ptr(x), _ptr(seed),
                 _ptr(g), _stream())
        return None, g.to(w.dtype), None, None


def hod(x: torch.Tensor, w: torch.Tensor, net: "api.Net", keep=None):
    """Carried derivatives T[npts][nout][na] with an analytic adjoint in w.
    keep: True (store mode), False (recompute mode) or None (store mode when
    it fits, see keep_fits)."""
    return HodFunction.apply(x, w, net, keep)
