"""ctypes binding of the CPU FP64 oracle (oracle.c).

TEST INFRASTRUCTURE ONLY.  Imported by the tests, by
``__graft_entry__.smoke()`` and by the ``cpu_baseline`` leg of ``bench.py``
as the checker of the CUDA path; the product package never imports it.

The oracle restates the reference's table construction
(lib/multi_index_bell_module.f90:128-429), its forward pass
(lib/train_module.f90:241-335, lib/net_module.f90:295-375), its adjoint
(lib/train_module.f90:360-450), the residual seeds of app/pinn_module.f90:
32-65 and of its systems (:86-162), the Adam step (lib/train_module.f90:656-683) and the primal natural
gradient step (app/optimizer_module.f90:221-522).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "liboracle.so")

SEED_GIVEN, SEED_HALFSQ, SEED_PINN, SEED_JROW = 0, 1, 2, 3

_lib = None


def build() -> str:
    """Compile the oracle with its Makefile (gcc, no FMA contraction)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO) or (
            os.path.getmtime(_SO) < os.path.getmtime(os.path.join(_HERE, "oracle.c"))
        ):
            build()
        L = ctypes.CDLL(_SO)
        P = ctypes.POINTER
        ci, cd, vp = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
        L.orc_tables_build.restype = vp
        L.orc_tables_build.argtypes = [ci, ci, ci, P(ci)]
        L.orc_tables_free.argtypes = [vp]
        L.orc_tables_sizes.argtypes = [vp, P(ci), P(ci), P(ci), P(ci)]
        L.orc_tables_copy.argtypes = [vp] + [vp] * 14
        L.orc_tanh_derivs.argtypes = [vp, cd, ci, vp]
        L.orc_act_derivs.argtypes = [vp, cd, ci, vp]
        L.orc_besj_all.argtypes = [ci, cd, vp]
        L.orc_kf_update.argtypes = [ci, vp, vp, ci, vp, vp, vp, cd, cd, vp, cd, cd, cd, vp]
        L.orc_kf_iekf_iter.argtypes = [ci, vp, vp, vp, ci, vp, vp, vp, cd, cd, vp, cd, cd, ci]
        L.orc_tables_set_activation.argtypes = [vp, ci]
        L.orc_weight_count.argtypes = [ci, P(ci)]
        L.orc_eval_point.argtypes = [vp, ci, P(ci), vp, vp, vp, vp]
        L.orc_grad_point.argtypes = [vp, ci, P(ci), vp, vp, vp, vp, vp]
        L.orc_grad_batch.argtypes = [vp, ci, P(ci), vp, ci, vp, vp, vp, vp, vp,
                                     vp, vp, ci]
        L.orc_eval_batch.argtypes = [vp, ci, P(ci), vp, ci, vp, vp, ci]
        L.orc_grad_sys_batch.argtypes = [vp, ci, P(ci), vp, ci, vp, vp, vp, vp, vp, vp, ci]
        L.orc_adam_step.argtypes = [ci, vp, vp, vp, vp, cd, cd, cd, cd, ci, ci]
        L.orc_ngd_step.argtypes = [ci, ci, vp, vp, ci, cd, vp]
        L.orc_ngd_metric.argtypes = [ci, ci, vp, vp]
        L.orc_ngd_metric.restype = None
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


class _SeedRule(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("nterm", ctypes.c_int),
                ("coeff", ctypes.c_void_p), ("ind", ctypes.c_void_p),
                ("nonlin", ctypes.c_void_p), ("fac", ctypes.c_double)]


class _SysRule(ctypes.Structure):
    _fields_ = [("nres", ctypes.c_int), ("nterm", ctypes.c_int),
                ("res", ctypes.c_void_p), ("coeff", ctypes.c_void_p),
                ("nfac", ctypes.c_void_p), ("comp", ctypes.c_void_p),
                ("slot", ctypes.c_void_p), ("wres", ctypes.c_void_p),
                ("fac", ctypes.c_double)]


class Tables:
    """One multi-index table set (init_hod_tables)."""

    def __init__(self, d0: int, k: int, seeds=None, activation: int = 0):
        L = lib()
        self.d0, self.k = d0, k
        if seeds is None or len(seeds) == 0:
            h = L.orc_tables_build(d0, k, 0, None)
        else:
            s = np.ascontiguousarray(np.asarray(seeds, dtype=np.int32).reshape(-1))
            h = L.orc_tables_build(d0, k, len(s) // d0,
                                   s.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        if not h:
            raise ValueError("oracle: bad table arguments")
        self._h = h
        if activation and L.orc_tables_set_activation(h, int(activation)) != 0:
            raise ValueError("oracle: activation not restated")
        self.activation = int(activation)
        na, nfq, npair, nbell = (ctypes.c_int(), ctypes.c_int(), ctypes.c_int(),
                                 ctypes.c_int())
        L.orc_tables_sizes(h, ctypes.byref(na), ctypes.byref(nfq),
                           ctypes.byref(npair), ctypes.byref(nbell))
        self.na, self.nfq, self.npair, self.nbell = (na.value, nfq.value,
                                                     npair.value, nbell.value)
        kk = max(k - 1, 0)
        self.alpha = np.zeros((self.na, d0), np.int32)
        self.deg = np.zeros(self.na, np.int32)
        self.ind_e1 = np.zeros(d0, np.int32)
        self.fq_start = np.zeros((self.na, kk), np.int32)
        self.fq_num = np.zeros((self.na, kk), np.int32)
        self.fq_ib = np.zeros(max(self.nfq, 1), np.int32)
        self.fq_id = np.zeros(max(self.nfq, 1), np.int32)
        self.fq_c = np.zeros(max(self.nfq, 1), np.float64)
        self.pair_start = np.zeros(self.na, np.int32)
        self.pair_num = np.zeros(self.na, np.int32)
        self.pair_ia = np.zeros(max(self.npair, 1), np.int32)
        self.pair_id = np.zeros(max(self.npair, 1), np.int32)
        self.pair_binom = np.zeros(max(self.npair, 1), np.float64)
        self.tpc = np.zeros((k + 2, k + 3), np.float64)
        L.orc_tables_copy(h, *[_p(a) for a in (
            self.alpha, self.deg, self.ind_e1, self.fq_start, self.fq_num,
            self.fq_ib, self.fq_id, self.fq_c, self.pair_start, self.pair_num,
            self.pair_ia, self.pair_id, self.pair_binom, self.tpc)])

    def __del__(self):
        try:
            lib().orc_tables_free(self._h)
        except Exception:
            pass

    def slot(self, a) -> int:
        """1-based slot of multi-index a (0 if not carried)."""
        a = tuple(int(v) for v in a)
        for i, b in enumerate(self.alpha):
            if tuple(int(v) for v in b) == a:
                return i + 1
        return 0

    def act_derivs(self, a: float, nq: int) -> np.ndarray:
        d = np.zeros(nq + 1)
        lib().orc_act_derivs(self._h, float(a), nq, _p(d))
        return d

    def tanh_derivs(self, a: float, nq: int) -> np.ndarray:
        d = np.zeros(nq + 1)
        lib().orc_tanh_derivs(self._h, float(a), nq, _p(d))
        return d


def _dims(dims):
    d = (ctypes.c_int * len(dims))(*[int(v) for v in dims])
    return d


def weight_count(dims) -> int:
    return int(sum(dims[l] * (dims[l - 1] + 1) for l in range(1, len(dims))))


def eval_point(tab: Tables, dims, w, x):
    t = np.zeros(tab.na)
    tall = np.zeros((dims[-1], tab.na))
    w = np.ascontiguousarray(w, np.float64)
    x = np.ascontiguousarray(x, np.float64)
    rc = lib().orc_eval_point(tab._h, len(dims), _dims(dims), _p(w), _p(x),
                              _p(t), _p(tall))
    if rc != 0:
        raise ValueError("oracle eval: bad shape")
    return t, tall


def grad_point(tab: Tables, dims, w, x, seedm):
    """Forward + adjoint of one point; seedm [nout][na] or [na]."""
    g = np.zeros(weight_count(dims))
    t = np.zeros(tab.na)
    s = np.zeros((dims[-1], tab.na))
    sm = np.asarray(seedm, np.float64)
    s.reshape(-1)[: sm.size] = sm.reshape(-1)
    w = np.ascontiguousarray(w, np.float64)
    x = np.ascontiguousarray(x, np.float64)
    rc = lib().orc_grad_point(tab._h, len(dims), _dims(dims), _p(w), _p(x),
                              _p(s), _p(g), _p(t))
    if rc != 0:
        raise ValueError("oracle grad: bad shape")
    return g, t


def _rule(kind, terms=(), fac=1.0):
    coeff = np.array([t[0] for t in terms] or [0.0], np.float64)
    ind = np.array([t[1] for t in terms] or [1], np.int32)
    nonlin = np.array([int(t[2]) for t in terms] or [0], np.int32)
    r = _SeedRule(kind, len(terms), _p(coeff), _p(ind), _p(nonlin), float(fac))
    return r, (coeff, ind, nonlin)


def grad_batch(tab: Tables, dims, w, X, kind=SEED_HALFSQ, terms=(), fac=1.0,
               seeds=None, nthreads=0, want_t=True):
    """Batched forward + seed + adjoint.  Returns (grad, T, loss, rows).

    terms: (coeff, slot, nonlin) triples for SEED_PINN / SEED_JROW.
    """
    X = np.ascontiguousarray(X, np.float64)
    npts = X.shape[0]
    nw = weight_count(dims)
    g = np.zeros(nw)
    T = np.zeros((npts, tab.na)) if want_t else None
    rows = np.zeros((npts, nw)) if kind == SEED_JROW else None
    sd = np.ascontiguousarray(seeds, np.float64) if seeds is not None else None
    loss = ctypes.c_double(0.0)
    r, keep = _rule(kind, terms, fac)
    w = np.ascontiguousarray(w, np.float64)
    rc = lib().orc_grad_batch(tab._h, len(dims), _dims(dims), _p(w), npts,
                              _p(X), ctypes.byref(r), _p(sd), _p(g),
                              _p(rows), _p(T), ctypes.byref(loss), nthreads)
    if rc != 0:
        raise ValueError("oracle grad_batch: bad arguments")
    return g, T, loss.value, rows


def grad_sys_batch(tab: Tables, dims, w, X, nres, terms, wres=None, fac=1.0, src=None,
                   nthreads=0, want_t=True):
    """Forward + system seed + adjoint (calc_sys_residual / set_sys_seed).

    terms: (residual, coeff, [(component, slot), ...]) with 1-based residual,
    component and slot.  src[npts][nres] may be None.  Returns (grad,
    T[npts][nout][na] or None, loss)."""
    X = np.ascontiguousarray(X, np.float64)
    npts, nout = X.shape[0], dims[-1]
    res = np.array([t[0] for t in terms], np.int32)
    coeff = np.array([t[1] for t in terms], np.float64)
    nfac = np.array([len(t[2]) for t in terms], np.int32)
    comp = np.array([f[0] for t in terms for f in t[2]], np.int32)
    slot = np.array([f[1] for t in terms for f in t[2]], np.int32)
    wr = np.ascontiguousarray(wres, np.float64) if wres is not None else None
    r = _SysRule(nres, len(terms), _p(res), _p(coeff), _p(nfac), _p(comp), _p(slot), _p(wr),
                 float(fac))
    sv = np.ascontiguousarray(src, np.float64) if src is not None else None
    g = np.zeros(weight_count(dims))
    T = np.zeros((npts, nout, tab.na)) if want_t else None
    loss = ctypes.c_double(0.0)
    w = np.ascontiguousarray(w, np.float64)
    rc = lib().orc_grad_sys_batch(tab._h, len(dims), _dims(dims), _p(w), npts, _p(X),
                                  ctypes.byref(r), _p(sv), _p(g), _p(T), ctypes.byref(loss),
                                  nthreads)
    if rc != 0:
        raise ValueError("oracle grad_sys_batch: bad arguments")
    return g, T, loss.value


def besj_all(n: int, x: float) -> np.ndarray:
    """J_0(x) .. J_n(x) (the oracle's Miller recurrence)."""
    bj = np.zeros(n + 1)
    lib().orc_besj_all(int(n), float(x), _p(bj))
    return bj


class Kalman:
    """The reference's extended Kalman filter (kalman_t, kf_init,
    kf_update_grad; lib/kalman_module.f90) over the flat weights."""

    def __init__(self, dims, p0, lam_ini, lam0, decoupled=False, q=0.0, gate=0.0):
        self.nw = weight_count(dims)
        self.lam, self.lam0, self.q, self.gate = float(lam_ini), float(lam0), float(q), float(gate)
        self.ngated = ctypes.c_int(0)
        if decoupled:  # one block per neuron over (bias, fan-in), kf_block_map
            self.bsz = np.array([dims[l - 1] + 1 for l in range(1, len(dims))
                                 for _ in range(dims[l])], np.int32)
            self.boff = np.concatenate([[0], np.cumsum(self.bsz)[:-1]]).astype(np.int32)
            self.P = np.concatenate([p0 * np.eye(n).reshape(-1) for n in self.bsz])
        else:
            self.bsz = self.boff = None
            self.P = p0 * np.eye(self.nw).reshape(-1)

    def update(self, w, jrow, xi, scale=1.0):
        """One observation: w (float64, updated in place), jrow = dy/dw."""
        assert w.dtype == np.float64 and w.flags.c_contiguous
        lam = ctypes.c_double(self.lam)
        jr = np.ascontiguousarray(jrow, np.float64)
        nb = 0 if self.bsz is None else len(self.bsz)
        rc = lib().orc_kf_update(self.nw, _p(w), _p(self.P), nb, _p(self.bsz), _p(self.boff),
                                 _p(jr), float(xi), float(scale), ctypes.byref(lam), self.lam0,
                                 self.q, self.gate, ctypes.byref(self.ngated))
        if rc != 0:
            raise ValueError("oracle kf_update: nonpositive innovation denominator")
        self.lam = lam.value

    def iekf_begin(self, w):
        """kf_iekf_begin: the prior is the current weights."""
        self.wprior = np.array(w, np.float64)

    def iekf_iter(self, w, jrow, resid, rnoise, final):
        """kf_iekf_iter: one relinearisation from jrow = dR/dw and R at the
        current weights w (updated in place)."""
        assert w.dtype == np.float64 and w.flags.c_contiguous
        lam = ctypes.c_double(self.lam)
        jr = np.ascontiguousarray(jrow, np.float64)
        nb = 0 if self.bsz is None else len(self.bsz)
        rc = lib().orc_kf_iekf_iter(self.nw, _p(w), _p(self.wprior), _p(self.P), nb,
                                    _p(self.bsz), _p(self.boff), _p(jr), float(resid),
                                    float(rnoise), ctypes.byref(lam), self.lam0, self.q,
                                    int(bool(final)))
        if rc != 0:
            raise ValueError("oracle kf_iekf_iter: bad noise or nonpositive denominator")
        self.lam = lam.value


def eval_batch(tab: Tables, dims, w, X, nthreads=0):
    X = np.ascontiguousarray(X, np.float64)
    T = np.zeros((X.shape[0], tab.na))
    w = np.ascontiguousarray(w, np.float64)
    rc = lib().orc_eval_batch(tab._h, len(dims), _dims(dims), _p(w), X.shape[0],
                              _p(X), _p(T), nthreads)
    if rc != 0:
        raise ValueError("oracle eval_batch: bad arguments")
    return T


def adam_step(w, g, m, v, eta, b1, b2, eps, nbatch, istep):
    for a in (w, m, v):
        assert a.dtype == np.float64 and a.flags.c_contiguous
    g = np.ascontiguousarray(g, np.float64)
    lib().orc_adam_step(len(w), _p(w), _p(g), _p(m), _p(v), eta, b1, b2, eps,
                        nbatch, istep)


def ngd_step(rows, b, nb, mu):
    rows = np.ascontiguousarray(rows, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    u = np.zeros(rows.shape[1])
    rc = lib().orc_ngd_step(rows.shape[1], rows.shape[0], _p(rows), _p(b), nb,
                            mu, _p(u))
    if rc != 0:
        raise ValueError("oracle ngd: singular metric")
    return u


def ngd_metric(rows):
    """G = J^T J in the reference's loop order (app/optimizer_module.f90:
    310-321), undivided."""
    rows = np.ascontiguousarray(rows, np.float64)
    G = np.zeros((rows.shape[1], rows.shape[1]))
    lib().orc_ngd_metric(rows.shape[1], rows.shape[0], _p(rows), _p(G))
    return G


def check_weights(dims) -> np.ndarray:
    """The deterministic weights of the reference's self-check,
    w(l,j,i) = 0.1 sin(1.7 l + 0.9 j + 0.3 i) + 0.05
    (app/hod_check_module.f90:100-107), in the flat layer layout."""
    out = []
    for l in range(2, len(dims) + 1):
        for j in range(1, dims[l - 1] + 1):
            for i in range(0, dims[l - 2] + 1):
                out.append(0.1 * math.sin(1.7 * l + 0.9 * j + 0.3 * i) + 0.05)
    return np.array(out, np.float64)
