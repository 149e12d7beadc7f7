"""Python host side of the device library: a ctypes binding of dnnf90.h and
dnnf90_b200.h, and a small object layer over the handles.

The raw functions keep the reference's names, argument meaning and return
codes (lib/dnnf90.h; the reference's own Python host is tools/example_py.py,
which binds the same symbols through ctypes).  The object layer raises
``Dnnf90Error`` on a negative code.

The library is loaded from dnnf90_b200/_lib; there is no other
implementation to fall back to, so a missing library is an error.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libdnnf90_b200.so")

PREC_F64 = 0
PREC_SPLIT = 1
SEED_HALFSQ, SEED_PINN, SEED_JROW, SEED_SYS = 1, 2, 3, 4

# the symbols the headers declare (include/dnnf90.h, include/dnnf90_b200.h)
REFERENCE_SYMBOLS = [
    "dnnf90_tables_init_dense", "dnnf90_tables_init_closure", "dnnf90_nderiv",
    "dnnf90_alpha", "dnnf90_tabset_dense", "dnnf90_tabset_closure",
    "dnnf90_tabset_nderiv", "dnnf90_net_create_ts", "dnnf90_net_load",
    "dnnf90_tabset_activation", "dnnf90_net_load_ts", "dnnf90_net_create",
    "dnnf90_net_set_layer", "dnnf90_net_free", "dnnf90_work_create",
    "dnnf90_work_free", "dnnf90_eval", "dnnf90_twork_create",
    "dnnf90_twork_free", "dnnf90_grad_create", "dnnf90_grad_free",
    "dnnf90_grad_zero", "dnnf90_grad_point", "dnnf90_adam_step",
]
EXTENSION_SYMBOLS = [
    "dnnf90_net_set_precision", "dnnf90_nweights", "dnnf90_net_get_layer",
    "dnnf90_net_save", "dnnf90_eval_batch", "dnnf90_eval_batch_multi",
    "dnnf90_grad_batch", "dnnf90_seed_rule_create", "dnnf90_seed_rule_free",
    "dnnf90_grad_rule_batch", "dnnf90_jrow_batch", "dnnf90_grad_read",
    "dnnf90_ngd_step", "dnnf90_set_weights_dev", "dnnf90_forward_dev",
    "dnnf90_backward_dev", "dnnf90_grad_rule_dev", "dnnf90_jrow_dev",
    "dnnf90_twork_set_chunk", "dnnf90_last_error", "dnnf90_device_available",
    "dnnf90_launch_count", "dnnf90_profile_enable", "dnnf90_profile_read",
    "dnnf90_ngd_step_noalloc", "dnnf90_committee_step", "dnnf90_committee_info",
    "dnnf90_tune_report", "dnnf90_tune_force", "dnnf90_tabset_free",
    "dnnf90_seed_rule_sys", "dnnf90_grad_sys_batch", "dnnf90_grad_value_batch",
    "dnnf90_ngd_step_dual", "dnnf90_kf_create", "dnnf90_kf_free", "dnnf90_kf_update_rows",
    "dnnf90_kf_update_rows_dev", "dnnf90_kf_read", "dnnf90_kf_iekf_begin",
    "dnnf90_kf_iekf_iter", "dnnf90_ngd_gram_dev", "dnnf90_ngd_solve_dev",
    "dnnf90_ngd_step_dual_dev", "dnnf90_kf_pass", "dnnf90_kf_pass_iekf", "dnnf90_kf_pass_sys",
    "dnnf90_kf_status", "dnnf90_keep_fits",
]

_lib = None


class Dnnf90Error(RuntimeError):
    def __init__(self, fn, rc):
        msg = ""
        try:
            msg = lib().dnnf90_last_error().decode()
        except Exception:
            pass
        super().__init__(f"{fn} returned {rc}" + (f": {msg}" if msg else ""))
        self.rc = rc


def lib():
    """The loaded device library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m dnnf90_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    i, d, p, P = ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.POINTER
    pi, pd, cs = P(ctypes.c_int), P(ctypes.c_double), ctypes.c_char_p
    sig = {
        "dnnf90_tables_init_dense": [i, i],
        "dnnf90_tables_init_closure": [i, i, i, pi],
        "dnnf90_nderiv": [],
        "dnnf90_alpha": [i, pi],
        "dnnf90_tabset_dense": [i, i],
        "dnnf90_tabset_closure": [i, i, i, pi],
        "dnnf90_tabset_nderiv": [i],
        "dnnf90_net_create_ts": [i, i, pi],
        "dnnf90_net_load": [cs],
        "dnnf90_tabset_activation": [i, i],
        "dnnf90_tabset_free": [i],
        "dnnf90_net_load_ts": [i, cs],
        "dnnf90_net_create": [i, pi],
        "dnnf90_net_set_layer": [i, i, pd],
        "dnnf90_net_free": [i],
        "dnnf90_work_create": [i],
        "dnnf90_work_free": [i],
        "dnnf90_eval": [i, i, pd, pd],
        "dnnf90_twork_create": [i],
        "dnnf90_twork_free": [i],
        "dnnf90_grad_create": [i],
        "dnnf90_grad_free": [i],
        "dnnf90_grad_zero": [i],
        "dnnf90_grad_point": [i, i, pd, pd, i],
        "dnnf90_adam_step": [i, i, d, d, d, d, i, i],
        "dnnf90_net_set_precision": [i, i],
        "dnnf90_nweights": [i],
        "dnnf90_net_get_layer": [i, i, pd],
        "dnnf90_net_save": [i, cs],
        "dnnf90_eval_batch": [i, i, i, pd, pd],
        "dnnf90_eval_batch_multi": [i, i, i, pd, pd],
        "dnnf90_grad_batch": [i, i, i, pd, pd, i],
        "dnnf90_seed_rule_create": [i, i, pd, pi, pi, d],
        "dnnf90_seed_rule_free": [i],
        "dnnf90_grad_rule_batch": [i, i, i, pd, i, i, pd, pd],
        "dnnf90_jrow_batch": [i, i, i, pd, i, pd, pd, pd],
        "dnnf90_grad_read": [i, pd],
        "dnnf90_ngd_step": [i, i, pd, pd, i, d, i, pd],
        "dnnf90_ngd_step_dual": [i, i, pd, pd, i, d, i, pd],
        "dnnf90_set_weights_dev": [i, p, p],
        "dnnf90_forward_dev": [i, i, i, p, p, i, p],
        "dnnf90_backward_dev": [i, i, i, p, p, p, p],
        "dnnf90_grad_rule_dev": [i, i, i, p, i, p, p, p, p],
        "dnnf90_jrow_dev": [i, i, i, p, i, p, p, p],
        "dnnf90_twork_set_chunk": [i, i],
        "dnnf90_keep_fits": [i, i, i, pi],
        "dnnf90_last_error": [],
        "dnnf90_device_available": [],
        "dnnf90_launch_count": [],
        "dnnf90_profile_enable": [i],
        "dnnf90_profile_read": [ctypes.c_char_p, i],
        "dnnf90_ngd_step_noalloc": [i, i, p, p, i, d, p, p],
        "dnnf90_committee_step": [i, pi, pi, pi, pi, p, p, p, p],
        "dnnf90_committee_info": [pi, P(ctypes.c_float)],
        "dnnf90_tune_report": [ctypes.c_char_p, i],
        "dnnf90_tune_force": [i, i],
        "dnnf90_seed_rule_sys": [i, i, pi, pd, pi, pi, pi, pd, d],
        "dnnf90_grad_sys_batch": [i, i, i, pd, pd, i, i, pd, pd],
        "dnnf90_grad_value_batch": [i, i, i, pd, pd, d, i, pd],
        "dnnf90_kf_create": [i, d, d, d, i, d, d],
        "dnnf90_kf_free": [i],
        "dnnf90_kf_update_rows": [i, i, pd, pd, pd],
        "dnnf90_kf_update_rows_dev": [i, i, p, p, p, p, p],
        "dnnf90_kf_read": [i, pd, pi, pd],
        "dnnf90_kf_iekf_begin": [i],
        "dnnf90_kf_iekf_iter": [i, pd, d, d, i],
        "dnnf90_ngd_gram_dev": [i, i, p, i, p, p],
        "dnnf90_ngd_solve_dev": [i, p, p, i, d, p, p],
        "dnnf90_ngd_step_dual_dev": [i, i, p, p, i, d, p, p],
        "dnnf90_kf_pass": [i, i, i, pd, i, d],
        "dnnf90_kf_pass_iekf": [i, i, i, pd, i, d, i],
        "dnnf90_kf_pass_sys": [i, i, i, pd, pd, i, pd, i],
        "dnnf90_kf_status": [i],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = {"dnnf90_last_error": ctypes.c_char_p,
                     "dnnf90_launch_count": ctypes.c_longlong}.get(name, ctypes.c_int)
    _lib = L
    return L


def _pd(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if a is not None else None


def _pi(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int)) if a is not None else None


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def check(name, rc):
    if rc < 0:
        raise Dnnf90Error(name, rc)
    return rc


def call(name, *args):
    return check(name, getattr(lib(), name)(*args))


def device_available() -> bool:
    return bool(lib().dnnf90_device_available())


def launch_count() -> int:
    """Kernels launched by the library so far in this process."""
    return int(lib().dnnf90_launch_count())


def profile_enable(on: bool = True):
    lib().dnnf90_profile_enable(1 if on else 0)


# names of the Bell kernel variants by id (the forward's, the adjoint's)
FWD_VARIANTS = {0: "v5-global", 1: "v5-shared", 2: "v8", 3: "tiled"}
ADJ_VARIANTS = {0: "v5-global", 1: "v5-shared", 2: "v7", 3: "tiled"}


def tune_report() -> list:
    """The Bell kernels' autotuner choices, one per tuned launch shape:
    (kernel, d0, k, |A|, width, precision, chosen variant id, [trial ms per
    variant])."""
    n = lib().dnnf90_tune_report(None, 0)
    buf = ctypes.create_string_buffer(n + 64)
    lib().dnnf90_tune_report(buf, len(buf))
    out = []
    for line in buf.value.decode().splitlines():
        f = line.split()
        out.append((f[0], int(f[1]), int(f[2]), int(f[3]), int(f[4]), f[5], int(f[6]),
                    [float(v) for v in f[7:]]))
    return out


def tune_force(which: int, variant: int) -> None:
    """Pin the Bell forward (which 0) or adjoint (which 1) kernel variant;
    variant -1 hands the choice back to the autotuner.  which 2 switches
    the tanh series forward on where it applies (1) or off (0, -1: the
    default)."""
    call("dnnf90_tune_force", which, variant)


def profile_read() -> dict:
    """{kernel name: (launches, total device ms)} since the last read,
    from CUDA events recorded on each launch's own stream."""
    n = lib().dnnf90_profile_read(None, 0)
    buf = ctypes.create_string_buffer(max(n, 1) + 4096)
    lib().dnnf90_profile_read(buf, len(buf))
    out = {}
    for line in buf.value.decode().splitlines():
        name, cnt, ms = line.split()
        out[name] = (int(cnt), float(ms))
    return out


class TableSet:
    """An independent table set (dnnf90_tabset_dense / _closure)."""

    def __init__(self, d0: int, k: int, seeds=None, activation: int = 0):
        self.d0, self.k = int(d0), int(k)
        if seeds is None:
            self.tid = call("dnnf90_tabset_dense", self.d0, self.k)
        else:
            s = np.ascontiguousarray(np.asarray(seeds, np.int32).reshape(-1))
            self.tid = call("dnnf90_tabset_closure", self.d0, self.k, len(s) // self.d0, _pi(s))
        if activation:
            call("dnnf90_tabset_activation", self.tid, int(activation))
        self.na = call("dnnf90_tabset_nderiv", self.tid)
        # the module-level tables now hold this set (as in the reference)
        self.alpha = np.zeros((self.na, self.d0), np.int32)
        a = np.zeros(self.d0, np.int32)
        for ia in range(self.na):
            call("dnnf90_alpha", ia + 1, _pi(a))
            self.alpha[ia] = a

    def free(self) -> None:
        """Release the handle (networks made on the set keep their copy)."""
        if getattr(self, "tid", 0) > 0:
            call("dnnf90_tabset_free", self.tid)
            self.tid = 0

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def slot(self, a) -> int:
        """1-based slot of multi-index a, 0 if it is not carried."""
        hit = np.nonzero((self.alpha == np.asarray(a, np.int32)).all(axis=1))[0]
        return int(hit[0]) + 1 if len(hit) else 0


class Net:
    """A network on a table set, with its device work spaces."""

    def __init__(self, tables: TableSet, dims, weights=None, precision=PREC_F64):
        self.tables = tables
        self.dims = [int(v) for v in dims]
        d = np.asarray(self.dims, np.int32)
        self.nid = call("dnnf90_net_create_ts", tables.tid, len(d), _pi(d))
        self.nw = call("dnnf90_nweights", self.nid)
        self.na = tables.na
        self.nout = self.dims[-1]
        self.wid = call("dnnf90_work_create", self.nid)
        self.tid = call("dnnf90_twork_create", self.nid)
        self.set_precision(precision)
        if weights is not None:
            self.set_weights(weights)

    def set_precision(self, prec: int):
        call("dnnf90_net_set_precision", self.nid, int(prec))
        self.precision = int(prec)

    def set_weights(self, w):
        w = _f64(w).reshape(-1)
        assert w.size == self.nw, (w.size, self.nw)
        off = 0
        for l in range(2, len(self.dims) + 1):
            n = self.dims[l - 1] * (self.dims[l - 2] + 1)
            call("dnnf90_net_set_layer", self.nid, l, _pd(np.ascontiguousarray(w[off:off + n])))
            off += n

    def get_weights(self):
        out = []
        for l in range(2, len(self.dims) + 1):
            a = np.zeros(self.dims[l - 1] * (self.dims[l - 2] + 1))
            call("dnnf90_net_get_layer", self.nid, l, _pd(a))
            out.append(a)
        return np.concatenate(out)

    def eval(self, X):
        X = _f64(X)
        if X.ndim == 1:
            t = np.zeros(self.na)
            call("dnnf90_eval", self.nid, self.wid, _pd(X), _pd(t))
            return t
        t = np.zeros((X.shape[0], self.na))
        call("dnnf90_eval_batch", self.nid, self.wid, X.shape[0], _pd(X), _pd(t))
        return t

    def eval_multi(self, X):
        X = _f64(X)
        t = np.zeros((X.shape[0], self.nout, self.na))
        call("dnnf90_eval_batch_multi", self.nid, self.wid, X.shape[0], _pd(X), _pd(t))
        return t

    def grad(self):
        return Grad(self)

    def free(self):
        for name, h in (("dnnf90_work_free", "wid"), ("dnnf90_twork_free", "tid")):
            if getattr(self, h, 0) > 0:
                getattr(lib(), name)(getattr(self, h))
                setattr(self, h, 0)
        if getattr(self, "nid", 0) > 0:
            lib().dnnf90_net_free(self.nid)
            self.nid = 0


class Grad:
    """A gradient accumulator (dnnf90_grad_create) of a network."""

    def __init__(self, net: Net):
        self.net = net
        self.gid = call("dnnf90_grad_create", net.nid)

    def zero(self):
        call("dnnf90_grad_zero", self.gid)

    def point(self, x, seed):
        call("dnnf90_grad_point", self.net.nid, self.net.tid, _pd(_f64(x)), _pd(_f64(seed)),
             self.gid)

    def batch(self, X, seeds):
        X, seeds = _f64(X), _f64(seeds)
        call("dnnf90_grad_batch", self.net.nid, self.net.tid, X.shape[0], _pd(X), _pd(seeds),
             self.gid)

    def rule_batch(self, X, rule: "SeedRule", want_t=False):
        X = _f64(X)
        loss = np.zeros(1)
        t = np.zeros((X.shape[0], self.net.na)) if want_t else None
        call("dnnf90_grad_rule_batch", self.net.nid, self.net.tid, X.shape[0], _pd(X),
             rule.rid, self.gid, _pd(loss), _pd(t))
        return (float(loss[0]), t) if want_t else float(loss[0])

    def sys_batch(self, X, rule: "SeedRule", src=None, want_t=False):
        """Forward, system seed (sources src[npts][nres], None = zero) and
        adjoint over a batch, added to this accumulator.  Returns the loss,
        and T[npts][nout][na] if want_t."""
        X = _f64(X)
        loss = np.zeros(1)
        tm = np.zeros((X.shape[0], self.net.nout, self.net.na)) if want_t else None
        sv = _f64(src) if src is not None else None
        call("dnnf90_grad_sys_batch", self.net.nid, self.net.tid, X.shape[0], _pd(X), _pd(sv),
             rule.rid, self.gid, _pd(loss), _pd(tm))
        return (float(loss[0]), tm) if want_t else float(loss[0])

    def value_batch(self, X, y, coef=1.0):
        """Value-only fit L = coef/2 sum (N(x) - y)^2 over a batch, added to
        this accumulator (net_grad_batch).  Returns the loss."""
        X, y = _f64(X), _f64(np.asarray(y, np.float64).reshape(-1))
        loss = np.zeros(1)
        call("dnnf90_grad_value_batch", self.net.nid, self.net.tid, X.shape[0], _pd(X), _pd(y),
             float(coef), self.gid, _pd(loss))
        return float(loss[0])

    def read(self):
        g = np.zeros(self.net.nw)
        call("dnnf90_grad_read", self.gid, _pd(g))
        return g

    def adam(self, eta, beta1, beta2, eps, nbatch, istep):
        call("dnnf90_adam_step", self.net.nid, self.gid, float(eta), float(beta1),
             float(beta2), float(eps), int(nbatch), int(istep))

    def free(self):
        if self.gid > 0:
            lib().dnnf90_grad_free(self.gid)
            self.gid = 0


class SeedRule:
    """A device seed rule (dnnf90_seed_rule_create).

    terms: (coeff, slot, nonlin) triples, slot 1-based.
    """

    def __init__(self, kind: int, terms=(), fac: float = 1.0):
        self.kind = kind
        c = np.array([t[0] for t in terms] or [0.0], np.float64)
        s = np.array([t[1] for t in terms] or [1], np.int32)
        n = np.array([int(t[2]) for t in terms] or [0], np.int32)
        self.rid = call("dnnf90_seed_rule_create", int(kind), len(terms), _pd(c), _pi(s),
                        _pi(n), float(fac))

    @classmethod
    def system(cls, nres, terms, wres=None, fac: float = 1.0) -> "SeedRule":
        """A system rule (dnnf90_seed_rule_sys).  terms: (residual, coeff,
        [(component, slot), ...]) with 1-based residual, component and slot."""
        self = cls.__new__(cls)
        self.kind = SEED_SYS
        res = np.array([t[0] for t in terms], np.int32)
        coeff = np.array([t[1] for t in terms], np.float64)
        nfac = np.array([len(t[2]) for t in terms], np.int32)
        comp = np.array([f[0] for t in terms for f in t[2]], np.int32)
        slot = np.array([f[1] for t in terms for f in t[2]], np.int32)
        wr = _f64(np.asarray(wres, np.float64)) if wres is not None else None
        self.rid = call("dnnf90_seed_rule_sys", int(nres), len(terms), _pi(res), _pd(coeff),
                        _pi(nfac), _pi(comp), _pi(slot), _pd(wr), float(fac))
        return self

    def free(self):
        if self.rid > 0:
            lib().dnnf90_seed_rule_free(self.rid)
            self.rid = 0


def jacobian_rows(net: Net, X, rule: SeedRule):
    X = _f64(X)
    rows = np.zeros((X.shape[0], net.nw))
    resid = np.zeros(X.shape[0])
    t = np.zeros((X.shape[0], net.na))
    call("dnnf90_jrow_batch", net.nid, net.tid, X.shape[0], _pd(X), rule.rid, _pd(rows),
         _pd(resid), _pd(t))
    return rows, resid, t


def ngd_step(net: Net, rows, b, nb: int, mu: float, prec: int = PREC_F64, dual: bool = False):
    """Damped Gauss-Newton step u = (J^T J / nb + mu I)^{-1} (b / nb); dual
    takes the Gram-space route (dnnf90_ngd_step_dual), for nrow < nw."""
    rows, b = _f64(rows), _f64(b)
    u = np.zeros(net.nw)
    call("dnnf90_ngd_step_dual" if dual else "dnnf90_ngd_step", net.nid, rows.shape[0],
         _pd(rows), _pd(b), int(nb), float(mu), int(prec), _pd(u))
    return u


class Kalman:
    """Extended Kalman filter on a network's weights (kalman_t,
    lib/kalman_module.f90): dnnf90_kf_create / dnnf90_kf_update_rows."""

    def __init__(self, net: Net, p0: float, lam_ini: float, lam0: float,
                 decoupled: bool = False, q: float = 0.0, gate: float = 0.0):
        self.net = net
        self.decoupled = bool(decoupled)
        self.kid = 0
        self.kid = check("dnnf90_kf_create",
                         lib().dnnf90_kf_create(net.nid, float(p0), float(lam_ini),
                                                float(lam0), int(decoupled), float(q),
                                                float(gate)))

    def update_rows(self, rows, xi, scale=None):
        """Rank-one updates from rows[k] = dy/dw with innovations xi[k]."""
        rows, xi = _f64(np.atleast_2d(rows)), _f64(np.atleast_1d(xi))
        sc = None if scale is None else _f64(np.broadcast_to(scale, xi.shape))
        call("dnnf90_kf_update_rows", self.kid, rows.shape[0], _pd(rows), _pd(xi),
             None if sc is None else _pd(sc))

    def pass_points(self, X, rule: "SeedRule", rnoise: float = 1.0, niter: int = 0):
        """One filter update per point, each from the point's row and
        residual at the weights the previous update left (dnnf90_kf_pass);
        niter >= 1 takes the iterated update with niter relinearisations
        per point (dnnf90_kf_pass_iekf)."""
        X = _f64(np.atleast_2d(X))
        if niter:
            call("dnnf90_kf_pass_iekf", self.kid, self.net.tid, X.shape[0], _pd(X), rule.rid,
                 float(rnoise), int(niter))
        else:
            call("dnnf90_kf_pass", self.kid, self.net.tid, X.shape[0], _pd(X), rule.rid,
                 float(rnoise))

    def pass_system(self, X, rule: "SeedRule", src=None, rnoise=None, niter: int = 0):
        """One update per point and residual of a system rule, each from the
        residual's row and value at the current weights (dnnf90_kf_pass_sys)."""
        X = _f64(np.atleast_2d(X))
        sv = None if src is None else _f64(src)
        rn = None if rnoise is None else _f64(np.atleast_1d(rnoise))
        call("dnnf90_kf_pass_sys", self.kid, self.net.tid, X.shape[0], _pd(X), _pd(sv),
             rule.rid, _pd(rn), int(niter))

    def iekf_begin(self):
        """The network's current weights become the prior of the iteration."""
        call("dnnf90_kf_iekf_begin", self.kid)

    def iekf_iter(self, row, resid, rnoise, final):
        """One relinearisation from dR/dw and R at the current weights."""
        call("dnnf90_kf_iekf_iter", self.kid, _pd(_f64(row)), float(resid), float(rnoise),
             int(bool(final)))

    def state(self):
        lam = ctypes.c_double()
        ng = ctypes.c_int()
        call("dnnf90_kf_read", self.kid, ctypes.byref(lam), ctypes.byref(ng), None)
        return lam.value, ng.value

    def cov(self):
        """Dense [nw][nw], or the decoupled blocks concatenated (flat)."""
        dims = self.net.dims
        if self.decoupled:
            n = sum(d * (dims[l - 1] + 1) ** 2 for l, d in enumerate(dims) if l > 0)
            P = np.zeros(n)
        else:
            P = np.zeros((self.net.nw, self.net.nw))
        call("dnnf90_kf_read", self.kid, None, None, _pd(P))
        return P

    def free(self):
        if self.kid > 0:
            lib().dnnf90_kf_free(self.kid)
            self.kid = 0

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def committee_step(nets, rules, xs, grads, loss, stream=None):
    """One training step of independent networks in one CUDA graph
    (dnnf90_committee_step).  xs, grads: per-member torch CUDA tensors
    (points [npts][d0] FP64, gradients [nw] FP64, overwritten); loss: a
    torch CUDA FP64 tensor [len(nets)] (overwritten).  Returns (policy,
    graph ms) of the graph that ran."""
    n = len(nets)
    ia = ctypes.c_int * n
    pa = ctypes.c_void_p * n
    nids = ia(*[m.nid for m in nets])
    tids = ia(*[m.tid for m in nets])
    rids = ia(*[r.rid for r in rules])
    npts = ia(*[int(x.shape[0]) for x in xs])
    xp = pa(*[x.data_ptr() for x in xs])
    gp = pa(*[g.data_ptr() for g in grads])
    if stream is None:
        import torch
        stream = torch.cuda.current_stream().cuda_stream
    call("dnnf90_committee_step", n, nids, tids, rids, npts, ctypes.cast(xp, ctypes.c_void_p),
         ctypes.cast(gp, ctypes.c_void_p), loss.data_ptr(), stream)
    pol = ctypes.c_int(-1)
    ms = ctypes.c_float(0.0)
    lib().dnnf90_committee_info(ctypes.byref(pol), ctypes.byref(ms))
    return pol.value, ms.value
