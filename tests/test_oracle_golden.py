"""Pins the CPU oracle to the reference's own vectors before it is trusted
as the checker of the CUDA path."""
import math

import numpy as np
import pytest

import pyoracle as po
from conftest import per_order_error, rel_err


def test_shipped_golden_regressions(golden):
    # zwork/hod_4d_{k3,k7,k7_active}/hod_golden.dat; the reference's own
    # [REF] check passes at 1e-10 and reports 2.2e-19 / 2.8e-17
    for case in golden["hod_cases"]:
        tab = po.Tables(4, case["k"], case["seeds"])
        w = po.check_weights(case["dims"])
        t, _ = po.eval_point(tab, case["dims"], w, case["x"])
        assert len(case["t"]) == tab.na
        err = np.max(np.abs(t - np.array(case["t"])))
        assert err < 1e-15, (case["case"], err)


def test_jet_goldens(golden):
    # tools/make_hod_golden.py (independent Taylor jet) on further shapes
    for case in golden["jet_cases"]:
        d0 = case["dims"][0]
        tab = po.Tables(d0, case["k"], case["seeds"])
        w = po.check_weights(case["dims"])
        t, _ = po.eval_point(tab, case["dims"], w, case["x"])
        errs = per_order_error(t, case["t"], tab.deg)
        assert max(errs.values()) < 1e-13, (case["dims"], errs)


def test_alpha_order(golden):
    a = golden["alpha_order"]
    tab = po.Tables(a["d0"], a["k"])
    assert tab.alpha.tolist() == a["alpha"]


def test_table_counts_from_logs(golden):
    for c in golden["counts"]:
        tab = po.Tables(c["d0"], c["k"], c["seeds"])
        assert (tab.na, tab.nbell) == (c["na"], c["nbell"]), c["log"]
    # fq / pair sizes of the ZK7 set
    tab = po.Tables(4, 7)
    assert (tab.na, tab.nfq, tab.npair) == (330, 18172, 6105)


def _dirkat_net(dk):
    d0, W = dk["d0"], dk["width"]
    w_ref = dk["w_ref"]
    w, p = [], 0
    for fan, n in [(d0, W), (W, W), (W, 1)]:
        for _ in range(n):
            w.append(w_ref[p + fan])          # bias is stored last per neuron
            w.extend(w_ref[p:p + fan])
            p += fan + 1
    return [d0, W, W, 1], np.array(w), np.array(dk["x"]).reshape(dk["npt"], d0)


def test_directional_known_answers(golden):
    # bench/cpp/README.md:97-105: loss = sum_n (d^K N / dx_1^K)^2 and dL/dw_1
    dk = golden["dirkat"]
    dims, w, X = _dirkat_net(dk)
    for ks, (lref, gref) in dk["table"].items():
        K = int(ks)
        tab = po.Tables(4, K, [[K, 0, 0, 0]])
        s = tab.slot((K, 0, 0, 0))
        g, T, _, _ = po.grad_batch(tab, dims, w, X, kind=po.SEED_PINN,
                                   terms=[(1.0, s, 0)], fac=2.0)
        loss = float(np.sum(T[:, s - 1] ** 2))
        assert abs(loss / lref - 1) < 1e-11, (K, loss, lref)
        # flat index 1: first hidden neuron, weight of x_1
        assert abs(g[1] / gref - 1) < 5e-9, (K, g[1], gref)


def test_oracle_adjoint_against_finite_differences():
    # Hod_check style: adjoint vs central differences of the full loss
    # (app/hod_check_module.f90:225-411, hw = 1e-5)
    dims = [3, 5, 4, 1]
    tab = po.Tables(3, 3)
    rng = np.random.default_rng(7)
    w = rng.normal(0, 0.5, po.weight_count(dims))
    X = rng.uniform(-1, 1, (6, 3))
    g, _, loss, _ = po.grad_batch(tab, dims, w, X, kind=po.SEED_HALFSQ)
    hw = 1e-5
    for i in range(0, len(w), 3):
        wp, wm = w.copy(), w.copy()
        wp[i] += hw
        wm[i] -= hw
        lp = po.grad_batch(tab, dims, wp, X)[2]
        lm = po.grad_batch(tab, dims, wm, X)[2]
        fd = (lp - lm) / (2 * hw)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_ngd_step_solves_the_damped_system():
    rng = np.random.default_rng(3)
    J = rng.normal(size=(40, 12))
    b = rng.normal(size=12)
    u = po.ngd_step(J, b, 40, 1e-3)
    G = J.T @ J / 40 + 1e-3 * np.eye(12)
    assert rel_err(G @ u, b / 40) < 1e-12


def test_adam_matches_the_formula():
    w = np.array([0.5, -0.2]); m = np.zeros(2); v = np.zeros(2)
    g = np.array([0.1, 0.3])
    po.adam_step(w, g, m, v, 0.01, 0.9, 0.999, 1e-8, 2, 1)
    gv = g / 2
    exp = np.array([0.5, -0.2]) - 0.01 * gv / (np.abs(gv) + 1e-8)
    assert np.max(np.abs(w - exp)) < 1e-12


def test_oracle_sin_and_erf_derivatives():
    """sigma^(q) of the sin and erf activations against their closed forms
    (act_derivs_ts, lib/multi_index_bell_module.f90:723-850)."""
    import math
    ts = po.Tables(2, 5, activation=1)
    for a in (-1.3, 0.0, 0.7, 2.9):
        d = ts.act_derivs(a, 6)
        ref = [math.sin(a), math.cos(a), -math.sin(a), -math.cos(a)] * 2
        assert np.allclose(d, ref[:7], rtol=0, atol=1e-15)
    te = po.Tables(2, 5, activation=2)
    for a in (-2.5, -0.4, 0.0, 1.1, 3.0):
        d = te.act_derivs(a, 5)
        g = 2.0 / math.sqrt(math.pi) * math.exp(-a * a)
        # erf' = g, erf'' = -2a g, erf''' = (4a^2 - 2) g, erf'''' = (12a - 8a^3) g,
        # erf''''' = (16a^4 - 48a^2 + 12) g
        ref = [math.erf(a), g, -2 * a * g, (4 * a * a - 2) * g, (12 * a - 8 * a ** 3) * g,
               (16 * a ** 4 - 48 * a * a + 12) * g]
        assert np.allclose(d, ref, rtol=1e-13, atol=1e-15), (a, d, ref)


def test_bessel_values_and_derivatives_against_scipy():
    """The oracle's J_n (Miller's backward recurrence) and the J0 / J1
    derivative combinations of besj0_derivs / besj1_derivs
    (lib/multi_index_bell_module.f90:757-826) against scipy."""
    import scipy.special as sp
    xs = np.concatenate([np.linspace(-40, 40, 801), [0.0, 1e-300, 1e-30, 1e-10, -1e-6, 1e-3]])
    for x in xs:
        assert np.max(np.abs(po.besj_all(12, x) - sp.jv(np.arange(13), x))) < 2e-15, x
    for act, order in ((3, 0), (4, 1)):
        tab = po.Tables(2, 7, activation=act)
        for a in (-7.3, -1.2, 0.0, 0.4, 3.3, 15.0):
            d = tab.act_derivs(a, 9)
            ref = [sp.jvp(order, a, q) for q in range(10)]
            assert np.max(np.abs(d - ref)) < 1e-14, (act, a)
