"""The C-ABI library without a GPU: it loads, exports every declared symbol,
builds the same table sets as the oracle (the slot order is interface), keeps
the reference's handle and error-code contract, and refuses compute loudly
when no device is present."""
import ctypes
import os
import re
import tempfile

import numpy as np
import pytest

import pyoracle as po
from dnnf90_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for h in ("dnnf90.h", "dnnf90_b200.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        names += re.findall(r"^(?:int|long long|const char \*)\s*(dnnf90_\w+)\(", src, re.M)
    return names


def test_library_exports_every_declared_symbol():
    L = api.lib()
    names = declared_symbols()
    assert set(api.REFERENCE_SYMBOLS) <= set(names)
    assert len([n for n in names if n in api.REFERENCE_SYMBOLS]) == 24
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(api.REFERENCE_SYMBOLS + api.EXTENSION_SYMBOLS)


@pytest.mark.parametrize("d0,k,seeds", [
    (4, 3, None), (4, 7, None), (2, 3, [[0, 1], [1, 0], [3, 0]]),
    (3, 2, [[1, 0, 0], [0, 2, 0], [0, 0, 2]]), (4, 7, [[7, 0, 0, 0], [0, 0, 0, 1], [2, 2, 1, 0]]),
    (1, 5, None), (6, 2, None)])
def test_tables_match_the_oracle(d0, k, seeds):
    ts = api.TableSet(d0, k, seeds)
    ref = po.Tables(d0, k, seeds)
    assert ts.na == ref.na
    assert np.array_equal(ts.alpha, ref.alpha)
    # module-level tables follow the last set built (tabset_from_current)
    assert api.lib().dnnf90_nderiv() == ref.na


def test_module_tables_and_alpha():
    L = api.lib()
    assert L.dnnf90_tables_init_dense(4, 3) == 0
    assert L.dnnf90_nderiv() == 35
    a = (ctypes.c_int * 4)()
    assert L.dnnf90_alpha(35, a) == 0 and list(a) == [0, 0, 0, 3]
    assert L.dnnf90_alpha(0, a) == -1 and L.dnnf90_alpha(36, a) == -1


def test_argument_checks_of_the_reference():
    # table_args_ok / net_args_ok (lib/c_api_module.f90:72-96)
    L = api.lib()
    assert L.dnnf90_tables_init_dense(0, 3) == -1
    assert L.dnnf90_tables_init_dense(4, 16) == -1
    assert L.dnnf90_tabset_dense(4, 0) == -1
    bad = (ctypes.c_int * 2)(4, 0)
    assert L.dnnf90_tabset_closure(2, 3, 1, bad) == -1  # component > k
    neg = (ctypes.c_int * 2)(-1, 0)
    assert L.dnnf90_tables_init_closure(2, 3, 1, neg) == -1
    t = L.dnnf90_tabset_dense(2, 2)
    assert t > 0
    assert L.dnnf90_tabset_activation(t, 5) == -2
    assert L.dnnf90_tabset_activation(t, 1) == 0
    assert L.dnnf90_tabset_activation(999, 0) == -1
    dims1 = (ctypes.c_int * 1)(2)
    assert L.dnnf90_net_create_ts(t, 1, dims1) == -1      # nlayer < 2
    wrong = (ctypes.c_int * 3)(3, 4, 1)
    assert L.dnnf90_net_create_ts(t, 3, wrong) == -1      # d0 mismatch
    zero = (ctypes.c_int * 3)(2, 0, 1)
    assert L.dnnf90_net_create_ts(t, 3, zero) == -1
    assert L.dnnf90_net_load(b"/nonexistent/nn_weight.dat") == -2
    assert L.dnnf90_work_free(0) == -1 and L.dnnf90_grad_zero(65) == -1


def test_stale_handles_are_refused():
    # tools/example_c_handles.c: a work space built for a freed network is
    # refused after the slot is reused by a wider one
    L = api.lib()
    t = L.dnnf90_tabset_dense(1, 2)
    dA = (ctypes.c_int * 3)(1, 4, 1)
    dB = (ctypes.c_int * 3)(1, 32, 1)
    A = L.dnnf90_net_create_ts(t, 3, dA)
    w = L.dnnf90_work_create(A)
    tw = L.dnnf90_twork_create(A)
    g = L.dnnf90_grad_create(A)
    assert A > 0 and w > 0 and tw > 0 and g > 0
    assert L.dnnf90_net_free(A) == 0
    B = L.dnnf90_net_create_ts(t, 3, dB)
    assert B == A
    x = (ctypes.c_double * 1)(0.3)
    out = (ctypes.c_double * 16)()
    assert L.dnnf90_eval(B, w, x, out) == -1
    seed = (ctypes.c_double * 3)(1, 0, 0)
    assert L.dnnf90_grad_point(B, tw, x, seed, g) == -1
    assert L.dnnf90_adam_step(B, g, 0.1, 0.9, 0.999, 1e-8, 1, 1) == -1
    for h, f in ((w, L.dnnf90_work_free), (tw, L.dnnf90_twork_free), (g, L.dnnf90_grad_free)):
        assert f(h) == 0
    assert L.dnnf90_net_free(B) == 0
    assert L.dnnf90_net_free(B) == -1


def test_weight_file_round_trip(golden):
    # nn_weight.dat of the reference (zwork/hod_4d_k3): load, read back,
    # save, load again
    L = api.lib()
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "nn_weight.dat")
        open(p, "w").write(golden["weight_file"])
        assert L.dnnf90_tables_init_dense(4, 3) == 0
        nid = L.dnnf90_net_load(p.encode())
        assert nid > 0
        tok = golden["weight_file"].split()
        nums = [float(v) for v in tok if re.match(r"^-?\d\.\d+E[-+]\d+$", v)]
        got = []
        for l, (n, m) in zip((2, 3, 4), ((10, 4), (10, 10), (1, 10))):
            a = np.zeros(n * (m + 1))
            assert L.dnnf90_net_get_layer(nid, l, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == 0
            got.append(a)
        got = np.concatenate(got)
        assert got.size == len(nums) and np.array_equal(got, np.array(nums))
        p2 = os.path.join(d, "again.dat")
        assert L.dnnf90_net_save(nid, p2.encode()) == 0
        nid2 = L.dnnf90_net_load(p2.encode())
        assert nid2 > 0
        for l, (n, m) in zip((2, 3, 4), ((10, 4), (10, 10), (1, 10))):
            a = np.zeros(n * (m + 1))
            L.dnnf90_net_get_layer(nid2, l, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
            off = {2: 0, 3: 50, 4: 160}[l]
            assert np.array_equal(a, got[off:off + a.size])
        # a file trained with another activation is refused by a tanh set
        bad = golden["weight_file"].replace("func 0", "func 3", 1)
        p3 = os.path.join(d, "bad.dat")
        open(p3, "w").write(bad)
        assert L.dnnf90_net_load(p3.encode()) == -2
        L.dnnf90_net_free(nid)
        L.dnnf90_net_free(nid2)


def test_no_device_fails_loudly():
    if api.device_available():
        pytest.skip("a GPU is present")
    ts = api.TableSet(2, 2)
    net = api.Net(ts, [2, 4, 1])
    with pytest.raises(api.Dnnf90Error) as e:
        net.eval(np.zeros(2))
    assert e.value.rc == -3
    g = net.grad()
    with pytest.raises(api.Dnnf90Error):
        g.point(np.zeros(2), np.zeros(ts.na))
    g.free()
    # the Kalman filter and the natural-gradient entries need the device too
    with pytest.raises(api.Dnnf90Error) as e:
        api.Kalman(net, 1.0, 0.98, 0.99)
    assert e.value.rc == -3
    with pytest.raises(api.Dnnf90Error) as e:
        api.call("dnnf90_ngd_solve_dev", net.nw, 1, 1, 1, 1e-3, 1, None)
    assert e.value.rc == -3
    # argument checks come first
    fits = ctypes.c_int(7)
    assert api.lib().dnnf90_keep_fits(net.nid, net.tid, -1, ctypes.byref(fits)) == -1
    assert api.lib().dnnf90_keep_fits(net.nid, net.tid, 10, None) == -1
    assert api.lib().dnnf90_keep_fits(net.nid, net.tid, 10, ctypes.byref(fits)) == -3
    assert fits.value == 7
    assert api.lib().dnnf90_kf_create(net.nid, 0.0, 0.98, 0.99, 0, 0.0, 0.0) == -1
    assert api.lib().dnnf90_kf_update_rows(1, 1, None, None, None) == -1
    net.free()


def test_tabset_free_releases_the_handle():
    L = api.lib()
    ids = [L.dnnf90_tabset_dense(2, 2) for _ in range(3)]
    assert all(i > 0 for i in ids)
    assert L.dnnf90_tabset_free(ids[1]) == 0
    assert L.dnnf90_tabset_free(ids[1]) == -1       # already released
    assert L.dnnf90_tabset_nderiv(ids[1]) == -1
    again = L.dnnf90_tabset_dense(2, 2)
    assert 0 < again <= ids[1]                        # handles are reused lowest first
    for i in (ids[0], ids[2], again):
        assert L.dnnf90_tabset_free(i) == 0
    assert L.dnnf90_tabset_free(0) == -1 and L.dnnf90_tabset_free(65) == -1


def test_headers_parse_as_plain_c(tmp_path):
    """include/*.h is the boundary a C host compiles against: both headers
    parse as pedantic C99 (no C++ in the signatures) and as C++."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if not gcc:
        pytest.skip("no C compiler")
    src = tmp_path / "h.c"
    src.write_text('#include "dnnf90.h"\n#include "dnnf90_b200.h"\nint main(void){return 0;}\n')
    inc = os.path.join(ROOT, "include")
    subprocess.run([gcc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-fsyntax-only",
                    "-I", inc, str(src)], check=True)
    gxx = shutil.which("g++")
    if gxx:
        subprocess.run([gxx, "-std=c++17", "-Wall", "-Werror", "-fsyntax-only", "-I", inc,
                        "-x", "c++", str(src)], check=True)
