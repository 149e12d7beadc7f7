#!/usr/bin/env python3
"""Generate tests/golden/golden.json from the reference tree.

Run with DNNF90_REFERENCE set to the reference source tree; the output
is committed, so the tests never read the reference at run time.

Contents:
  hod_cases   the three shipped golden regressions (zwork/hod_4d_k3,
              hod_4d_k7, hod_4d_k7_active: hod_golden.dat, the network shape
              of input_nn.dat, the closure seeds of alpha_seeds.dat).  The
              weights are the self-check formula of
              app/hod_check_module.f90:100-107.
  jet_cases   further shapes evaluated by the reference's own independent
              Taylor-jet tool, tools/make_hod_golden.py, run unmodified on a
              scratch case directory (weight-file shape, alpha order and x
              are the inputs it reads).
  alpha_order zwork/hod_4d_k3/hod_alpha_order.dat (slot order fixture).
  counts      table sizes printed in the reference's logs ("NUM_alpha" and
              "Bell table terms" of init_hod_tables).
  weight_file zwork/hod_4d_k3/nn_weight.dat, a weight file in the
              reference's nn_weight.dat format (lib/net_module.f90:146-243).
  dirkat      the directional known-answer test: bench/julia/wx_ref.txt
              (4-8-8-1 weights, per neuron [w_1..w_fanin, bias], and 20
              points) with the loss and dL/dw_1 of bench/cpp/README.md:97-105.
"""
from __future__ import annotations

import json
import os
import re
import subprocess
import sys
import tempfile

REF = os.environ.get("DNNF90_REFERENCE")
if not REF:
    sys.exit("set DNNF90_REFERENCE to the reference source tree (its zwork/ goldens and "
             "tools/make_hod_golden.py are read from there)")
HERE = os.path.dirname(os.path.abspath(__file__))


def read_golden(path):
    lines = [l for l in open(path).read().split("\n") if l.strip()]
    x = [float(v) for v in lines[0].split()]
    vals = {}
    for l in lines[1:]:
        ia, v = l.split()
        vals[int(ia)] = float(v)
    return x, [vals[i] for i in sorted(vals)]


def read_dims(input_nn):
    lines = open(input_nn).read().split("\n")
    for i, l in enumerate(lines):
        f = l.split()
        if f and f[0] == "Nlayer":
            n = int(f[1])
            return [int(lines[i + 1 + k].split()[0]) for k in range(n)]
    raise ValueError(input_nn)


def read_seeds(path):
    rows = [l.split() for l in open(path) if l.strip()]
    n = int(rows[0][0])
    return [[int(v) for v in r] for r in rows[1 : 1 + n]]


def alpha_list(d0, k, seeds=None):
    import itertools

    out = []
    for p in range(k + 1):
        for c in itertools.combinations_with_replacement(range(d0), p):
            a = [0] * d0
            for t in c:
                a[t] += 1
            if seeds is None or any(all(a[i] <= s[i] for i in range(d0)) for s in seeds):
                out.append(a)
    return out


def jet_case(dims, k, x, seeds=None):
    """Run tools/make_hod_golden.py --write on a scratch case directory."""
    d0 = dims[0]
    alphas = alpha_list(d0, k, seeds)
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "nn_weight.dat"), "w") as f:
            f.write("0\nfunc 0\nActivation_out 0\n%d\n" % len(dims))
            for v in dims:
                f.write("%d\n" % v)
        with open(os.path.join(d, "hod_alpha_order.dat"), "w") as f:
            f.write("# column order\n# ia |alpha| alpha\n")
            for i, a in enumerate(alphas, 1):
                f.write("%d  %d  %s\n" % (i, sum(a), " ".join(str(v) for v in a)))
        with open(os.path.join(d, "hod_golden.dat"), "w") as f:
            f.write(" ".join("%.17e" % v for v in x) + "\n")
        subprocess.run([sys.executable, os.path.join(REF, "tools", "make_hod_golden.py"),
                        d, "--write"], check=True, capture_output=True)
        _, vals = read_golden(os.path.join(d, "hod_golden.dat"))
    return {"dims": dims, "k": k, "seeds": seeds, "x": x, "t": vals}


def main():
    out = {"hod_cases": [], "jet_cases": [], "counts": [], "dirkat": None}
    for case, seedfile in [("hod_4d_k3", None), ("hod_4d_k7", None),
                           ("hod_4d_k7_active", "alpha_seeds.dat")]:
        cdir = os.path.join(REF, "zwork", case)
        x, vals = read_golden(os.path.join(cdir, "hod_golden.dat"))
        dims = read_dims(os.path.join(cdir, "input_nn.dat"))
        m = re.search(r"Hod_K\s+(\d+)", open(os.path.join(cdir, "input_nn.dat")).read())
        seeds = read_seeds(os.path.join(cdir, seedfile)) if seedfile else None
        out["hod_cases"].append({"case": case, "dims": dims, "k": int(m.group(1)),
                                 "seeds": seeds, "x": x, "t": vals})
    order = []
    for l in open(os.path.join(REF, "zwork", "hod_4d_k3", "hod_alpha_order.dat")):
        f = l.split()
        if f and f[0].isdigit():
            order.append([int(v) for v in f[2:]])
    out["alpha_order"] = {"d0": 4, "k": 3, "alpha": order}
    # table sizes from the logs: (d0, k, seeds) -> NUM_alpha, Bell terms
    for log, d0, k, seeds in [
        ("zwork/hod_4d_k3/a_reference.log", 4, 3, None),
        ("zwork/hod_4d_k7/a_reference.log", 4, 7, None),
        ("bench/scal_dense/a.log", 4, 7, None),
        ("bench/kdv/a.log", 2, 3, [[0, 1], [1, 0], [3, 0]]),
        ("zwork/tutorial_heat2d/a.log", 3, 2, [[0, 0, 0], [1, 0, 0], [0, 2, 0], [0, 0, 2]]),
    ]:
        txt = open(os.path.join(REF, log)).read()
        na = int(re.search(r"NUM_alpha \(multi-indices carried\) = (\d+)", txt).group(1))
        nb = int(re.search(r"Bell table terms\s+= (\d+)", txt).group(1))
        out["counts"].append({"log": log, "d0": d0, "k": k, "seeds": seeds, "na": na, "nbell": nb})
    # jet goldens on further shapes, including the benchmark shapes
    out["jet_cases"].append(jet_case([4, 32, 32, 1], 3, [0.21, -0.34, 0.15, 0.42]))
    out["jet_cases"].append(jet_case([2, 64, 64, 64, 1], 3, [0.7, 0.3],
                                     seeds=[[0, 1], [1, 0], [3, 0]]))
    out["jet_cases"].append(jet_case([3, 64, 64, 1], 2, [0.3, 0.6, 0.2],
                                     seeds=[[0, 0, 0], [1, 0, 0], [0, 2, 0], [0, 0, 2]]))
    out["jet_cases"].append(jet_case([4, 16, 16, 16, 1], 5, [-0.5, 0.25, 0.8, -0.1]))
    # directional known-answer test
    tok = open(os.path.join(REF, "bench", "julia", "wx_ref.txt")).read().split()
    kmax, npt, nw, d0 = (int(v) for v in tok[:4])
    vals = [float(v) for v in tok[4:]]
    readme = open(os.path.join(REF, "bench", "cpp", "README.md")).read()
    table = {}
    for m in re.finditer(r"^\| (\d) \| ([-+0-9.e]+) \| ([-+0-9.e]+) \|$", readme, re.M):
        table[int(m.group(1))] = (float(m.group(2)), float(m.group(3)))
    out["dirkat"] = {"d0": d0, "width": 8, "npt": npt, "w_ref": vals[:nw],
                     "x": vals[nw:], "table": {str(k): v for k, v in sorted(table.items())}}
    # a weight file of the reference's own format (net_load / net_save)
    out["weight_file"] = open(os.path.join(REF, "zwork", "hod_4d_k3", "nn_weight.dat")).read()
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f, indent=0)
    print("wrote", os.path.join(HERE, "golden.json"))


if __name__ == "__main__":
    main()
