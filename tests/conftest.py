import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA path)")


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        return json.load(f)


def per_order_error(T, Tref, deg):
    """Normwise error per derivative order p (the reference's convention,
    app/hod_check_module.f90:216,302): max |T - Tref| / max |Tref| over
    every point and every slot of order p."""
    T, Tref = np.asarray(T), np.asarray(Tref)
    out = {}
    for p in sorted(set(int(d) for d in deg)):
        m = np.asarray(deg) == p
        den = np.max(np.abs(Tref[..., m]))
        out[p] = float(np.max(np.abs(T[..., m] - Tref[..., m])) / (den if den > 0 else 1.0))
    return out


def rel_err(a, b):
    a, b = np.asarray(a), np.asarray(b)
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (den if den > 0 else 1.0))


def xavier_weights(dims, seed):
    """Xavier-normal weights, std = sqrt(2/(fan_in+fan_out)), zero biases
    (init_glorot, app/init_weight_module.f90:245-265), flat layer layout."""
    rng = np.random.default_rng(seed)
    out = []
    for l in range(1, len(dims)):
        fi, fo = dims[l - 1], dims[l]
        W = np.zeros((fo, fi + 1))
        W[:, 1:] = rng.normal(0.0, np.sqrt(2.0 / (fi + fo)), (fo, fi))
        out.append(W.reshape(-1))
    return np.concatenate(out)
