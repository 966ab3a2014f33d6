import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tic-tac_b200", "python"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")
CASES = ["mt_swave_n16", "lo_j1_J3_n8", "mt_j2_J1_n8"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_case(name):
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    opts = dict(o.split("=", 1) for o in g["opts"])
    meta = dict(
        opts=opts,
        Nphi=int(opts.get("Nphi", 48)),
        Nx=int(opts.get("Nx", 48)),
        tensor_force=opts.get("tensor_force", "true") == "true",
        iso=opts.get("isospin_breaking_1S0", "true") == "true",
        Np=len(g["p_WP"]) - 1,
        Nq=len(g["q_WP"]) - 1,
    )
    return g, meta


def rel(a, b):
    """Normwise relative difference max|a - b| / max|b|."""
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(1e-300, float(np.max(np.abs(b)))))


# U elements below this fraction of the largest |U| of their channel are zero by
# symmetry up to rounding (e.g. 1e-18 between uncoupled deuteron components of a
# central potential); their relative error is taken against the fraction.
ZERO_FLOOR = 1e-6


def rel_elem(a, b):
    """Per-element relative difference max_i |a_i - b_i| / |b_i|: the metric's
    "relative error in every on-shell U element".  Elements with |b_i| below
    ZERO_FLOOR * max|b| are measured against ZERO_FLOOR * max|b|."""
    a = np.asarray(a).reshape(-1)
    b = np.asarray(b).reshape(-1)
    if b.size == 0:
        return 0.0
    den = np.maximum(np.abs(b), ZERO_FLOOR * float(np.max(np.abs(b))))
    den = np.where(den > 0, den, 1e-300)
    return float(np.max(np.abs(a - b) / den))


@pytest.fixture(scope="session")
def has_gpu():
    import tictac_b200 as tt
    return tt.device_count() > 0
