import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_golden(name):
    path = os.path.join(GOLDEN, f"{name}.npz")
    if not os.path.exists(path):
        pytest.skip(f"golden file {name}.npz not generated")
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


GOLDEN_CASES = {
    "d2": dict(geometry=(24, 16), nc=2, kappa=-0.15, beta=3.0),
    "d4": dict(geometry=(2, 4, 4, 6), nc=3, kappa=0.13, beta=5.6),
    "d4su2": dict(geometry=(4, 4, 2, 4), nc=2, kappa=0.12, beta=2.3),
    "d2su3": dict(geometry=(6, 8), nc=3, kappa=0.11, beta=5.0),
}

# adjoint-representation cases (tests/golden/make_golden.py ADJOINT_CASES)
ADJOINT_CASES = {
    "adj_d2su2": dict(geometry=(8, 6), nc=2, kappa=0.17),
    "adj_d4su3": dict(geometry=(2, 4, 2, 4), nc=3, kappa=0.12),
    "adj_d4su2": dict(geometry=(4, 2, 2, 4), nc=2, kappa=0.13),
}

# gauge-observable / smearing cases (tests/golden/make_golden.py OBSERVABLE_CASES)
OBSERVABLE_CASES = {
    "obs_su3": dict(geometry=(4, 4, 4, 6), nc=3),
    "obs_su2": dict(geometry=(4, 6, 4, 4), nc=2),
}

# fermion-measurement cases (tests/golden/make_golden.py MEASUREMENT_CASES)
MEASUREMENT_CASES = {
    "meas_d2": dict(geometry=(8, 6), nc=2, kappa=0.12, representation="fundamental"),
    "meas_d4": dict(geometry=(2, 4, 2, 6), nc=3, kappa=0.11, representation="fundamental"),
    "meas_adj": dict(geometry=(4, 6), nc=2, kappa=0.1, representation="adjoint"),
}


def relerr(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    den = max(np.linalg.norm(b.ravel()), 1e-300)
    return float(np.linalg.norm((a - b).ravel()) / den)


@pytest.fixture(scope="session")
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu-marked test run without a CUDA device")
    return torch.device("cuda:0")
