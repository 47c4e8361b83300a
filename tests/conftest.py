"""Shared fixtures.  GPU tests are marked `gpu`; everything else runs on CPU."""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")
if GOLDEN not in sys.path:
    sys.path.insert(0, GOLDEN)  # fixture builders shared with the tests


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (sm_100a)")


@pytest.fixture(scope="session")
def O():
    """The CPU oracle (test infrastructure); builds its C part on first use."""
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        subprocess.run(["make", "-f", os.path.join(ROOT, "oracle", "Makefile")], check=True,
                       capture_output=True)
    from oracle import oracle
    return oracle


@pytest.fixture(scope="session")
def REF(O):
    ref = O.ref_lib()
    if ref is None:
        pytest.skip("reference shim library not built")
    return ref


@pytest.fixture(scope="session")
def gold_ref():
    return dict(np.load(os.path.join(GOLDEN, "reference_small.npz")))


@pytest.fixture(scope="session")
def gold_orc():
    return dict(np.load(os.path.join(GOLDEN, "oracle_small.npz")))


@pytest.fixture(scope="session")
def L():
    """The CUDA library (GPU tests only)."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lamino_b200
    lamino_b200.lib()
    return lamino_b200


def rel(a, b):
    a = np.asarray(a, dtype=np.complex128 if np.iscomplexobj(a) or np.iscomplexobj(b) else np.float64)
    b = np.asarray(b, dtype=a.dtype)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
