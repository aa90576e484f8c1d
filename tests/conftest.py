import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

import belief_network_wrapper as W  # noqa: E402  (registers belief_propagation_b200)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def bp():
    return W.bp


@pytest.fixture(scope="session")
def synth():
    return W.bp.synth


@pytest.fixture(scope="session")
def restatement():
    import oracle as O
    return O.Restatement()


@pytest.fixture(scope="session")
def reference():
    import oracle as O
    if not O.reference_available():
        pytest.skip("reference checker (oracle/_ref) not built here")
    return O.Reference()


@pytest.fixture(scope="session")
def O():
    import oracle
    return oracle


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def native():
    from belief_propagation_b200 import native as N
    N.load()
    return N


def load_golden(name):
    path = os.path.join(GOLDEN, name)
    if not os.path.exists(path):
        pytest.skip(f"fixture {name} missing")
    return dict(np.load(path, allow_pickle=False))
