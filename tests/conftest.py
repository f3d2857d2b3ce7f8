import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
import oracle  # noqa: E402  (test infrastructure: the checker)

REFERENCE = oracle.reference_root()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA path through the C ABI")


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.fixture(scope="session")
def golden_small():
    return dict(np.load(os.path.join(GOLDEN, "ref_T4L4.npz")))


KAT_CONF = os.path.join(GOLDEN, "L4T8conf")  # the reference's test/data/L4T8conf, copied by make_golden.py
KAT_PLAQUETTE = 0.6350055722288719          # test/nissa/src/plaquette_computation.cpp:7-8


@pytest.fixture(scope="session")
def golden_geom():
    return dict(np.load(os.path.join(GOLDEN, "ref_geom.npz")))


@pytest.fixture(scope="session")
def golden_cg():
    return dict(np.load(os.path.join(GOLDEN, "ref_T16L8_cg.npz")))


@pytest.fixture(scope="session")
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu-marked tests")
    return 0
