import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_outputs.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN)


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.build(with_ref=False)
    return oracle.orc()


@pytest.fixture(scope="session")
def ref():
    import oracle
    if not oracle.ref_available():
        pytest.skip("reference build not available")
    return oracle.ref()


@pytest.fixture(scope="session")
def fem():
    import fe_demo_cpp_b200
    from fe_demo_cpp_b200 import build
    build.build()
    fe_demo_cpp_b200.load()
    return fe_demo_cpp_b200


@pytest.fixture(scope="session")
def cuda(fem):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a GPU test ran without a visible CUDA device")
    return torch.device("cuda:0")
