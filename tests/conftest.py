import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (run on a B200)")


@pytest.fixture(scope="session")
def port():
    """The oracle's C restatement (built on demand; test infrastructure)."""
    from oracle.oracle import Port
    return Port()


@pytest.fixture(scope="session")
def reference():
    """The reference itself, compiled from its sources (absent on GPU machines)."""
    from oracle.oracle import Reference
    if not Reference.available():
        pytest.skip("oracle/_ref/libbbk_ref.so not built (reference sources absent)")
    return Reference()


@pytest.fixture(scope="session")
def bbk():
    import blockedbunchkaufmanldlt_b200 as bbk
    if not os.path.exists(bbk.LIB_PATH):
        bbk.build()
    bbk.lib()
    return bbk


@pytest.fixture(scope="session")
def cuda(bbk):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    return torch.device("cuda:0")
