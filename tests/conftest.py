import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Restatement
    return Restatement()


@pytest.fixture(scope="session")
def reference():
    from oracle.oracle import Reference, REF_SEQ_SO
    if not REF_SEQ_SO.exists():
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    return Reference()


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    from alp_b200 import _abi
    _abi.call("alpb_init", 0)
    return torch.device("cuda", 0)
