import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def pytest_sessionstart(session):
    """A fresh checkout has no built library (built files stay out of git):
    build the sm_100a library and the CLI once before the tests load them.
    A tree that has them is used as it is."""
    from tinypt_b200 import build as b

    if not b.LIB.exists() or not b.CLI.exists():
        b.build()


def cuda_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle

    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def gpu():
    if not cuda_available():
        pytest.fail("a GPU test ran on a machine without CUDA")
    import torch

    torch.cuda.init()
    return torch.device("cuda:0")
