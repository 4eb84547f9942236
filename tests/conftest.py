import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle_mod():
    """The CPU oracle (checker), built on first use."""
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def lib():
    """The product library, loaded through its C ABI."""
    from linkcell_b200 import _capi
    from linkcell_b200 import build as B
    B.build()
    return _capi.load()


@pytest.fixture(scope="session")
def kats():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "reference_kats.json")) as fh:
        return json.load(fh)


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu(lib):
    """Skip-free GPU guard: a gpu-marked test fails loudly without a device."""
    import torch
    assert torch.cuda.is_available(), "gpu test needs a CUDA device"
    assert lib.lc_gpu_available() == 1, "library does not see the CUDA device"
    return torch.device("cuda", 0)
