"""pytest configuration: the `gpu` marker and shared fixtures.

`-m "not gpu"` runs the CPU suite (oracle pinning, host logic, ABI symbols);
`-m gpu` runs the parity tests that call the CUDA library through its C ABI.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libdcsr_b200.so")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def dcsr():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dcsr_b200 import api
    api.lib()
    return api
