import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "hi-slam2_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libhislam2_b200.so")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


@pytest.fixture(scope="session")
def ref_ops():
    """The reference's own droid_backends operators built in oracle/_ref (None if absent)."""
    from oracle import build_ref
    return build_ref.load()


@pytest.fixture(scope="session")
def ref_corr(ref_ops):
    """The reference's correlation operators (the same module as ref_ops)."""
    return ref_ops
