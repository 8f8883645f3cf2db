import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs with -m gpu")


def _build_once():
    # Build the product library and the CPU oracle in-tree if they are missing or stale.
    from fdk_b200 import build as B

    try:
        B.build()
    except Exception as e:  # no nvcc on this machine: the prebuilt library must be present
        if not os.path.exists(B.LIB):
            raise RuntimeError(f"libfdk_b200.so missing and cannot be built: {e}")
    from oracle import oracle as O

    O.lib()


_build_once()


@pytest.fixture(scope="session")
def has_gpu():
    import torch

    return torch.cuda.is_available()


@pytest.fixture(autouse=True)
def _gpu_guard(request):
    if request.node.get_closest_marker("gpu"):
        import torch

        if not torch.cuda.is_available():
            pytest.skip("no CUDA device")
