import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "fivohydro.jl_b200"))
sys.path.insert(0, str(ROOT / "tests"))
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the libfivo2d.so kernels)")
    config.addinivalue_line("markers", "slow: long CPU run (oracle convergence ladders)")


@pytest.fixture(scope="session")
def gpu_lib():
    """libfivo2d.so, loaded; fails loudly when it is missing or no GPU is visible."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test collected on a machine without a CUDA device")
    from fivo2d import _abi as A
    return A.load_library()
