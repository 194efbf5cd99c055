import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running physics validation")
    # The product library is built in-tree (nvcc cross-compiles without a GPU);
    # build it if a fresh checkout runs the tests before __graft_entry__.build().
    lib = os.path.join(ROOT, "cudapic_b200", "libcudapic.so")
    if not os.path.exists(lib):
        import subprocess
        subprocess.run([sys.executable, os.path.join(ROOT, "cudapic_b200", "build.py")], check=True)


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def cudapic():
    """The product package; its library must exist (built by __graft_entry__.build)."""
    import cudapic_b200
    return cudapic_b200


@pytest.fixture(scope="session")
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    major, _ = torch.cuda.get_device_capability(0)
    if major < 10:
        pytest.fail("libcudapic is built for sm_100a; device capability %d.x" % major)
    return torch.device("cuda", 0)


@pytest.fixture(scope="session")
def tables(oracle):
    """Oracle cross-section tables at the reference gas density."""
    ph = oracle.phys_from_params()
    return oracle.cross_sections(ph.gas_density)
