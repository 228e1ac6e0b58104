import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "cs5013-project_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

# the reference checkout (read only by the golden-file tests); absent on a GPU box
REFERENCE = os.environ.get("VANN_REFERENCE_DIR", "/root/reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the libvann.so kernels)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def vann_mod():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import vann

    vann.lib()  # fails loudly if libvann.so is missing
    return vann


def have_reference() -> bool:
    return os.path.isdir(os.path.join(REFERENCE, "vamana")) and os.path.exists(
        os.path.join(REFERENCE, "vamana", "vout", "vamana.out"))
