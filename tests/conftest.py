import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA engine through the C ABI")


def idx(n, x, y, z, Nx, Ny, Nz):
    """ArrayNIJK address (tests/test_webgpu.mjs idx helper)."""
    return n * Nx * Ny * Nz + x * Ny * Nz + y * Nz + z


def free_space(Nx, Ny, Nz):
    """createFreeSpaceCoefficients (tests/test_webgpu.mjs:62-80): vv=ii=1, vi=iv=0.3."""
    t = 3 * Nx * Ny * Nz
    return dict(vv=np.ones(t, np.float32), vi=np.full(t, 0.3, np.float32),
                ii=np.ones(t, np.float32), iv=np.full(t, 0.3, np.float32))


@pytest.fixture(scope="session")
def cuda_engine_cls():
    """The CUDA engine class; skips cleanly on hosts without a GPU."""
    import torch  # plumbing only: device probe
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from efs_b200.build import build
    build()
    from efs_b200.engine import CudaEngine
    return CudaEngine
