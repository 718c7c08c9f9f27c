import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


@pytest.fixture(scope="session")
def qsgw():
    """The C-ABI library, initialised on cuda:0 (GPU tests only)."""
    import torch
    from ecalj_b200 import lib
    if not torch.cuda.is_available():
        pytest.fail("GPU test collected on a machine without CUDA")
    lib.load()
    lib.init(0)
    lib.share_torch_stream()
    yield lib
    lib.set_precision(lib.PREC_FP64)


def rel_fro(a, b):
    import numpy as np
    a = np.asarray(a); b = np.asarray(b)
    den = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (den if den > 0 else 1.0)
