import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "module.clutec.cuda_b200"
for p in (str(PKG), str(ROOT / "oracle"), str(ROOT)):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (sm_100a)")
    config.addinivalue_line("markers", "slow: full-size cases")


@pytest.fixture(scope="session")
def ct():
    import ctstereo
    ctstereo.lib()
    return ctstereo


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    o.lib()
    return o


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def to_dev(a, dev, pitch_align=256):
    """numpy 2-D array -> CUDA tensor view with a 256-byte aligned row pitch."""
    import numpy as np
    import torch
    import ctstereo
    t = torch.from_numpy(np.ascontiguousarray(a))
    out = ctstereo.alloc_image(a.shape[0], a.shape[1], t.dtype, device=dev)
    out.copy_(t.to(dev))
    return out
