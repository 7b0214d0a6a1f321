import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "paragauss-gpl_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def small_cases():
    from pgxc import cases
    import oracle as O
    out = {}
    for xc in ("VWN", "PBE"):
        c = cases.small_case(functional=xc, seed=11 if xc == "VWN" else 12)
        O.weight_case(c)
        out[xc] = c
    return out
