import os
import sys

import numpy as np
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


def fg_tolerance(rho, gam, rf, rfg):
    """Tolerance for df/dgamma.  Exchange and correlation gradient terms cancel
    by construction as s -> 0 (mu = beta pi^2/3), so the scale is the size of
    the exchange term |e_x| mu s2_fact / rho^(8/3), capped by what matters for
    the energy density, (|f| + |e_x|) / gamma."""
    xa = 0.75 * (3 / np.pi) ** (1 / 3)
    with np.errstate(divide="ignore", invalid="ignore"):
        ex = xa * rho ** (4 / 3)
        s2g = 1.0 / (4 * (3 * np.pi ** 2) ** (2 / 3)) / rho ** (8 / 3)
        sx = np.where(rho > 0, ex * 0.2195164512208958 * s2g, 0.0)
        se = np.where(gam > 0, (np.abs(rf) + ex) / gam, np.inf)
    return 1e-10 * (np.abs(rfg) + np.minimum(sx, se)) + 1e-300
