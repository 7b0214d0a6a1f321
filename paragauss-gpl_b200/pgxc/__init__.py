"""pgxc: B200-native exchange-correlation grid quadrature for ParaGauss.

The compute path is libpgxc.so (hand-written sm_100a CUDA behind the C ABI of
include/pgxc.h); this package is the host-side mirror used by tests, the
benchmark and Python callers.
"""
from . import abi  # noqa: F401
