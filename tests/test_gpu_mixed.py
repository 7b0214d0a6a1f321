"""INT8 ("mixed") GPU builds, dense and screened (FP64 basis, Ozaki-split
INT8 tcgen05 contractions with exact integer accumulation, FP64 functional
and sums) against the FP64 CPU oracle.

Bar: |dE_xc| < 1e-7 Eh, |dN_el| < 1e-7 and every V_xc element within 1e-7
(the mixed-mode targets are 1e-6 Eh on E_xc and 1e-7 on V_xc).
"""
import numpy as np
import pytest

import oracle as O
from pgxc import cases, lib

pytestmark = pytest.mark.gpu


def run_mixed(case, **kw):
    ref_ham, ref_exc, ref_nel = O.xc_build(case)
    kw.setdefault("screen_threshold", -1.0)
    with lib.Context(case, precision="mixed", **kw) as ctx:
        ham, exc, nel = ctx.build()
    return abs(exc - ref_exc), abs(nel - ref_nel), float(np.max(np.abs(ham - ref_ham)))


@pytest.mark.parametrize("xc", ["VWN", "PBE"])
def test_water_mixed(xc):
    c = cases.config(1)
    c.functional = xc
    O.weight_case(c)
    dE, dN, dV = run_mixed(c)
    print(f"water {xc} mixed: |dE|={dE:.2e} |dN|={dN:.2e} max|dV|={dV:.2e}")
    assert dE < 1e-7 and dN < 1e-7 and dV < 1e-7, (dE, dN, dV)


@pytest.mark.parametrize("xc,seed,lmax", [("PBE", 2, 2), ("VWN", 4, 3), ("PBE", 3, 3)])
def test_small_mixed_multi_chunk(xc, seed, lmax):
    c = cases.small_case(functional=xc, seed=seed, lmax=lmax, natoms=5, nocc=7)
    O.weight_case(c)
    dE, dN, dV = run_mixed(c, max_chunk_points=1024)
    assert dE < 1e-7 and dN < 1e-7 and dV < 1e-7, (dE, dN, dV)


def test_many_orbitals_two_chunks():
    """nocc > 128 takes two orbital chunks in the tensor-core density kernel."""
    c = cases.small_case(functional="PBE", seed=13, natoms=10, nocc=136, lmax=2)
    O.weight_case(c)
    dE, dN, dV = run_mixed(c)
    assert dE < 1e-7 and dN < 1e-7 and dV < 1e-7, (dE, dN, dV)


# ---------------------------------------------------------------------------
# screened layout: per-tile lists, gathered P, scatter-added V
# ---------------------------------------------------------------------------
SCREENED = pytest.mark.parametrize("thr", [0.0, 1e-10], ids=["exact", "1e-10"])


@SCREENED
@pytest.mark.parametrize("xc", ["VWN", "PBE"])
def test_water_mixed_screened(xc, thr):
    c = cases.config(1)
    c.functional = xc
    O.weight_case(c)
    dE, dN, dV = run_mixed(c, screen_threshold=thr)
    print(f"water {xc} mixed screened {thr}: |dE|={dE:.2e} |dN|={dN:.2e} max|dV|={dV:.2e}")
    assert dE < 1e-7 and dN < 1e-7 and dV < 1e-7, (dE, dN, dV)


@SCREENED
@pytest.mark.parametrize("xc,seed,lmax", [("PBE", 2, 2), ("VWN", 4, 3), ("PBE", 3, 3), ("VWN", 1, 2)])
def test_small_mixed_screened_multi_chunk(xc, seed, lmax, thr):
    c = cases.small_case(functional=xc, seed=seed, lmax=lmax, natoms=5, nocc=7)
    O.weight_case(c)
    dE, dN, dV = run_mixed(c, max_chunk_points=1024, screen_threshold=thr)
    assert dE < 1e-7 and dN < 1e-7 and dV < 1e-7, (dE, dN, dV)


def test_ch60_mixed_screened_full_size():
    """The benchmark workload: 60 atoms, 690 functions, 1.16M points, 1e-10 screening."""
    c = cases.config(2)
    O.weight_case(c)
    dE, dN, dV = run_mixed(c, screen_threshold=1e-10)
    print(f"CH60 PBE mixed screened 1e-10: |dE|={dE:.2e} |dN|={dN:.2e} max|dV|={dV:.2e}")
    assert dE < 1e-6 and dN < 1e-7 and dV < 1e-7, (dE, dN, dV)
