"""The 500-atom workload on the GPU: CHON500-PBE, 500 C/H/O/N atoms in a
28 A cube, 5,800 functions up to l = 3 (f shells on C, N, O), 9.73 M grid
points, 1,700 occupied orbitals.

The oracle cannot integrate the whole grid in test time (4 N nbas^2 is about
1.3e15 flop), so parity is checked on spatially compact sub-grids with the
full basis and the full density matrix (every function and every orbital
takes part), and the whole grid is checked through properties that do not
depend on its size: the FP64 and INT8 builds agree to the INT8 bar, and
the builds of two halves of the grid sum to the build of the whole.
"""
import numpy as np
import pytest

import oracle as O
from pgxc import cases, dist as D, lib

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def chon500():
    return cases.config(5)


def _build(case, **kw):
    with lib.Context(case, weighted=False, **kw) as ctx:
        return ctx.build()


@pytest.mark.parametrize("part", [1024, 300])
def test_chon500_subgrid_parity(chon500, part):
    """About 4,700 points of one Morton block; Becke weights on the device for
    the GPU builds, on the host for the oracle."""
    sub = D.shard_case(chon500, D.spatial_shards(chon500.grid_xyz, 2048)[part])
    O.weight_case(sub)
    ref_ham, ref_exc, ref_nel = O.xc_build(sub)
    for precision, thr, tol in (("fp64", 0.0, 1e-10), ("fp64", 1e-10, 1e-8), ("mixed", 1e-10, 1e-7)):
        ham, exc, nel = _build(sub, precision=precision, screen_threshold=thr)
        dE, dN, dV = abs(exc - ref_exc), abs(nel - ref_nel), float(np.max(np.abs(ham - ref_ham)))
        print(f"CHON500 part {part} {precision} {thr}: |dE|={dE:.2e} |dN|={dN:.2e} max|dV|={dV:.2e}")
        assert dE < tol and dN < tol and dV < tol, (precision, thr, dE, dN, dV)


def test_chon500_full_grid_int8_matches_fp64(chon500):
    h64, e64, n64 = _build(chon500, precision="fp64", screen_threshold=1e-10)
    h8, e8, n8 = _build(chon500, precision="mixed", screen_threshold=1e-10)
    dE, dN, dV = abs(e8 - e64), abs(n8 - n64), float(np.max(np.abs(h8 - h64)))
    print(f"CHON500 full grid: E_xc={e64:.10f} N_el={n64:.10f}; INT8 vs FP64 |dE|={dE:.2e} |dN|={dN:.2e} "
          f"max|dV|={dV:.2e}")
    assert np.isfinite(e64) and np.isfinite(n64)
    assert dE < 1e-6 and dN < 1e-7 and dV < 1e-7, (dE, dN, dV)


def test_chon500_halves_sum_to_whole(chon500):
    """FP64 with the exact cutoff: the sums do not depend on how the points
    are cut into tiles (INT8 scales and threshold screening are per tile)."""
    whole = _build(chon500, precision="fp64", screen_threshold=0.0)
    parts = [D.shard_case(chon500, idx) for idx in D.spatial_shards(chon500.grid_xyz, 2)]
    halves = [_build(p, precision="fp64", screen_threshold=0.0) for p in parts]
    h = halves[0][0] + halves[1][0]
    e = halves[0][1] + halves[1][1]
    n = halves[0][2] + halves[1][2]
    # the same points and functions; only the order of the additions differs
    assert abs(e - whole[1]) < 1e-12 * abs(whole[1]) and abs(n - whole[2]) < 1e-12 * abs(whole[2])
    assert float(np.max(np.abs(h - whole[0]))) < 1e-10
