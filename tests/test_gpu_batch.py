"""Batched builds of a molecule set (pgxc_batch_create / pgxc_batch_run): the
device builds of many screened contexts captured as the parallel branches of
one CUDA graph and replayed with one launch.

Checked: every molecule of a small set against the FP64 oracle (FP64 at 1e-10,
INT8 at 1e-7); the batch against the same contexts built one by one; replays
that follow new operand contents behind the fixed pointers; rejection of a
context in the dense layout.
"""
import numpy as np
import pytest

import oracle as O
from pgxc import cases, lib

pytestmark = pytest.mark.gpu


def _device_operands(torch, mols):
    dC = [torch.from_numpy(m.c_fortran()).cuda() for m in mols]
    docc = [torch.from_numpy(m.occ_fortran()).cuda() for m in mols]
    dham = [torch.zeros(m.xc_length, dtype=torch.float64, device="cuda") for m in mols]
    dsum = [torch.zeros(2, dtype=torch.float64, device="cuda") for m in mols]
    return dC, docc, dham, dsum


def _ptrs(ts):
    return [t.data_ptr() for t in ts]


@pytest.fixture(scope="module")
def small_set():
    mols = cases.molecule_set(6, seed=77, atoms=(3, 6))
    for m in mols:
        O.weight_case(m)
    return mols


@pytest.mark.parametrize("precision,thr,tol", [("fp64", 0.0, 1e-10), ("mixed", 1e-10, 1e-7)])
def test_batch_matches_oracle(small_set, precision, thr, tol):
    torch = pytest.importorskip("torch")
    ctxs = [lib.Context(m, precision=precision, screen_threshold=thr, max_chunk_points=4096) for m in small_set]
    dC, docc, dham, dsum = _device_operands(torch, small_set)
    try:
        with lib.Batch(ctxs, _ptrs(dC), _ptrs(docc), _ptrs(dham), _ptrs(dsum)) as b:
            b.run()
            b.run()  # a replay gives the same build
        for m, h, s in zip(small_set, dham, dsum):
            ref_h, ref_e, ref_n = O.xc_build(m)
            e, n = s.tolist()
            dE, dN, dV = abs(e - ref_e), abs(n - ref_n), float(np.max(np.abs(h.cpu().numpy() - ref_h)))
            assert dE < tol and dN < tol and dV < tol, (m.name, precision, dE, dN, dV)
    finally:
        for c in ctxs:
            c.close()


def test_batch_equals_one_by_one_and_follows_operands():
    torch = pytest.importorskip("torch")
    mols = cases.molecule_set(24, seed=5, atoms=(3, 16))
    ctxs = [lib.Context(m, precision="mixed", weighted=False, screen_threshold=1e-10, max_chunk_points=8192)
            for m in mols]
    dC, docc, dham, dsum = _device_operands(torch, mols)
    try:
        one = []
        for c, a, o, h, s in zip(ctxs, dC, docc, dham, dsum):
            c.build_device(a.data_ptr(), o.data_ptr(), h.data_ptr(), s.data_ptr())
            one.append((h.clone(), s.clone()))
        with lib.Batch(ctxs, _ptrs(dC), _ptrs(docc), _ptrs(dham), _ptrs(dsum)) as b:
            for h in dham:
                h.zero_()
            b.run()
            # INT8 contexts run as one set: per chunk one launch per kernel over all
            # molecules' tiles (these contexts' own 8192-point chunks do not apply)
            assert b.is_set()
            assert b.stats()["kernel_nodes"] < 8 * len(mols)
            for (h1, s1), h, s in zip(one, dham, dsum):
                # the same per-tile arithmetic: V is scatter-added with atomics (its last bits
                # depend on the order of the additions), and the set sums E_xc and N_el per
                # molecule over its tiles in another fixed order than a single build does
                assert torch.allclose(h, h1, rtol=0, atol=1e-10), float((h - h1).abs().max())
                assert torch.allclose(s, s1, rtol=1e-13, atol=0), (s, s1)
            # new contents behind the same pointers: halve the occupations
            for o in docc:
                o.mul_(0.5)
            b.run()
        for c, a, o, (h1, s1), s in zip(ctxs, dC, docc, one, dsum):
            hh = torch.zeros_like(h1)
            ss = torch.zeros_like(s1)
            c.build_device(a.data_ptr(), o.data_ptr(), hh.data_ptr(), ss.data_ptr())
            assert torch.allclose(s, ss, rtol=1e-14, atol=0)
            assert float(s[1]) < 0.6 * float(s1[1])  # about half the charge
    finally:
        for c in ctxs:
            c.close()


def test_batch_rejects_dense_context(small_set):
    torch = pytest.importorskip("torch")
    m = small_set[0]
    ctx = lib.Context(m, screen_threshold=-1.0)
    dC, docc, dham, dsum = _device_operands(torch, [m])
    try:
        with pytest.raises(lib.PgxcError) as e:
            lib.Batch([ctx], _ptrs(dC), _ptrs(docc), _ptrs(dham), _ptrs(dsum))
        assert "screened" in str(e.value)
    finally:
        ctx.close()


def test_set_with_small_chunks_matches_oracle():
    """A set cut into many chunks (256 points each): chunks span molecules and
    change functional; every molecule still matches the oracle."""
    torch = pytest.importorskip("torch")
    mols = cases.molecule_set(6, seed=9, atoms=(3, 6))
    ctxs = [lib.Context(m, precision="mixed", weighted=False, screen_threshold=1e-10) for m in mols]
    dC, docc, dham, dsum = _device_operands(torch, mols)
    try:
        with lib.Batch(ctxs, _ptrs(dC), _ptrs(docc), _ptrs(dham), _ptrs(dsum), max_chunk_points=256) as b:
            assert b.is_set()
            b.run()
        for m, h, s in zip(mols, dham, dsum):
            O.weight_case(m)
            ref_h, ref_e, ref_n = O.xc_build(m)
            e, n = s.tolist()
            assert abs(e - ref_e) < 1e-7 and abs(n - ref_n) < 1e-7, (m.name, e - ref_e, n - ref_n)
            assert float(np.max(np.abs(h.cpu().numpy() - ref_h))) < 1e-7
    finally:
        for c in ctxs:
            c.close()
