"""pgxc_becke_weights_noalloc: the allocation-free Becke entry point.

It exists for callers that cannot let the library allocate device memory
(their device arrays come from their own pool or data regions); the test
therefore allocates every buffer itself and hands the entry point device
pointers only.  Its result must match pgxc_becke_weights, the allocating
entry point, on two calls in a row with different geometries, so that the
scratch array shared by all calls (and left holding the previous call's
distances) cannot leak into the next result.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test.
"""
import ctypes as ct

import numpy as np
import pytest

from pgxc import abi, cases, lib

pytestmark = pytest.mark.gpu

TOL = 2e-16  # the tolerance of the Becke parity test against the oracle


def _device_call(case):
    import torch
    L = lib.lib()
    L.pgxc_becke_weights_noalloc.argtypes = [ct.c_int32, ct.c_void_p, ct.c_int64, ct.c_void_p, ct.c_void_p,
                                             ct.c_void_p, ct.c_void_p]
    coords = torch.from_numpy(np.ascontiguousarray(case.coords).reshape(-1)).cuda()
    pts = torch.from_numpy(np.ascontiguousarray(case.grid_xyz.T).reshape(-1)).cuda()
    owner = torch.from_numpy(np.ascontiguousarray(case.point_atom, dtype=np.int32)).cuda()
    w = torch.full((case.npts,), np.nan, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    st = L.pgxc_becke_weights_noalloc(len(case.coords), coords.data_ptr(), case.npts, pts.data_ptr(),
                                      owner.data_ptr(), w.data_ptr(), ct.c_void_p(stream.cuda_stream))
    assert st == 0, L.pgxc_last_error(None)
    stream.synchronize()
    return w.cpu().numpy()


def test_noalloc_matches_allocating_entry_on_two_calls():
    big = cases.small_case(functional="VWN", seed=41, natoms=6)
    small = cases.small_case(functional="PBE", seed=42, natoms=4)
    for case in (big, small):
        ref = lib.becke_weights(case)
        got = _device_call(case)
        assert np.all(np.isfinite(got))
        np.testing.assert_allclose(got, ref, rtol=0, atol=TOL)


def test_noalloc_rejects_geometry_beyond_scratch_limit():
    L = lib.lib()
    L.pgxc_becke_weights_noalloc.argtypes = [ct.c_int32, ct.c_void_p, ct.c_int64, ct.c_void_p, ct.c_void_p,
                                             ct.c_void_p, ct.c_void_p]
    dummy = ct.c_void_p(16)  # never dereferenced: the size check comes first
    st = L.pgxc_becke_weights_noalloc(513, dummy, 10, dummy, dummy, dummy, None)
    assert st == abi.PGXC_EINVAL
    assert b"513" in L.pgxc_last_error(None)
