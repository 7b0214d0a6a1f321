"""Grids built on the device (grid_main_calc + mkgrid's Becke step):
pgxc_atomic_grid against the host restatement (pgxc/grid.py, Lebedev-McLaren
rules of pgxc/lebedev.py), and contexts created on a grid spec against
contexts created on the same grid passed from the host."""
import ctypes as ct

import numpy as np
import pytest

from pgxc import abi, cases, lib
import oracle as O

pytestmark = pytest.mark.gpu


def device_grid(case):
    import torch
    L = lib.lib()
    m = abi.Marshalled(case, weighted=False)
    sp = abi.MarshalledSpec(case)
    n = ct.c_int64()
    assert L.pgxc_atomic_grid_size(ct.byref(m.geometry), ct.byref(sp.spec), ct.byref(n)) == 0
    g = torch.zeros(4 * n.value, dtype=torch.float64, device="cuda")
    own = torch.zeros(n.value, dtype=torch.int32, device="cuda")
    st = L.pgxc_atomic_grid(ct.byref(m.geometry), ct.byref(sp.spec), n.value, g.data_ptr(), own.data_ptr(), None)
    assert st == 0, L.pgxc_last_error(None)
    return g.cpu().numpy().reshape(4, -1), own.cpu().numpy()


@pytest.mark.parametrize("cfg", [1, "mixed"])
def test_device_grid_equals_host_grid_bit_for_bit(cfg):
    if cfg == 1:
        c = cases.config(1)
    else:
        c = cases.small_case(functional="PBE", seed=31, natoms=5, nrad=30, nang=302)
    g, own = device_grid(c)
    assert g.shape[1] == c.npts
    assert np.array_equal(g[0], c.grid_xyz[:, 0]) and np.array_equal(g[1], c.grid_xyz[:, 1])
    assert np.array_equal(g[2], c.grid_xyz[:, 2])
    assert np.array_equal(g[3], c.grid_wraw)
    assert np.array_equal(own, c.point_atom)


def test_bad_rule_is_rejected():
    c = cases.small_case(functional="VWN", seed=3)
    c.meta["nang"] = 100
    L = lib.lib()
    m = abi.Marshalled(c, weighted=False)
    sp = abi.MarshalledSpec(c)
    n = ct.c_int64()
    assert L.pgxc_atomic_grid_size(ct.byref(m.geometry), ct.byref(sp.spec), ct.byref(n)) == abi.PGXC_EINVAL


@pytest.mark.parametrize("precision,thr", [("fp64", 0.0), ("fp64", -1.0), ("mixed", 1e-10)])
def test_context_on_grid_equals_host_grid(precision, thr):
    c = cases.small_case(functional="PBE", seed=32, natoms=4, nrad=24, nang=194)
    with lib.Context(c, precision=precision, weighted=False, screen_threshold=thr) as ref:
        h0, e0, n0 = ref.build()
        w0 = ref.grid_weights()
    with lib.Context(c, precision=precision, screen_threshold=thr, on_grid=True) as ctx:
        h1, e1, n1 = ctx.build()
        w1 = ctx.grid_weights()
    assert np.array_equal(w0, w1)
    assert e0 == e1 and n0 == n1
    np.testing.assert_allclose(h1, h0, rtol=0, atol=1e-13)


def test_context_on_grid_matches_oracle():
    c = cases.config(1)
    O.weight_case(c)
    ref_ham, ref_exc, ref_nel = O.xc_build(c)
    with lib.Context(c, on_grid=True) as ctx:
        ham, exc, nel = ctx.build()
    assert abs(exc - ref_exc) < 1e-10 and abs(nel - ref_nel) < 1e-10
    assert np.max(np.abs(ham - ref_ham)) < 1e-10


def test_context_on_grid_has_the_nuclear_gradient():
    c = cases.small_case(functional="PBE", seed=33, natoms=3, nrad=16, nang=110)
    with lib.Context(c, weighted=False) as ref:
        g0, e0 = ref.xc_gradient()
    with lib.Context(c, on_grid=True) as ctx:
        g1, e1 = ctx.xc_gradient()
    assert abs(e1 - e0) < 1e-12
    np.testing.assert_allclose(g1, g0, rtol=0, atol=1e-12 * max(1.0, np.max(np.abs(g0))))
