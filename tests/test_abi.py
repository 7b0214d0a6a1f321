"""C-ABI checks that need no GPU: exported symbols, argument validation,
and the loud failure without a device (there is no CPU fallback)."""
import ctypes as ct
import os
import re

import numpy as np
import pytest

from conftest import ROOT, gpu_available
from pgxc import abi, cases, lib


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "pgxc.h")).read()
    return sorted(set(re.findall(r"\b(pgxc_[a-z_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = lib.lib()
    names = declared_symbols()
    assert len(names) >= 12
    for n in names:
        assert hasattr(L, n), n


def test_header_and_ctypes_struct_layouts_agree():
    # offsets checked against the C layout rules the header implies
    assert ct.sizeof(abi.Geometry) == 16
    assert ct.sizeof(abi.Grid) == 32
    assert ct.sizeof(abi.Options) == 40
    assert ct.sizeof(abi.Timings) == 80


def test_default_options():
    o = abi.Options()
    lib.lib().pgxc_default_options(ct.byref(o))
    assert (o.functional, o.ispin, o.precision, o.batch_points, o.device) == (abi.XC_VWN, 1, abi.PREC_FP64, 128, -1)
    assert o.screen_threshold == 0.0


def _create(case, **kw):
    m = abi.Marshalled(case)
    o = abi.Options()
    lib.lib().pgxc_default_options(ct.byref(o))
    o.functional = abi.XC_IDS[case.functional]
    for k, v in kw.items():
        setattr(o, k, v)
    h = ct.c_void_p()
    st = lib.lib().pgxc_create(ct.byref(m.geometry), ct.byref(m.basis), ct.byref(m.grid), ct.byref(o), ct.byref(h))
    if h.value:
        lib.lib().pgxc_destroy(h)
    return st, lib.lib().pgxc_last_error(None).decode()


@pytest.fixture(scope="module")
def case():
    c = cases.small_case(functional="VWN", seed=3)
    c.grid_w = c.grid_wraw.copy()
    return c


def test_rejects_bad_options(case):
    assert _create(case, functional=max(abi.XC_IDS.values()) + 1)[0] == abi.PGXC_EINVAL
    assert _create(case, functional=0)[0] == abi.PGXC_EINVAL
    assert _create(case, ispin=3)[0] == abi.PGXC_EINVAL
    assert _create(case, precision=7)[0] == abi.PGXC_EINVAL


def test_rejects_unordered_shells(case):
    bad = cases.Case(**{**case.__dict__})
    bad.shell_l = case.shell_l[::-1].copy()
    st, msg = _create(bad)
    assert st == abi.PGXC_EINVAL and "ordered" in msg


def test_rejects_high_l_and_nonfinite(case):
    bad = cases.Case(**{**case.__dict__})
    bad.shell_l = case.shell_l.copy()
    bad.shell_l[-1] = 4
    assert _create(bad)[0] in (abi.PGXC_ENOTSUP, abi.PGXC_EINVAL)
    bad = cases.Case(**{**case.__dict__})
    bad.norms = case.norms.copy()
    bad.norms[0] = np.nan
    assert _create(bad)[0] == abi.PGXC_ENONFINITE
    bad = cases.Case(**{**case.__dict__})
    bad.exponents = case.exponents.copy()
    bad.exponents[0] = -1.0
    assert _create(bad)[0] == abi.PGXC_EINVAL


def test_open_shell_needs_the_screened_layout(case):
    """ispin=2 is built by the screened layout only; the dense layout
    (screen_threshold < 0) reports it unsupported before touching a device."""
    st, msg = _create(case, ispin=2, screen_threshold=-1.0)
    assert st == abi.PGXC_ENOTSUP and "screened" in msg
    assert _create(case, ispin=2)[0] != abi.PGXC_ENOTSUP


@pytest.mark.skipif(gpu_available(), reason="checks the no-device path")
def test_no_device_fails_loudly(case):
    st, msg = _create(case)
    assert st == abi.PGXC_ENODEV, (st, msg)
    f = np.zeros(2)
    st = lib.lib().pgxc_xc_functionals(abi.XC_VWN, 1, 2, abi.f64p(np.ones(2)), abi.f64p(None), abi.f64p(f),
                                       abi.f64p(np.zeros(2)), abi.f64p(None))
    assert st == abi.PGXC_ENODEV


def test_strerror():
    for s in range(0, -8, -1):
        assert lib.lib().pgxc_strerror(s)


def test_grid_spec_size_matches_the_host_grid():
    """pgxc_atomic_grid_size needs no device: shells with r < 40 bohr times the rule."""
    import ctypes as ct
    for c in (cases.config(1), cases.small_case(functional="PBE", seed=31, natoms=5, nrad=30, nang=302)):
        m = abi.Marshalled(c, weighted=False)
        sp = abi.MarshalledSpec(c)
        n = ct.c_int64()
        assert lib.lib().pgxc_atomic_grid_size(ct.byref(m.geometry), ct.byref(sp.spec), ct.byref(n)) == 0
        assert n.value == c.npts
    sp.spec.nang = 100
    assert lib.lib().pgxc_atomic_grid_size(ct.byref(m.geometry), ct.byref(sp.spec), ct.byref(n)) == abi.PGXC_EINVAL
    assert ct.sizeof(abi.GridSpec) == 24
