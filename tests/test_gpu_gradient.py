"""Post-SCF XC nuclear gradient on the device (pgxc_xc_gradient) against the
oracle's independent restatement (itself checked against finite differences
in tests/test_gradient.py); every layout, both spins, LDA, GGA and meta-GGA."""
import numpy as np
import pytest

import oracle as O
from pgxc import cases, lib

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("layout", [("fp64", -1.0), ("fp64", 0.0), ("mixed", 1e-10)],
                         ids=["dense", "screened", "int8-screened"])
@pytest.mark.parametrize("xc,ispin,lmax", [("VWN", 1, 2), ("PBE", 1, 3), ("BLYP", 1, 2), ("PBE", 2, 2),
                                           ("B3LYP", 2, 3), ("HCTH407", 1, 2)])
def test_gradient_matches_oracle(xc, ispin, lmax, layout):
    precision, thr = layout
    if ispin == 2 and thr < 0:
        pytest.skip("the dense layout is closed shell")
    case = cases.small_case(functional=xc, seed=62, natoms=4, nocc=5, ispin=ispin, lmax=lmax)
    ref, re = O.xc_gradient(case)
    with lib.Context(case, weighted=False, precision=precision, screen_threshold=thr) as ctx:
        g, e = ctx.xc_gradient()
    scale = max(1.0, float(np.max(np.abs(ref))))
    assert abs(e - re) < 1e-10 * max(1.0, abs(re))
    np.testing.assert_allclose(g, ref, rtol=0, atol=1e-10 * scale)
    np.testing.assert_allclose(g.sum(0), 0.0, atol=1e-9 * scale)


@pytest.mark.parametrize("layout", [("fp64", 0.0), ("mixed", 1e-10)], ids=["screened", "int8-screened"])
@pytest.mark.parametrize("xc,ispin", [("TPSS", 1), ("TPSS", 2), ("M06L", 2), ("VSXC", 1)])
def test_mgga_gradient_matches_oracle(xc, ispin, layout):
    """Meta-GGAs: tau and df/dtau per point, and the tau terms (d_k d_j phi Y_j)
    in the orbital sums; the oracle's form is checked against finite
    differences in tests/test_gradient.py."""
    precision, thr = layout
    case = cases.small_case(functional=xc, seed=64, natoms=4, nocc=5, ispin=ispin, lmax=2)
    ref, re = O.xc_gradient(case)
    with lib.Context(case, weighted=False, precision=precision, screen_threshold=thr) as ctx:
        g, e = ctx.xc_gradient()
    scale = max(1.0, float(np.max(np.abs(ref))))
    assert abs(e - re) < 1e-10 * max(1.0, abs(re))
    np.testing.assert_allclose(g, ref, rtol=0, atol=1e-10 * scale)
    np.testing.assert_allclose(g.sum(0), 0.0, atol=1e-9 * scale)


def test_gradient_needs_the_raw_grid():
    case = cases.small_case(functional="PBE", seed=63)
    O.weight_case(case)
    with lib.Context(case, screen_threshold=0.0) as ctx:
        with pytest.raises(lib.PgxcError):
            ctx.xc_gradient()
