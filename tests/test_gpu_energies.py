"""Post-SCF XC energies (pgxc_xc_energies): the energies of many functionals
on one density, each against the oracle's build with that functional."""
import numpy as np
import pytest

import oracle as O
from pgxc import abi, cases, lib

pytestmark = pytest.mark.gpu

GGA_SET = ["PBE", "revPBE", "PBEsol", "BP86", "PW91", "BPW91", "BLYP", "B3LYP", "PBE0", "HCTH", "HCTH407",
           "VMT", "VT84", "PBEN", "NRECMV92", "LB94", "VWN", "XALPHA", "PWLDA",
           "RBP", "RPW91"]


@pytest.mark.parametrize("precision,thr,tol", [("fp64", 0.0, 1e-10), ("mixed", 1e-10, 1e-7)], ids=["fp64", "int8"])
@pytest.mark.parametrize("ispin", [1, 2])
def test_energies_of_many_functionals(precision, thr, tol, ispin):
    c = cases.small_case(functional="PBE", seed=51, lmax=3, natoms=5, nocc=7, ispin=ispin)
    O.weight_case(c)
    with lib.Context(c, precision=precision, screen_threshold=thr, max_chunk_points=1024) as ctx:
        e, n = ctx.xc_energies(GGA_SET)
        h1, e1, n1 = ctx.build()                 # an ordinary build still follows
    ref_n = None
    for xc, got in zip(GGA_SET, e):
        c.functional = xc
        _, ref, ref_n = O.xc_build(c)
        assert abs(got - ref) < tol, (xc, got - ref)
    assert abs(n - ref_n) < tol
    c.functional = "PBE"
    _, rp, _ = O.xc_build(c)
    assert abs(e1 - rp) < tol and abs(e[0] - e1) < tol


@pytest.mark.parametrize("ispin", [1, 2])
@pytest.mark.parametrize("ctx_xc", ["PBE", "TPSS"])
def test_mgga_energies(ctx_xc, ispin):
    """Meta-GGA energies on the density of a GGA context of the FP64 build (tau
    formed on demand) and of a meta-GGA context (tau formed in every build),
    beside GGA and LDA ones, each against the oracle's build with that
    functional."""
    c = cases.small_case(functional=ctx_xc, seed=53, lmax=2, natoms=4, nocc=6, ispin=ispin)
    O.weight_case(c)
    names = ["TPSS", "M06L", "PBE", "M06", "VSXC", "VWN"]
    with lib.Context(c, precision="fp64", screen_threshold=0.0, max_chunk_points=1024) as ctx:
        e, n = ctx.xc_energies(names)
        e2, _ = ctx.xc_energies(["M06L"])        # a second pass reuses the tau buffer
    for xc, got in zip(names, e):
        c.functional = xc
        _, ref, ref_n = O.xc_build(c)
        assert abs(got - ref) < 1e-10, (xc, got - ref)
    assert abs(n - ref_n) < 1e-10
    assert abs(e2[0] - e[1]) < 1e-11


def test_mgga_energies_need_fp64_gradients():
    c = cases.small_case(functional="PBE", seed=54)
    O.weight_case(c)
    with lib.Context(c, precision="mixed", screen_threshold=1e-10) as ctx:
        with pytest.raises(lib.PgxcError):
            ctx.xc_energies(["TPSS"])            # INT8 GGA context: FP32 gradient planes
        e, _ = ctx.xc_energies(["PBE"])          # the context stays usable
        assert np.isfinite(e[0])


def test_energies_argument_errors():
    c = cases.small_case(functional="VWN", seed=52)
    O.weight_case(c)
    with lib.Context(c, screen_threshold=0.0) as ctx:
        with pytest.raises(lib.PgxcError):
            ctx.xc_energies(["PBE"])             # no density gradients in an LDA context
        e, _ = ctx.xc_energies(["VWN", "XALPHA", "PWLDA"])
        assert len(e) == 3
    with lib.Context(c, screen_threshold=-1.0) as ctx:
        with pytest.raises(lib.PgxcError):
            ctx.xc_energies(["VWN"])             # the dense layout has no energies pass
