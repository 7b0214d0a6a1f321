"""Symmetry-adapted GPU builds (pgxc_set_symmetry, pgxc_build_sym) against the
oracle's restatement of the reference's irrep and partner loops, in every
layout; bars 1e-10 (FP64) and 1e-7 (INT8)."""
import numpy as np
import pytest

import oracle as O
from pgxc import lib
from pgxc import symmetry as Y

pytestmark = pytest.mark.gpu

LAYOUTS = pytest.mark.parametrize("precision,thr,tol", [("fp64", -1.0, 1e-10), ("fp64", 0.0, 1e-10),
                                                        ("mixed", 1e-10, 1e-7)],
                                  ids=["fp64-dense", "fp64-screened", "int8-screened"])


@LAYOUTS
@pytest.mark.parametrize("group,xc", [("C2v", "VWN"), ("C2v", "PBE"), ("C3v", "PBE"), ("C3v", "BLYP")])
def test_symmetric_build_matches_oracle(group, xc, precision, thr, tol):
    case, ad, Cs, occs = Y.symmetric_case(group, functional=xc)
    O.weight_case(case)
    ref, re, rn = O.xc_build_sym(case, ad, Cs, occs)
    with lib.Context(case, precision=precision, screen_threshold=thr, max_chunk_points=2048) as ctx:
        ctx.set_symmetry(ad)
        assert ctx.sym_xc_length == len(ref)
        ham, e, n = ctx.build_sym(Cs, occs)
    assert abs(e - re) < tol and abs(n - rn) < tol, (e - re, n - rn)
    assert float(np.max(np.abs(ham - ref))) < tol


@pytest.mark.parametrize("precision,thr,tol", [("fp64", 0.0, 1e-10), ("mixed", 1e-10, 1e-7)], ids=["fp64", "int8"])
@pytest.mark.parametrize("group,xc", [("C3v", "PBE"), ("C2v", "VWN")])
def test_symmetric_open_shell(group, xc, precision, thr, tol):
    case, ad, Cs, occs = Y.symmetric_case(group, functional=xc, ispin=2)
    occs = [np.stack([o[:, 0], 0.5 * o[:, 1]], 1) for o in occs]
    O.weight_case(case)
    ref, re, rn = O.xc_build_sym(case, ad, Cs, occs)
    with lib.Context(case, precision=precision, screen_threshold=thr) as ctx:
        ctx.set_symmetry(ad)
        ham, e, n = ctx.build_sym(Cs, occs)
    assert abs(e - re) < tol and abs(n - rn) < tol
    assert float(np.max(np.abs(ham - ref))) < tol


def test_identity_adaptation_equals_c1_build_and_accumulates():
    case, _, _, _ = Y.symmetric_case("C2v", functional="PBE")
    O.weight_case(case)
    rng = np.random.default_rng(8)
    C = rng.normal(size=(case.nbas, 6, 1)) / np.sqrt(case.nbas)
    occ = np.full((6, 1), 2.0)
    case.C, case.occ, case.nocc = C, occ, 6
    ident = Y.Adaptation(["A"], np.array([case.nbas], dtype=np.int32), np.array([1], dtype=np.int32),
                         [[np.eye(case.nbas)]])
    with lib.Context(case, screen_threshold=0.0) as ctx:
        h1, e1, n1 = ctx.build()
        ctx.set_symmetry(ident)
        h2, e2, n2 = ctx.build_sym([C], [occ])
        h3, _, _ = ctx.build_sym([C], [occ], ham=h2.copy())   # accumulates (+=)
        h4, e4, n4 = ctx.build()                               # plain builds still work afterwards
    assert abs(e1 - e2) < 1e-12 and abs(n1 - n2) < 1e-12 and e4 == e1
    np.testing.assert_allclose(h2, h1, rtol=0, atol=1e-12)
    np.testing.assert_allclose(h3, 2 * h2, rtol=0, atol=1e-12)


def test_symmetry_argument_errors():
    case, ad, Cs, occs = Y.symmetric_case("C2v", functional="VWN")
    O.weight_case(case)
    with lib.Context(case, screen_threshold=0.0) as ctx:
        with pytest.raises(lib.PgxcError):
            ctx.build_sym(Cs, occs)           # no symmetry set yet
        bad = Y.Adaptation(ad.names, ad.dims, ad.partners, [list(U) for U in ad.U])
        bad.U[0][0] = np.vstack([bad.U[0][0], np.ones((1, bad.U[0][0].shape[1]))])  # a row past nbas
        with pytest.raises(lib.PgxcError):
            ctx.set_symmetry(bad)
        ctx.set_symmetry(ad)
        with pytest.raises(lib.PgxcError):
            ctx.build_sym(Cs[:-1] + [np.full_like(Cs[-1], np.nan)], occs)


@pytest.mark.parametrize("precision,thr,tol", [("fp64", 0.0, 1e-10), ("mixed", 1e-10, 1e-7)], ids=["fp64", "int8"])
def test_reduced_grid_build_matches_full_grid_oracle(precision, thr, tol):
    """The library on the reference's symmetry-reduced grid (unique atoms,
    weights times n_equal_atoms) against the oracle on the full grid."""
    from test_symmetry import reduced_and_full
    case, ad, Cs, occs = Y.symmetric_case("C2v", functional="PBE")
    O.weight_case(case)
    red, full = reduced_and_full(case)
    ref, re, rn = O.xc_build_sym(full, ad, Cs, occs)
    with lib.Context(red, precision=precision, screen_threshold=thr) as ctx:
        ctx.set_symmetry(ad)
        ham, e, n = ctx.build_sym(Cs, occs)
    assert abs(e - re) < tol and abs(n - rn) < tol
    assert float(np.max(np.abs(ham - ref))) < tol


@pytest.mark.parametrize("ispin", [1, 2])
def test_pseudo2d_symmetrisation_on_the_device(ispin):
    """pgxc_set_pseudo2d: the built matrix equals the oracle's restatement of
    xc_pseudo2d_sym applied to the build without it (bit for bit: the same
    halvings of sums and differences)."""
    case, ad, Cs, occs = Y.symmetric_case("C3v", functional="PBE", ispin=ispin)
    dims = list(ad.dims)
    i = int(np.argmax(dims))              # declare blocks in the largest irrep
    d = dims[i]
    first, half, pos = [], [], 0
    for h in (2, 3, 1):
        if pos + 2 * h > d:
            break
        first.append(pos)
        half.append(h)
        pos += 2 * h + 1
    nblocks = [0] * len(dims)
    nblocks[i] = len(first)
    with lib.Context(case, screen_threshold=0.0) as ctx:
        ctx.set_symmetry(ad)
        h0, e0, n0 = ctx.build_sym(Cs, occs)
        ctx.set_pseudo2d(nblocks, first, half)
        h1, e1, n1 = ctx.build_sym(Cs, occs)
        ctx.set_pseudo2d(None)
        h2, _, _ = ctx.build_sym(Cs, occs)
    want = O.pseudo2d_sym(h0, ispin, dims, nblocks, first, half)
    np.testing.assert_allclose(h1, want, rtol=0, atol=1e-14)
    assert not np.allclose(h1, h0)
    np.testing.assert_allclose(h2, h0, rtol=0, atol=1e-14)
    assert e1 == e0 and n1 == n0


def test_pseudo2d_rejects_bad_blocks():
    case, ad, Cs, occs = Y.symmetric_case("C2v", functional="VWN")
    with lib.Context(case, screen_threshold=0.0) as ctx:
        ctx.set_symmetry(ad)
        d = ad.dims[0]
        with pytest.raises(lib.PgxcError):
            ctx.set_pseudo2d([1] + [0] * (len(ad.dims) - 1), [0], [d])   # 2 * half > dims


@pytest.mark.parametrize("precision,thr", [("fp64", -1.0), ("fp64", 0.0), ("mixed", 1e-10)],
                         ids=["fp64-dense", "fp64-screened", "int8-screened"])
@pytest.mark.parametrize("group,xc,ispin", [("C2v", "PBE", 1), ("C3v", "BLYP", 1), ("C2v", "VWN", 2)])
def test_symmetric_gradient_matches_c1_oracle(group, xc, ispin, precision, thr):
    """pgxc_xc_gradient_sym against the oracle's C1 gradient of the same
    density (the irreps' orbitals expanded with U), full raw grid; 1e-10 of
    the largest component."""
    if ispin == 2 and thr < 0:
        pytest.skip("open shell needs the screened layout")
    case, ad, Cs, occs = Y.symmetric_case(group, functional=xc, ispin=ispin)
    C, occ = Y.c1_orbitals(ad, Cs, occs)
    c1 = Y.cases.Case(**{**case.__dict__})
    c1.C, c1.occ, c1.nocc = C, occ, C.shape[1]
    ref, re = O.xc_gradient(c1)
    with lib.Context(case, precision=precision, weighted=False, screen_threshold=thr) as ctx:
        ctx.set_symmetry(ad)
        g, e = ctx.xc_gradient_sym(Cs, occs)
        with pytest.raises(lib.PgxcError):
            ctx.xc_gradient(C, occ)   # a symmetric context takes the irreps' orbitals
    scale = float(np.max(np.abs(ref)))
    assert abs(e - re) < 1e-10 * max(1.0, abs(re))
    assert float(np.max(np.abs(g - ref))) < 1e-10 * max(scale, 1.0), float(np.max(np.abs(g - ref)))


def test_symmetric_gradient_on_reduced_grid_averages_to_full():
    """On the reference's symmetry-reduced grid the device gradient is
    grad_xc before post_scf_average_gradient: averaged over the group it
    equals the device gradient on the full grid, and the oracle's."""
    from test_symmetry import average_gradient, reduced_raw_grid
    case, ad, Cs, occs = Y.symmetric_case("C2v", functional="PBE")
    ops, _ = Y.c2v()
    red = reduced_raw_grid(case, {0: 1, 1: 2, 3: 2})
    with lib.Context(case, precision="fp64", weighted=False, screen_threshold=0.0) as ctx:
        ctx.set_symmetry(ad)
        g_full, e_full = ctx.xc_gradient_sym(Cs, occs)
    with lib.Context(red, precision="fp64", weighted=False, screen_threshold=0.0) as ctx:
        ctx.set_symmetry(ad)
        g_red, e_red = ctx.xc_gradient_sym(Cs, occs)
    C, occ = Y.c1_orbitals(ad, Cs, occs)
    c1 = Y.cases.Case(**{**case.__dict__})
    c1.C, c1.occ, c1.nocc = C, occ, C.shape[1]
    ref, _ = O.xc_gradient(c1)
    assert abs(e_red - e_full) < 1e-10 * abs(e_full)
    np.testing.assert_allclose(average_gradient(case.coords, ops, g_red), g_full, rtol=0, atol=1e-10)
    np.testing.assert_allclose(g_full, ref, rtol=0, atol=1e-10)


def test_symmetric_gradient_argument_errors():
    case, ad, Cs, occs = Y.symmetric_case("C2v", functional="VWN")
    with lib.Context(case, precision="fp64", weighted=False, screen_threshold=0.0) as ctx:
        with pytest.raises(lib.PgxcError):
            ctx.xc_gradient_sym(Cs, occs)     # no symmetry set
        ctx.set_symmetry(ad)
        with pytest.raises(lib.PgxcError):
            ctx.xc_gradient_sym(Cs[:-1] + [np.full_like(Cs[-1], np.nan)], occs)
    O.weight_case(case)
    with lib.Context(case, precision="fp64", screen_threshold=0.0) as ctx:   # Becke-weighted grid: no gradient
        ctx.set_symmetry(ad)
        with pytest.raises(lib.PgxcError):
            ctx.xc_gradient_sym(Cs, occs)
