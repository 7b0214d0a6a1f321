"""Symmetry-adapted builds in the oracle (no GPU): the restatement of the
reference's irrep and partner loops (orbitals per partner, occ / partners in
the density, 1/partners in V, triangles of the irreps one after the other)
against the C1 oracle build of the same density projected onto the irreps,
V_i = 1/np_i sum_p U_ip^T V_C1 U_ip."""
import numpy as np
import pytest

import oracle as O
from pgxc import abi
from pgxc import symmetry as Y


def _c1_projected(case, ad, Cs, occs):
    C, occ = Y.c1_orbitals(ad, Cs, occs)
    case.C, case.occ, case.nocc = C, occ, C.shape[1]
    ham, e, n = O.xc_build(case)
    V = np.stack([O.unpack(ham, case.nbas, case.ispin, s) for s in range(case.ispin)])
    return Y.project(ad, V, case.ispin), e, n


@pytest.mark.parametrize("group,xc,ispin", [("C2v", "VWN", 1), ("C2v", "PBE", 1), ("C3v", "PBE", 1),
                                            ("C3v", "BLYP", 2), ("C2v", "PW91", 2)])
def test_symmetric_build_matches_projected_c1_build(group, xc, ispin):
    case, ad, Cs, occs = Y.symmetric_case(group, functional=xc, ispin=ispin)
    O.weight_case(case)
    h1, e1, n1 = O.xc_build_sym(case, ad, Cs, occs)
    h2, e2, n2 = _c1_projected(case, ad, Cs, occs)
    assert abs(e1 - e2) < 1e-11 and abs(n1 - n2) < 1e-11
    np.testing.assert_allclose(h1, h2, rtol=0, atol=1e-12)


def test_adaptation_is_orthonormal_and_complete():
    for g in Y.GROUPS:
        case, ad, _, _ = Y.symmetric_case(g)
        U = np.concatenate([M for Ui in ad.U for M in Ui], axis=1)
        assert U.shape == (case.nbas, case.nbas)
        np.testing.assert_allclose(U.T @ U, np.eye(case.nbas), atol=1e-12)
        assert int((ad.dims * ad.partners).sum()) == case.nbas
    assert list(Y.symmetric_case("C3v")[1].partners) == [1, 1, 2]


def test_one_irrep_identity_is_the_c1_build():
    case, _, _, _ = Y.symmetric_case("C2v", functional="PBE")
    O.weight_case(case)
    rng = np.random.default_rng(4)
    C = rng.normal(size=(case.nbas, 5, 1)) / np.sqrt(case.nbas)
    occ = np.full((5, 1), 2.0)
    ident = Y.Adaptation(["A"], np.array([case.nbas], dtype=np.int32), np.array([1], dtype=np.int32),
                         [[np.eye(case.nbas)]])
    h1, e1, n1 = O.xc_build_sym(case, ident, [C], [occ])
    case.C, case.occ, case.nocc = C, occ, 5
    h2, e2, n2 = O.xc_build(case)
    assert abs(e1 - e2) < 1e-12 and abs(n1 - n2) < 1e-12
    np.testing.assert_allclose(h1, h2, rtol=0, atol=1e-13)


def test_partner_order_does_not_change_the_energy():
    """The density sums over partners with occ / partners, so E_xc and N_el do
    not depend on the order in which the partners of the E irrep are given."""
    case, ad, Cs, occs = Y.symmetric_case("C3v", functional="PBE")
    O.weight_case(case)
    _, e1, n1 = O.xc_build_sym(case, ad, Cs, occs)
    swapped = Y.Adaptation(ad.names, ad.dims, ad.partners, [list(reversed(Ui)) for Ui in ad.U])
    _, e2, n2 = O.xc_build_sym(case, swapped, Cs, occs)
    assert abs(e1 - e2) < 1e-11 and abs(n1 - n2) < 1e-11


def reduced_and_full(case):
    """For the C2v case: the unique atoms' grids with weights times
    n_equal_atoms (the reference's grid), and the full grid of their images."""
    C2 = np.diag([-1.0, -1.0, 1.0])
    unique = {0: [np.eye(3)], 1: [np.eye(3), C2], 3: [np.eye(3), C2]}   # O; H pair; C pair
    pts, w_red, w_full, xyz_full = [], [], [], []
    for a, ops in unique.items():
        k = case.point_atom == a
        pts.append(case.grid_xyz[k])
        w_red.append(case.grid_w[k] * len(ops))
        for R in ops:
            xyz_full.append(case.grid_xyz[k] @ R.T)
            w_full.append(case.grid_w[k])
    full = Y.cases.Case(**{**case.__dict__})
    full.grid_xyz, full.grid_w = np.concatenate(xyz_full), np.concatenate(w_full)
    full.grid_wraw, full.point_atom = full.grid_w.copy(), np.zeros(len(full.grid_w), dtype=np.int32)
    red = Y.cases.Case(**{**case.__dict__})
    red.grid_xyz, red.grid_w = np.concatenate(pts), np.concatenate(w_red)
    red.grid_wraw, red.point_atom = red.grid_w.copy(), np.zeros(len(red.grid_w), dtype=np.int32)
    return red, full


def test_symmetry_reduced_grid_equals_full_grid():
    """The reference integrates on the grids of the unique atoms only, with
    weights times n_equal_atoms (mkgrid, grid_module.f90:3120-3125).  For the
    symmetry-adapted build that equals the build on the full grid made of the
    images of those grids under the group."""
    case, ad, Cs, occs = Y.symmetric_case("C2v", functional="PBE")
    O.weight_case(case)
    red, full = reduced_and_full(case)
    h1, e1, n1 = O.xc_build_sym(full, ad, Cs, occs)
    h2, e2, n2 = O.xc_build_sym(red, ad, Cs, occs)
    assert len(red.grid_w) < len(full.grid_w)
    assert abs(e1 - e2) < 1e-10 * abs(e1) and abs(n1 - n2) < 1e-10 * n1
    np.testing.assert_allclose(h2, h1, rtol=0, atol=1e-11)


def reduced_raw_grid(case, unique):
    """The reference's symmetry-reduced raw grid: the grids of one atom per
    class of equal atoms ({atom: n_equal_atoms}), raw weights times
    n_equal_atoms, each point moving with that atom."""
    keep = np.isin(case.point_atom, list(unique))
    red = Y.cases.Case(**{**case.__dict__})
    red.grid_xyz = case.grid_xyz[keep]
    red.point_atom = case.point_atom[keep]
    red.grid_wraw = case.grid_wraw[keep] * np.array([unique[int(a)] for a in red.point_atom])
    red.grid_w = None
    return red


def average_gradient(coords, ops, g):
    """post_scf_average_gradient (modules/post_scf_module.f90:1953-1982): the
    projection of a per-atom gradient on the totally symmetric displacements,
    (1/|G|) sum_R D(R) g with D(R) moving atom a's vector, rotated, to the
    atom at R R_a."""
    out = np.zeros_like(g)
    for R in ops:
        moved = coords @ R.T
        perm = [int(np.argmin(np.linalg.norm(coords - m, axis=1))) for m in moved]
        for a, b in enumerate(perm):
            out[b] += R @ g[a]
    return out / len(ops)


def test_reduced_grid_gradient_averages_to_full_grid_gradient():
    """The reference's symmetric XC gradient: the gradient of the reduced grid
    (every atom's derivative, points moving with their unique atom) averaged
    over the group equals the gradient on the full grid, whose atomic grids
    (Lebedev rules, invariant under the sign changes of x, y, z) are the
    group's images of the reduced ones.  Oracle only, C1 orbitals of the
    symmetric density."""
    case, ad, Cs, occs = Y.symmetric_case("C2v", functional="PBE")
    C, occ = Y.c1_orbitals(ad, Cs, occs)
    case.C, case.occ, case.nocc = C, occ, C.shape[1]
    ops, _ = Y.c2v()
    g_full, e_full = O.xc_gradient(case)
    red = reduced_raw_grid(case, {0: 1, 1: 2, 3: 2})
    g_red, e_red = O.xc_gradient(red)
    assert len(red.grid_wraw) < len(case.grid_wraw)
    assert abs(e_red - e_full) < 1e-10 * abs(e_full)
    assert np.max(np.abs(average_gradient(case.coords, ops, g_full) - g_full)) < 1e-10
    assert np.max(np.abs(g_red - g_full)) > 1e-6   # the reduced grid alone is not symmetric
    np.testing.assert_allclose(average_gradient(case.coords, ops, g_red), g_full, rtol=0, atol=1e-10)


@pytest.mark.parametrize("xc", ["TPSS", "M06L", "VSXC"])
def test_symmetric_mgga_build_matches_projected_c1_build(xc):
    """The oracle's irrep and partner loops with tau (occ / partners per
    partner, the tau term per irrep) against the C1 build of the expanded
    orbitals projected with U."""
    case, ad, Cs, occs = Y.symmetric_case("C2v", functional=xc)
    O.weight_case(case)
    h1, e1, n1 = O.xc_build_sym(case, ad, Cs, occs)
    C, occ = Y.c1_orbitals(ad, Cs, occs)
    c1 = Y.cases.Case(**{**case.__dict__})
    c1.C, c1.occ, c1.nocc = C, occ, C.shape[1]
    hc, ec, nc = O.xc_build(c1)
    hp = Y.project(ad, O.unpack(hc, c1.nbas)[None])
    assert abs(e1 - ec) < 1e-12 and abs(n1 - nc) < 1e-12
    np.testing.assert_allclose(h1, hp, rtol=0, atol=1e-12)
