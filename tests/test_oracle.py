"""Self-consistency tests of the FP64 CPU oracle (no GPU).

The reference holds no golden vectors at the XC-build boundary, so the
oracle is pinned by known-answer properties: derivatives against finite
differences (the pattern of the reference's test-xc harness,
guile/paragauss.scm:347-363), dE_xc/dC = 2 occ V C, charge normalisation,
basis normalisation and invariances.
"""
import numpy as np
import pytest

import oracle as O
from pgxc import cases


RHO = np.array([1e-12, 1e-6, 1e-3, 0.05, 0.7, 3.0, 120.0])
GAM = np.array([1e-20, 1e-9, 1e-5, 0.02, 0.9, 10.0, 5e4])


ALL_XC = ["VWN", "PBE", "revPBE", "PBEsol", "BP86"]


@pytest.mark.parametrize("xc", ALL_XC)
def test_functional_derivatives_fd(xc):
    rho = RHO.copy()
    gam = GAM.copy()
    f, fr, fg = O.functionals(xc, 1, rho, gam)
    h = 1e-6 * rho
    fp, _, _ = O.functionals(xc, 1, rho + h, gam)
    fm, _, _ = O.functionals(xc, 1, rho - h, gam)
    num = (fp - fm) / (2 * h)
    np.testing.assert_allclose(fr[:, 0], num, rtol=2e-6, atol=1e-12)
    if xc != "VWN":
        hg = 1e-4 * gam
        gp, _, _ = O.functionals(xc, 1, rho, gam + hg)
        gm, _, _ = O.functionals(xc, 1, rho, gam - hg)
        # only where the gamma dependence is above the rounding of f
        ok = np.abs(fg[:, 0] * hg) > 1e-9 * np.abs(f)
        assert ok.sum() >= 4
        np.testing.assert_allclose(fg[ok, 0], ((gp - gm) / (2 * hg))[ok], rtol=1e-6)


@pytest.mark.parametrize("xc", ALL_XC)
def test_functional_spin_consistency(xc):
    """ispin=2 with rho_a = rho_b = rho/2 reproduces the ispin=1 functional."""
    rho = RHO.copy()
    gam = GAM.copy()
    f1, fr1, fg1 = O.functionals(xc, 1, rho, gam)
    r2 = np.stack([rho / 2, rho / 2], 1)
    g2 = np.stack([gam / 4, gam / 4, gam / 4], 1)
    f2, fr2, fg2 = O.functionals(xc, 2, r2, g2)
    np.testing.assert_allclose(f2, f1, rtol=1e-12, atol=1e-300)
    np.testing.assert_allclose(fr2[:, 0], fr1[:, 0], rtol=1e-10, atol=1e-14)
    if xc != "VWN":
        # d/dg_aa + d/dg_bb + d/dg_ab of g = g_aa + g_bb + 2 g_ab
        np.testing.assert_allclose((fg2[:, 0] + fg2[:, 1] + fg2[:, 2]) / 4, fg1[:, 0], rtol=1e-9, atol=1e-14)


def test_pbe_variants_closed_form():
    """revPBE differs from PBE only in the exchange kappa (1.245): the
    difference of the two is e_x (G_rev - G_pbe), G = kappa mu s^2/(kappa + mu s^2)
    (g_becke86_form); without a gradient PBEsol and revPBE equal PBE."""
    rho, gam = RHO[1:], GAM[1:]
    pi = 3.14159265358979324
    ex = -(3 / 4) * (3 / pi) ** (1 / 3) * rho ** (4 / 3)
    s2 = gam / (4 * (3 * pi ** 2) ** (2 / 3) * rho ** (8 / 3))
    mu = 0.066725 * pi ** 2 / 3
    g = lambda k, m: k * m * s2 / (k + m * s2)
    fp, _, _ = O.functionals("PBE", 1, rho, gam)
    fr, _, _ = O.functionals("revPBE", 1, rho, gam)
    want = ex * (g(1.245, mu) - g(0.804, mu))
    assert np.all(np.abs((fr - fp) - want) <= 1e-9 * np.abs(want) + 1e-13 * np.abs(fp)), (fr - fp, want)
    z = np.zeros_like(rho)
    for xc in ("revPBE", "PBEsol"):
        np.testing.assert_array_equal(O.functionals(xc, 1, rho, z)[0], O.functionals("PBE", 1, rho, z)[0])


def test_functional_zero_density():
    for xc in ALL_XC:
        f, fr, fg = O.functionals(xc, 1, np.zeros(3), np.zeros(3))
        assert np.all(np.isfinite(f)) and np.all(np.abs(f) < 1e-40)
        assert np.all(np.isfinite(fr)) and np.all(np.isfinite(fg))


def test_slater_closed_form():
    rho = np.array([0.01, 0.3, 2.0])
    f, fr, _ = O.functionals("VWN", 1, rho)
    fx = -(3 / 4) * (3 / np.pi) ** (1 / 3) * rho ** (4 / 3)
    # VWN correlation is a small negative addition
    assert np.all(f < fx) and np.all(f > 1.3 * fx)


def test_basis_normalised_and_gradients(small_cases):
    w = O.weight_case(cases.config(1))
    S = O.overlap(w)
    # self-overlaps of normalised contracted functions are 1 (to grid accuracy)
    np.testing.assert_allclose(np.diag(S), 1.0, atol=1e-3)
    c = small_cases["PBE"]
    rng = np.random.default_rng(3)
    pts = c.coords[0] + rng.normal(scale=1.2, size=(40, 3))
    phi, gr = O.orbitals(c, pts)
    h = 1e-5
    for d in range(3):
        e = np.zeros(3)
        e[d] = h
        pp, _ = O.orbitals(c, pts + e, grads=False)
        pm, _ = O.orbitals(c, pts - e, grads=False)
        np.testing.assert_allclose(gr[:, d, :], (pp - pm) / (2 * h), rtol=1e-5, atol=1e-8)


@pytest.mark.parametrize("xc", ALL_XC)
def test_dE_dC_equals_2_occ_V_C(small_cases, xc):
    if xc in small_cases:
        c = small_cases[xc]
    else:
        c = cases.small_case(functional=xc, seed=13)
        O.weight_case(c)
    ham, e0, _ = O.xc_build(c)
    V = O.unpack(ham, c.nbas)
    grad = 2 * c.occ[:, 0][None, :] * (V @ c.C[:, :, 0])
    rng = np.random.default_rng(5)
    d = rng.normal(size=c.C.shape)
    h = 1e-5
    C0 = c.C.copy()
    c.C = C0 + h * d
    _, ep, _ = O.xc_build(c)
    c.C = C0 - h * d
    _, em, _ = O.xc_build(c)
    c.C = C0
    num = (ep - em) / (2 * h)
    ana = np.sum(grad * d[:, :, 0])
    assert abs(num - ana) < 1e-6 * max(1.0, abs(ana)), (num, ana)


def test_charge_and_batching(small_cases):
    c = small_cases["PBE"]
    h1, e1, n1 = O.xc_build(c, vla=128)
    h2, e2, n2 = O.xc_build(c, vla=37, nthreads=1)
    assert abs(e1 - e2) < 1e-11 and abs(n1 - n2) < 1e-11
    np.testing.assert_allclose(h1, h2, atol=1e-12)
    # orbitals were orthonormalised on a coarser grid: charge is close to 2*nocc
    assert abs(n1 - 2 * c.nocc) < 0.05 * 2 * c.nocc


def test_translation_invariance():
    c = cases.small_case(functional="PBE", seed=21)
    O.weight_case(c)
    h1, e1, n1 = O.xc_build(c)
    shift = np.array([0.37, -1.25, 2.5])
    c.coords = c.coords + shift
    c.grid_xyz = c.grid_xyz + shift
    h2, e2, n2 = O.xc_build(c)
    assert abs(e1 - e2) < 1e-10 * abs(e1)
    np.testing.assert_allclose(h1, h2, atol=1e-10)


def test_open_shell_matches_closed_shell():
    """ispin=2 with identical alpha/beta orbitals (occ 1) equals ispin=1 (occ 2)."""
    for xc in ("VWN", "PBE"):
        c = cases.small_case(functional=xc, seed=31)
        O.weight_case(c)
        h1, e1, n1 = O.xc_build(c)
        c.ispin = 2
        c.C = np.concatenate([c.C, c.C], axis=2)
        c.occ = np.ones((c.nocc, 2))
        h2, e2, n2 = O.xc_build(c)
        assert abs(e1 - e2) < 1e-10 * abs(e1)
        assert abs(n1 - n2) < 1e-10 * n1
        np.testing.assert_allclose(h2[0::2], h1, atol=1e-10)
        np.testing.assert_allclose(h2[1::2], h1, atol=1e-10)


def test_becke_partition_of_unity(small_cases):
    """Becke weights of all atoms at a point sum to one."""
    c = small_cases["VWN"]
    pts = c.grid_xyz[::97]
    tot = np.zeros(len(pts))
    for a in range(len(c.coords)):
        cc = cases.Case(**{**c.__dict__})
        cc.grid_xyz = pts
        cc.grid_wraw = np.ones(len(pts))
        cc.point_atom = np.full(len(pts), a, dtype=np.int32)
        tot += O.becke(cc)
    np.testing.assert_allclose(tot, 1.0, atol=1e-13)
