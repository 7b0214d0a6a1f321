"""The oracle's TPSS (meta-GGA) point functional: derivatives against
central differences, the closed shell against the open-shell form at equal
spins, and the uniform-gas limit (TPSS reduces to Slater + PW92 there).
The reference holds no golden vectors for TPSS; these pins are the
functional's own properties."""
import numpy as np
import pytest

import oracle as O

CT = 0.3 * (3 * np.pi ** 2) ** (2.0 / 3.0)   # tau of the uniform gas = CT rho^(5/3)


def _points(rng, n=64, ispin=1):
    rho = 10.0 ** rng.uniform(-3, 1, size=(n, ispin))
    s = rng.uniform(0.05, 2.0, size=(n, ispin))              # reduced gradients
    kf = (3 * np.pi ** 2 * rho * ispin) ** (1 / 3)
    gs = (2 * kf * s * rho) ** 2 / ispin                      # |grad rho_s|^2
    tw = gs / (8 * rho)
    tu = CT * (ispin * rho) ** (5 / 3) / ispin
    tau = np.maximum(tw, tu) * rng.uniform(1.0, 3.0, size=(n, ispin))  # tau >= tau_W
    if ispin == 1:
        return rho, gs, tau
    gab = np.sqrt(gs[:, 0] * gs[:, 1]) * rng.uniform(-0.9, 0.9, size=n)
    return rho, np.column_stack([gs[:, 0], gs[:, 1], gab]), tau


@pytest.mark.parametrize("ispin", [1, 2])
def test_tpss_derivatives_match_central_differences(ispin):
    rng = np.random.default_rng(3 + ispin)
    rho, gam, tau = _points(rng, ispin=ispin)
    f, fr, fg, ft = O.functionals_mgga("TPSS", ispin, rho, gam, tau)
    assert np.all(np.isfinite(f)) and np.all(f < 0)
    for arr, der in ((rho, fr), (gam, fg), (tau, ft)):
        for k in range(arr.shape[1]):
            h = 1e-5 * np.maximum(np.abs(arr[:, k]), 1e-8)
            up, dn = arr.copy(), arr.copy()
            up[:, k] += h
            dn[:, k] -= h
            args = lambda a: (a if arr is rho else rho, a if arr is gam else gam, a if arr is tau else tau)
            fd = (O.functionals_mgga("TPSS", ispin, *args(up))[0] - O.functionals_mgga("TPSS", ispin, *args(dn))[0]) \
                / (2 * h)
            scale = np.abs(f) / np.maximum(np.abs(arr[:, k]), 1e-300)
            np.testing.assert_allclose(der[:, k], fd, rtol=2e-6, atol=1e-8 * float(np.max(scale)))


def test_tpss_closed_shell_equals_open_shell_at_equal_spins():
    rng = np.random.default_rng(11)
    rho, gam, tau = _points(rng, ispin=1)
    f1, fr1, fg1, ft1 = O.functionals_mgga("TPSS", 1, rho, gam, tau)
    r2 = np.column_stack([rho[:, 0] / 2, rho[:, 0] / 2])
    g2 = np.column_stack([gam[:, 0] / 4] * 3)
    t2 = np.column_stack([tau[:, 0] / 2, tau[:, 0] / 2])
    f2, fr2, fg2, ft2 = O.functionals_mgga("TPSS", 2, r2, g2, t2)
    np.testing.assert_allclose(f2, f1, rtol=1e-13)
    np.testing.assert_allclose(fr2[:, 0], fr1[:, 0], rtol=1e-10)
    np.testing.assert_allclose(0.25 * (fg2[:, 0] + fg2[:, 1] + fg2[:, 2]), fg1[:, 0], rtol=1e-10)
    np.testing.assert_allclose(0.5 * (ft2[:, 0] + ft2[:, 1]), ft1[:, 0], rtol=1e-10)


def test_tpss_uniform_gas_limit_is_slater_plus_pw92():
    """gamma = 0 and tau = CT rho^(5/3): the exchange enhancement is 1 and
    the correlation is PW92 (H(t = 0) = 0, z = 0)."""
    rho = np.logspace(-3, 1.5, 40)[:, None]
    f, _, _, _ = O.functionals_mgga("TPSS", 1, rho, np.zeros_like(rho), CT * rho ** (5 / 3))
    ref, _, _ = O.functionals("PWLDA", 1, rho)
    np.testing.assert_allclose(f, ref, rtol=1e-12)


@pytest.mark.parametrize("xc", ["M06L", "M06", "VSXC"])
def test_vs_family_open_shell_derivatives_match_central_differences(xc):
    rng = np.random.default_rng(31)
    rho, gam, tau = _points(rng, ispin=2)
    f, fr, fg, ft = O.functionals_mgga(xc, 2, rho, gam, tau)
    assert np.all(np.isfinite(f))
    np.testing.assert_array_equal(fg[:, 2], 0.0)   # gamma_ab does not enter these functionals
    for arr, der, ks in ((rho, fr, (0, 1)), (gam, fg, (0, 1)), (tau, ft, (0, 1))):
        for k in ks:
            h = 1e-5 * np.abs(arr[:, k])
            up, dn = arr.copy(), arr.copy()
            up[:, k] += h
            dn[:, k] -= h
            args = lambda a: (a if arr is rho else rho, a if arr is gam else gam, a if arr is tau else tau)
            fd = (O.functionals_mgga(xc, 2, *args(up))[0] - O.functionals_mgga(xc, 2, *args(dn))[0]) / (2 * h)
            scale = np.abs(f) / np.abs(arr[:, k])
            np.testing.assert_allclose(der[:, k], fd, rtol=2e-6, atol=1e-8 * float(np.max(scale)))


@pytest.mark.parametrize("xc,factor", [("M06L", 1.0), ("M06", 1.0), ("VSXC", 0.5)])
def test_vs_family_closed_shell_is_the_open_form_at_equal_spins(xc, factor):
    """The closed shell is the open-shell form at rho/2, gamma/4, tau/2;
    M06-L and M06 take the chain rule of that, VSXC half of it (the
    reference's vsxc_X / vsxc_C wrappers scale by 0.5, 0.25, 0.5)."""
    rng = np.random.default_rng(12)
    rho, gam, tau = _points(rng, ispin=1)
    f1, fr1, fg1, ft1 = O.functionals_mgga(xc, 1, rho, gam, tau)
    r2 = np.column_stack([rho[:, 0] / 2, rho[:, 0] / 2])
    g2 = np.column_stack([gam[:, 0] / 4, gam[:, 0] / 4, gam[:, 0] / 4])
    t2 = np.column_stack([tau[:, 0] / 2, tau[:, 0] / 2])
    f2, fr2, fg2, ft2 = O.functionals_mgga(xc, 2, r2, g2, t2)
    np.testing.assert_allclose(f1, f2, rtol=1e-13)
    np.testing.assert_allclose(fr1[:, 0], factor * fr2[:, 0], rtol=1e-10)
    np.testing.assert_allclose(fg1[:, 0], factor * 0.5 * fg2[:, 0], rtol=1e-10)
    np.testing.assert_allclose(ft1[:, 0], factor * ft2[:, 0], rtol=1e-10)


def test_minnesota_uniform_gas_limits():
    """gamma = 0, tau = CT rho^(5/3): M06-L reduces to Slater + PW92 (a0 + d0 = 1
    in exchange, c0 + d0 = 1 in both correlation series) and the grid part of
    M06 to 0.73 Slater + PW92 (a0 + d0 = 0.73; the 0.27 is exact exchange)."""
    rho = np.logspace(-3, 1.5, 40)[:, None]
    tau = CT * rho ** (5 / 3)
    pwlda, _, _ = O.functionals("PWLDA", 1, rho)
    slater, _, _ = O.functionals("XALPHA", 1, rho)
    f6l, _, _, _ = O.functionals_mgga("M06L", 1, rho, np.zeros_like(rho), tau)
    f6, _, _, _ = O.functionals_mgga("M06", 1, rho, np.zeros_like(rho), tau)
    np.testing.assert_allclose(f6l, pwlda, rtol=1e-12)
    np.testing.assert_allclose(f6, pwlda - 0.27 * slater, rtol=1e-11)
