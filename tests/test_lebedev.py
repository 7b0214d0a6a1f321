"""The Lebedev-McLaren angular rules (INIGRD, modules/grid_module.f90:1359-2100).

Each rule must put its points on the unit sphere, carry weights that sum to
one, and integrate every monomial x^a y^b z^c of total degree up to the rule's
order exactly (to the 12 digits INIGRD writes its constants with).
"""
import math

import numpy as np
import pytest

from pgxc import grid as G, lebedev

# points -> polynomial degree integrated exactly (the L of INIGRD's messages)
DEGREE = {6: 3, 8: 3, 12: 3, 14: 5, 26: 7, 38: 9, 50: 11, 78: 13, 86: 15, 110: 17, 146: 19, 194: 23, 302: 29}


def dfact(n):
    return 1 if n <= 0 else n * dfact(n - 2)


def sphere_mean(a, b, c):
    """(1/4 pi) * integral of x^a y^b z^c over the unit sphere."""
    if a % 2 or b % 2 or c % 2:
        return 0.0
    return dfact(a - 1) * dfact(b - 1) * dfact(c - 1) / dfact(a + b + c + 1)


@pytest.mark.parametrize("n", sorted(lebedev.RULES))
def test_rule_is_exact_to_its_degree(n):
    pts, w = lebedev.rule(n)
    assert pts.shape == (n, 3)
    np.testing.assert_allclose(np.linalg.norm(pts, axis=1), 1.0, atol=1e-14)
    assert abs(w.sum() - 1.0) < 1e-10
    # every point distinct
    assert len({tuple(np.round(p, 12)) for p in pts}) == n
    L = DEGREE[n]
    worst = 0.0
    for a in range(L + 1):
        for b in range(L + 1 - a):
            for c in range(L + 1 - a - b):
                q = float(np.sum(w * pts[:, 0] ** a * pts[:, 1] ** b * pts[:, 2] ** c))
                worst = max(worst, abs(q - sphere_mean(a, b, c)))
    assert worst < 1e-10, worst


def test_degree_is_not_higher_than_stated():
    """The next even degree is not integrated by the 194-point rule."""
    pts, w = lebedev.rule(194)
    errs = []
    for a in range(0, 25, 2):
        for b in range(0, 25 - a, 2):
            c = 24 - a - b
            q = float(np.sum(w * pts[:, 0] ** a * pts[:, 1] ** b * pts[:, 2] ** c))
            errs.append(abs(q - sphere_mean(a, b, c)))
    assert max(errs) > 1e-9


def test_order_codes_map_to_point_counts():
    for code, n in lebedev.NANG_TO_POINTS.items():
        assert n in lebedev.RULES


def test_atomic_grid_uses_the_rule():
    coords = np.array([[0.0, 0.0, 0.0]])
    xyz, w, owner = G.atomic_grids(coords, np.array([8]), 10, 302)
    r, wr = G.radial_grid(10, G.POPLE_RADIUS[8])
    assert len(w) == len(r) * 302
    # the one-centre weights integrate exp(-r^2) over space: pi^(3/2)
    f = np.exp(-np.sum(xyz ** 2, axis=1))
    xyz2, w2, _ = G.atomic_grids(coords, np.array([8]), 200, 302)
    assert abs(np.sum(w2 * np.exp(-np.sum(xyz2 ** 2, axis=1))) - math.pi ** 1.5) < 1e-6
    assert np.all(owner == 0) and np.all(np.isfinite(f))
