"""Post-SCF XC nuclear gradient in the oracle (no GPU): against central
differences of the energy on the grid that moves with its atoms, with the
Becke weights recomputed at each displaced geometry; and translation
invariance (the gradients sum to zero)."""
import numpy as np
import pytest

import oracle as O
from pgxc import cases


def _energy(case):
    c = cases.Case(**{**case.__dict__})
    O.weight_case(c)
    return O.xc_build(c)[1]


def _displaced(case, atom, k, h):
    c = cases.Case(**{**case.__dict__})
    c.coords = case.coords.copy()
    c.coords[atom, k] += h
    c.grid_xyz = case.grid_xyz.copy()
    c.grid_xyz[case.point_atom == atom, k] += h     # the atom's grid moves with it
    return c


@pytest.mark.parametrize("xc,ispin", [("VWN", 1), ("PBE", 1), ("BLYP", 2), ("PBE", 2), ("PW91", 2),
                                     ("TPSS", 1), ("TPSS", 2), ("M06L", 2), ("VSXC", 2)])
def test_gradient_matches_finite_differences(xc, ispin):
    """(closed-shell LYP is left out: its df/dgamma is not the derivative of its energy; the same
    holds for the closed-shell derivatives of the VSXC family, which the meta-GGA cases therefore
    take open shell; the meta-GGAs add the terms of tau moving with the functions)"""
    case = cases.small_case(functional=xc, seed=61, natoms=3, nocc=4, ispin=ispin, nrad=14, lmax=2)
    g, e = O.xc_gradient(case)
    assert abs(e - _energy(case)) < 1e-11
    h = 1e-4
    for atom in range(len(case.coords)):
        for k in range(3):
            num = (_energy(_displaced(case, atom, k, h)) - _energy(_displaced(case, atom, k, -h))) / (2 * h)
            assert abs(g[atom, k] - num) < 2e-7 * max(1.0, abs(num)), (atom, k, g[atom, k], num)
    np.testing.assert_allclose(g.sum(0), 0.0, atol=1e-10)
