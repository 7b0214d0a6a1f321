"""Atom-centred integration grids (host side, once per geometry).

Radial part: the Pople/Gill Euler-Maclaurin grid exactly as ParaGauss's
RADIALGRID builds it (modules/grid_module.f90:1246-1301):
    r_i = R (i/(N+1-i))^2,  w_i = 2 R^3 (N+1) i^5 / (N+1-i)^7,
points with r >= 40 bohr are cut from the outside in.

Angular part: the Lebedev-McLaren rules of INIGRD (:1359-2100), restated in
pgxc/lebedev.py, unrotated (the orientation the reference uses when weight
gradients are on, angular_grid :1339-1341).

One-centre weights are w_ang * w_rad * 4 pi (grid_main_calc, :425-432);
points are ordered atom -> radial shell -> angular point, as AGRID is.
"""
import numpy as np

from . import lebedev

# Radii (bohr) of Gill, Johnson & Pople, Chem. Phys. Lett. 209, 506 (1993),
# the "Pople radius" option of ParaGauss's GRIDATOM namelist.
POPLE_RADIUS = {1: 1.0000, 6: 1.2308, 7: 1.0256, 8: 0.8791}

RAD_LIMIT = 40.0



def radial_grid(nrad, radius):
    """RADIALGRID: returns (r, w) with the r >= 40 cut applied.

    The integer powers of the reference, (I/RHNI)**2, RCUR**3, (I/RHNI)**5 and
    RHNI**2, are written as products evaluated left to right, the same
    operations the device grid builder rounds, so both give identical points.
    """
    rhn = nrad + 1.0
    i_top = nrad
    for i in range(nrad, 0, -1):
        t = i / (rhn - i)
        i_top = i
        if radius * (t * t) < RAD_LIMIT:
            break
    else:
        i_top = 0
    i = np.arange(1, i_top + 1, dtype=np.float64)
    rhni = rhn - i
    t = i / rhni
    t2 = t * t
    r = radius * t2
    r3 = radius * radius * radius
    w = 2.0 * r3 * rhn * (t2 * t2 * t) / (rhni * rhni)
    return r, w


def angular_grid(nang):
    """INIGRD: the Lebedev-McLaren rule with nang points; weights sum to 1."""
    return lebedev.rule(nang)


def atomic_grids(coords, Z, nrad, nang):
    """grid_main_calc without pruning (NPART=1): returns xyz, raw w, host atom."""
    apts, aw = angular_grid(nang)
    xs, ws, owner = [], [], []
    for a, (c, z) in enumerate(zip(coords, Z)):
        r, wr = radial_grid(nrad, POPLE_RADIUS[int(z)])
        p = (r[:, None, None] * apts[None, :, :]).reshape(-1, 3) + c[None, :]
        w = (wr[:, None] * aw[None, :]).reshape(-1) * 16.0 * np.arctan(1.0)
        xs.append(p)
        ws.append(w)
        owner.append(np.full(len(w), a, dtype=np.int32))
    return np.concatenate(xs), np.concatenate(ws), np.concatenate(owner)


def becke_weights_numpy(coords, xyz, owner):
    """Becke partition (becke0, :2442-2497, art = 0) in numpy.

    Used only to orthonormalise the synthetic orbitals on a coarse grid; the
    weights that the XC build integrates with come from the device kernel.
    """
    natm = len(coords)
    r = np.sqrt(((xyz[:, None, :] - coords[None, :, :]) ** 2).sum(-1))
    p = np.ones_like(r)
    for i in range(natm):
        for k in range(i):
            d = np.linalg.norm(coords[i] - coords[k])
            mu = (r[:, i] - r[:, k]) / d
            for _ in range(3):
                mu = mu * (3.0 - mu * mu) / 2.0
            p[:, i] *= (1 - mu) / 2
            p[:, k] *= (1 + mu) / 2
    return p[np.arange(len(owner)), owner] / p.sum(1)
