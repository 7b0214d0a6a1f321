"""Atom-centred integration grids (host side, once per geometry).

Radial part: the Pople/Gill Euler-Maclaurin grid exactly as ParaGauss's
RADIALGRID builds it (modules/grid_module.f90:1246-1301):
    r_i = R (i/(N+1-i))^2,  w_i = 2 R^3 (N+1) i^5 / (N+1-i)^7,
points with r >= 40 bohr are cut from the outside in.

Angular part: ParaGauss uses Lebedev-McLaren tables (INIGRD, :1359-2100).
Those tables are published data that this project does not reproduce; the
angular rule here is a Gauss-Legendre (cos theta) x uniform (phi) product
rule of similar size and exactness (degree 2*n_theta-1).  The grid is an
input of the XC build (grdpts), so the choice does not affect parity: the
oracle and the GPU integrate the identical points and weights.

One-centre weights are w_ang * w_rad * 4 pi (grid_main_calc, :425-432);
points are ordered atom -> radial shell -> angular point, as AGRID is.
"""
import numpy as np

# Radii (bohr) of Gill, Johnson & Pople, Chem. Phys. Lett. 209, 506 (1993),
# the "Pople radius" option of ParaGauss's GRIDATOM namelist.
POPLE_RADIUS = {1: 1.0000, 6: 1.2308, 7: 1.0256, 8: 0.8791}

RAD_LIMIT = 40.0

# angular rules standing in for the Lebedev sizes named by the workloads
ANGULAR_RULES = {194: (10, 20), 302: (12, 25), 110: (8, 14), 50: (5, 10)}


def radial_grid(nrad, radius):
    """RADIALGRID: returns (r, w) with the r >= 40 cut applied."""
    rhn = nrad + 1
    i_top = nrad
    for i in range(nrad, 0, -1):
        r = radius * (i / (rhn - i)) ** 2
        i_top = i
        if r < RAD_LIMIT:
            break
    i = np.arange(1, i_top + 1, dtype=np.float64)
    rhni = rhn - i
    r = radius * (i / rhni) ** 2
    w = 2 * radius ** 3 * rhn * (i / rhni) ** 5 / rhni ** 2
    return r, w


def angular_grid(n_theta, n_phi):
    """Product rule on the unit sphere; weights sum to 1."""
    x, wx = np.polynomial.legendre.leggauss(n_theta)
    phi = (np.arange(n_phi) + 0.5) * (2 * np.pi / n_phi)
    ct_, ph = np.meshgrid(x, phi, indexing="ij")
    st = np.sqrt(1 - ct_ ** 2)
    pts = np.stack([st * np.cos(ph), st * np.sin(ph), ct_], axis=-1).reshape(-1, 3)
    w = np.repeat(wx / 2.0, n_phi) / n_phi
    return pts, w


def atomic_grids(coords, Z, nrad, nang):
    """grid_main_calc without pruning (NPART=1): returns xyz, raw w, host atom."""
    nt, nph = ANGULAR_RULES[nang]
    apts, aw = angular_grid(nt, nph)
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
