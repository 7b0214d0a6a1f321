"""Symmetry-adapted bases for pgxc_set_symmetry / pgxc_build_sym.

The reference reads its symmetry adaptation (the coefficients of each
symmetry-adapted function over the equal atoms' functions, per irrep and
partner) from its symmetry module; this builds the same kind of table from
point-group operations for a molecule the caller describes:

  D(R)        the representation of operation R on the C1 basis,
              (R chi)(r) = chi(R^-1 r) = sum_b chi_b(r) D(R)_ba, from basis
              values at sample points (exact up to rounding);
  P^G_kl      (d/h) sum_R G(R)_kl D(R), the projectors of irrep G;
  partner 1   an orthonormal basis of the range of P^G_11,
  partner p   P^G_p1 applied to the partner-1 functions.

Groups are given as (operations, irreps), each irrep (name, matrices per
operation); C2V and C3V are provided.
"""
from dataclasses import dataclass

import numpy as np

from . import cases


def _rot_z(t):
    c, s = np.cos(t), np.sin(t)
    return np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])


def _mirror_z(t):
    """Reflection through the plane containing z and the direction at angle t."""
    c, s = np.cos(2 * t), np.sin(2 * t)
    return np.array([[c, s, 0.0], [s, -c, 0.0], [0.0, 0.0, 1.0]])


def c2v():
    ops = [np.eye(3), np.diag([-1.0, -1.0, 1.0]), np.diag([1.0, -1.0, 1.0]), np.diag([-1.0, 1.0, 1.0])]
    ch = {"A1": [1, 1, 1, 1], "A2": [1, 1, -1, -1], "B1": [1, -1, 1, -1], "B2": [1, -1, -1, 1]}
    return ops, [(k, [np.array([[float(x)]]) for x in v]) for k, v in ch.items()]


def c3v():
    t = 2 * np.pi / 3
    ops = [np.eye(3), _rot_z(t), _rot_z(2 * t), _mirror_z(0.0), _mirror_z(t), _mirror_z(2 * t)]
    a1 = [np.array([[1.0]])] * 6
    a2 = [np.array([[1.0]])] * 3 + [np.array([[-1.0]])] * 3
    e = [R[:2, :2].copy() for R in ops]  # (x, y) spans E
    return ops, [("A1", a1), ("A2", a2), ("E", e)]


GROUPS = {"C2v": c2v, "C3v": c3v}


def representation(case, R, npts=3000, seed=0):
    """D(R) on the C1 basis of case (nbas x nbas)."""
    rng = np.random.default_rng(seed)
    centre = case.coords.mean(0)
    X = centre + rng.normal(scale=2.0, size=(npts, 3))
    A = cases.basis_values(case, X)
    B = cases.basis_values(case, X @ R)   # chi(R^-1 x) for orthogonal R: rows x R
    D, *_ = np.linalg.lstsq(A, B, rcond=None)
    D[np.abs(D) < 1e-9] = 0.0
    return D


@dataclass
class Adaptation:
    names: list
    dims: np.ndarray       # int32 [n_irrep]
    partners: np.ndarray   # int32 [n_irrep]
    U: list                # U[i][p]: (nbas x dims_i)

    @property
    def n_irrep(self):
        return len(self.dims)

    def entries(self, tol=1e-12):
        """(irrep, partner, fn, ao, coef) arrays of the nonzero entries of U."""
        out = [[], [], [], [], []]
        for i, Ui in enumerate(self.U):
            for p, M in enumerate(Ui):
                a, f = np.nonzero(np.abs(M) > tol)
                out[0].append(np.full(len(a), i))
                out[1].append(np.full(len(a), p))
                out[2].append(f)
                out[3].append(a)
                out[4].append(M[a, f])
        i32 = lambda x: np.ascontiguousarray(np.concatenate(x), dtype=np.int32)
        return i32(out[0]), i32(out[1]), i32(out[2]), i32(out[3]), np.ascontiguousarray(np.concatenate(out[4]))

    def xc_length(self, ispin):
        return int(ispin * sum(int(d) * (int(d) + 1) // 2 for d in self.dims))


def adapt(case, group):
    """Symmetry adaptation of case's C1 basis under group (a GROUPS key or an
    (operations, irreps) pair).  The molecule must be symmetric under the
    operations, with identical bases on equal atoms."""
    ops, irreps = GROUPS[group]() if isinstance(group, str) else group
    h = len(ops)
    D = [representation(case, R) for R in ops]
    names, dims, partners, U = [], [], [], []
    for name, mats in irreps:
        d = mats[0].shape[0]
        P = lambda k, l: (d / h) * sum(m[k, l] * Dm for m, Dm in zip(mats, D))
        P11 = P(0, 0)
        # orthonormal basis of range(P11), deterministic: eigenvectors of the projector
        w, V = np.linalg.eigh(0.5 * (P11 + P11.T))
        B = V[:, w > 0.5]
        B[np.abs(B) < 1e-10] = 0.0
        names.append(name)
        dims.append(B.shape[1])
        partners.append(d)
        U.append([B] + [P(p, 0) @ B for p in range(1, d)])
    return Adaptation(names, np.array(dims, dtype=np.int32), np.array(partners, dtype=np.int32), U)


def symmetric_case(group, functional="PBE", seed=5, ispin=1, nrad=16, nang=50, nocc_per_irrep=2):
    """A small molecule with the symmetry of group, identical bases on equal
    atoms, its adaptation and random orbitals per irrep: (case, adaptation,
    C list, occ list)."""
    rng = np.random.default_rng(seed)
    if group == "C2v":
        els = ["O", "H", "H", "C", "C"]
        xyz = np.array([[0.0, 0.0, 0.3], [1.5, 0.0, -0.9], [-1.5, 0.0, -0.9], [0.0, 1.3, 1.4], [0.0, -1.3, 1.4]])
    elif group == "C3v":
        t = 2 * np.pi / 3
        els = ["N", "H", "H", "H", "C"]
        xyz = np.array([[0.0, 0.0, 0.2]] + [[1.8 * np.cos(k * t), 1.8 * np.sin(k * t), -0.5] for k in range(3)]
                       + [[0.0, 0.0, 2.6]])
    else:
        raise ValueError(group)
    # one basis per element, repeated on equal atoms
    shells = {"H": (2, 1), "C": (2, 2, 1), "N": (2, 2, 1), "O": (2, 2, 1)}
    per_el = {}
    for el in dict.fromkeys(els):
        per_el[el] = cases.make_basis([el], np.random.default_rng(seed + cases.Z_OF[el]), (0.1, 50.0), shells)
    parts = [per_el[el] for el in els]
    cat = lambda k: np.concatenate([p[k] for p in parts])
    shell_atom = np.concatenate([np.full(len(p["shell_l"]), a, dtype=np.int32) for a, p in enumerate(parts)])
    b = dict(shell_atom=shell_atom, shell_l=cat("shell_l"), shell_nexp=cat("shell_nexp"),
             shell_nunc=cat("shell_nunc"), shell_ncontr=cat("shell_ncontr"), exponents=cat("exponents"),
             norms=cat("norms"), contractions=cat("contractions"), nbas=int(sum(p["nbas"] for p in parts)))
    Z = np.array([cases.Z_OF[e] for e in els], dtype=np.int32)
    gx, gw, owner = cases.G.atomic_grids(xyz, Z, nrad, nang)
    case = cases.Case(name=f"sym-{group}-{functional}", coords=xyz, Z=Z, grid_xyz=gx, grid_wraw=gw,
                      point_atom=owner, functional=functional, nocc=0, ispin=ispin, **b)
    ad = adapt(case, group)
    Cs, occs = [], []
    for i, d in enumerate(ad.dims):
        n = int(min(nocc_per_irrep, d))
        Cs.append(rng.normal(size=(int(d), n, ispin)) / np.sqrt(max(int(d), 1)))
        occs.append(np.full((n, ispin), 2.0 / ispin))
    return case, ad, Cs, occs


def c1_orbitals(ad, Cs, occs):
    """The same density in the C1 basis: orbitals U_ip C_i with occupations
    occ_i / partners_i, stacked over (irrep, partner): (C (nbas, n, ispin), occ (n, ispin))."""
    cols, oc = [], []
    for i, Ui in enumerate(ad.U):
        for M in Ui:
            cols.append(np.einsum("af,fks->aks", M, Cs[i]))
            oc.append(occs[i] / ad.partners[i])
    return np.concatenate(cols, axis=1), np.concatenate(oc, axis=0)


def project(ad, V, ispin=1):
    """Packed symmetry-adapted matrix from full C1 matrices V[s] (nbas x nbas):
    V_i = 1/np_i sum_p U_ip^T V U_ip, the irreps' triangles in order per spin."""
    out = np.zeros(ad.xc_length(ispin))
    for s in range(ispin):
        c = s
        for i, Ui in enumerate(ad.U):
            Vi = sum(M.T @ V[s] @ M for M in Ui) / ad.partners[i]
            for j in range(int(ad.dims[i])):
                for k in range(j + 1):
                    out[c] = Vi[k, j]
                    c += ispin
    return out
