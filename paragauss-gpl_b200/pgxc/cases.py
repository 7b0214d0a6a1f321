"""Seeded synthetic inputs for the XC-build workloads.

Each case holds what ParaGauss hands to the XC build: atoms (bohr), the
orbital basis in unique_atom_basis_type form, the atomic grid and the
occupied orbitals (eigvec_occ, occ_num_occ).  No reference data is used;
geometries, exponents and coefficients are drawn from fixed seeds.

Conventions taken from the reference:
  * bohr = 0.52917706 Angstrom (modules/constants.f90:105-108);
  * one shell per (atom, l) holding N_exponents primitives and a
    contraction matrix (nexp, ncontr); here contractions are segmented (each
    contracted function uses its own 3-6 primitives) and N_uncontracted = 0;
  * primitive norms (2a/pi)^(3/4) (2 sqrt(a))^l / sqrt((2l-1)!!)
    (unique_atom_basis_norm_ob, modules/unique_atom_module.f90:426-444),
    contraction coefficients scaled so each contracted function has unit norm;
  * orbitals C are orthonormalised in the overlap metric S = phi^T W phi of a
    coarse quadrature of the same kind, so the integrated charge is close to,
    not exactly, sum(occ).
"""
from dataclasses import dataclass, field

import numpy as np

from . import grid as G

BOHR = 0.52917706          # Angstrom per bohr, modules/constants.f90:105
ANGSTROM = 1.0 / BOHR

Z_OF = {"H": 1, "C": 6, "N": 7, "O": 8}
# contracted functions per l for each element
SHELLS_DEFAULT = {"H": (2, 1), "C": (4, 3, 1), "N": (4, 3, 1), "O": (4, 3, 1)}
SHELLS_F = {"H": (2, 1), "C": (2, 1, 1, 1), "N": (2, 1, 1, 1), "O": (2, 1, 1, 1)}


@dataclass
class Case:
    name: str
    coords: np.ndarray
    Z: np.ndarray
    shell_atom: np.ndarray
    shell_l: np.ndarray
    shell_nexp: np.ndarray
    shell_nunc: np.ndarray
    shell_ncontr: np.ndarray
    exponents: np.ndarray
    norms: np.ndarray
    contractions: np.ndarray
    nbas: int
    grid_xyz: np.ndarray
    grid_wraw: np.ndarray
    point_atom: np.ndarray
    functional: str
    nocc: int
    ispin: int = 1
    C: np.ndarray = None        # (nbas, nocc, ispin) Fortran order
    occ: np.ndarray = None      # (nocc, ispin) Fortran order
    grid_w: np.ndarray = None   # Becke-weighted grid weights, when known
    sa_coef: np.ndarray = None
    sa_lmax: int = -1
    meta: dict = field(default_factory=dict)

    @property
    def npts(self):
        return len(self.grid_wraw)

    @property
    def xc_length(self):
        return self.ispin * self.nbas * (self.nbas + 1) // 2

    def density_matrix(self):
        """P_s = C_s diag(occ_s) C_s^T, (ispin, nbas, nbas)."""
        return np.stack([(self.C[:, :, s] * self.occ[:, s]) @ self.C[:, :, s].T
                         for s in range(self.ispin)])

    def c_fortran(self):
        return np.ascontiguousarray(self.C.transpose(2, 1, 0)).reshape(-1)

    def occ_fortran(self):
        return np.ascontiguousarray(self.occ.T).reshape(-1)

    def grdpts(self, weighted=True):
        w = self.grid_w if weighted else self.grid_wraw
        return np.ascontiguousarray(
            np.concatenate([self.grid_xyz[:, 0], self.grid_xyz[:, 1], self.grid_xyz[:, 2], w]))


def dfac(l):
    r = 1.0
    for k in range(1, 2 * l, 2):
        r *= k
    return r


def primitive_norm(l, a):
    return (2 * a / np.pi) ** 0.75 * (2 * np.sqrt(a)) ** l / np.sqrt(dfac(l))


def same_centre_overlap(l, a, b):
    """<g_a|g_b> of two normalised primitives of equal l on one centre."""
    return (2 * np.sqrt(a * b) / (a + b)) ** (l + 1.5)


def make_basis(elements, rng, exp_range, shells_table, prims=(3, 6)):
    lo, hi = np.log(exp_range[0]), np.log(exp_range[1])
    sa, sl, sne, snu, snc = [], [], [], [], []
    exps, norms, contr = [], [], []
    nbas = 0
    for a, el in enumerate(elements):
        for l, ncon in enumerate(shells_table[el]):
            if ncon == 0:
                continue
            blocks = []
            for _ in range(ncon):
                k = int(rng.integers(prims[0], prims[1] + 1))
                e = np.sort(np.exp(rng.uniform(lo, hi, size=k)))[::-1]
                c = rng.normal(size=k)
                S = same_centre_overlap(l, e[:, None], e[None, :])
                c = c / np.sqrt(c @ S @ c)
                blocks.append((e, c))
            nexp = sum(len(e) for e, _ in blocks)
            M = np.zeros((nexp, ncon))
            ee = np.zeros(nexp)
            o = 0
            for j, (e, c) in enumerate(blocks):
                ee[o:o + len(e)] = e
                M[o:o + len(e), j] = c
                o += len(e)
            sa.append(a); sl.append(l); sne.append(nexp); snu.append(0); snc.append(ncon)
            exps.append(ee)
            norms.append(primitive_norm(l, ee))
            contr.append(M.reshape(-1, order="F"))
            nbas += (2 * l + 1) * ncon
    i32 = lambda x: np.asarray(x, dtype=np.int32)
    return dict(shell_atom=i32(sa), shell_l=i32(sl), shell_nexp=i32(sne), shell_nunc=i32(snu),
                shell_ncontr=i32(snc), exponents=np.concatenate(exps), norms=np.concatenate(norms),
                contractions=np.concatenate(contr), nbas=nbas)


# ---------------------------------------------------------------------------
# numpy basis values (coarse overlap for orthonormalising the orbitals only)
# ---------------------------------------------------------------------------
def _solid_harmonics(x, y, z, lmax):
    r2 = x * x + y * y + z * z
    Y = [[np.ones_like(x)]]
    if lmax >= 1:
        Y.append([z, x, y])
    for l in range(2, lmax + 1):
        p1, p2 = Y[l - 1], Y[l - 2]
        cur = [None] * (2 * l + 1)
        cur[0] = ((2 * l - 1) * z * p1[0] - (l - 1) * r2 * p2[0]) / l
        for im in range(1, l - 1):
            rlm = 1 / np.sqrt(l * l - im * im)
            rl1m = np.sqrt((l - 1) ** 2 - im * im)
            a = (2 * l - 1) * z * rlm
            b = rl1m * r2 * rlm
            for mm in (2 * im - 1, 2 * im):
                cur[mm] = a * p1[mm] - b * p2[mm]
        im = l - 1
        a = (2 * l - 1) * z / np.sqrt(l * l - im * im)
        for mm in (2 * im - 1, 2 * im):
            cur[mm] = a * p1[mm]
        rll = np.sqrt((2 * l - 1) / (2 * l))
        q2, q1 = p1[2 * l - 3], p1[2 * l - 2]
        cur[2 * l - 1] = (x * q2 - y * q1) * rll
        cur[2 * l] = (y * q2 + x * q1) * rll
        Y.append(cur)
    return Y, r2


def basis_values(case, xyz):
    phi = np.zeros((len(xyz), case.nbas))
    eo = co = f = 0
    for s in range(len(case.shell_l)):
        a, l = case.shell_atom[s], case.shell_l[s]
        ne, nc = case.shell_nexp[s], case.shell_ncontr[s]
        e = case.exponents[eo:eo + ne]
        nrm = case.norms[eo:eo + ne]
        M = case.contractions[co:co + ne * nc].reshape(ne, nc, order="F")
        eo += ne
        co += ne * nc
        d = xyz - case.coords[a]
        Y, r2 = _solid_harmonics(d[:, 0], d[:, 1], d[:, 2], l)
        ar2 = r2[:, None] * e[None, :]
        prim = np.where(ar2 < 50.0, nrm[None, :] * np.exp(-np.minimum(ar2, 50.0)), 0.0)
        R = prim @ M
        for m in range(2 * l + 1):
            phi[:, f:f + nc] = Y[l][m][:, None] * R
            f += nc
    return phi


def orthonormal_orbitals(case, rng, nocc, coarse=(20, 50)):
    xyz, w, owner = G.atomic_grids(case.coords, case.Z, coarse[0], coarse[1])
    w = w * G.becke_weights_numpy(case.coords, xyz, owner)
    S = np.zeros((case.nbas, case.nbas))
    for lo in range(0, len(w), 20000):
        ph = basis_values(case, xyz[lo:lo + 20000])
        S += ph.T @ (ph * w[lo:lo + 20000, None])
    C = rng.normal(size=(case.nbas, nocc))
    M = C.T @ S @ C
    L = np.linalg.cholesky(M)
    C = np.linalg.solve(L, C.T).T   # C L^{-T}
    return C


# ---------------------------------------------------------------------------
# geometries
# ---------------------------------------------------------------------------
def water():
    els = ["O", "H", "H"]
    xyz = np.array([[0.0, 0.0, 0.0], [0.757, 0.586, 0.0], [-0.757, 0.586, 0.0]]) * ANGSTROM
    return els, xyz


def random_cluster(rng, counts, box_ang, dmin_ang):
    els = []
    for el, n in counts:
        els += [el] * n
    els = list(np.array(els)[rng.permutation(len(els))])
    pts = []
    while len(pts) < len(els):
        p = rng.uniform(0, box_ang, size=3)
        if all(np.linalg.norm(p - q) >= dmin_ang for q in pts):
            pts.append(p)
    return els, np.array(pts) * ANGSTROM


def build_case(name, els, xyz, *, seed, exp_range, nrad, nang, functional, nocc, shells=None,
               ispin=1, orthonormalise=True):
    rng = np.random.default_rng(seed)
    shells = shells or SHELLS_DEFAULT
    b = make_basis(els, rng, exp_range, shells)
    Z = np.array([Z_OF[e] for e in els], dtype=np.int32)
    gx, gw, owner = G.atomic_grids(xyz, Z, nrad, nang)
    case = Case(name=name, coords=np.asarray(xyz, dtype=np.float64), Z=Z, grid_xyz=gx, grid_wraw=gw,
                point_atom=owner, functional=functional, nocc=nocc, ispin=ispin, **b)
    case.meta = dict(seed=seed, nrad=nrad, nang=nang, exp_range=exp_range, elements=list(els))
    if orthonormalise:
        C = orthonormal_orbitals(case, rng, nocc)
    else:
        C = rng.normal(size=(case.nbas, nocc)) / np.sqrt(case.nbas)
    if ispin == 1:
        case.C = C[:, :, None]
        case.occ = np.full((nocc, 1), 2.0)
    else:
        C2 = orthonormal_orbitals(case, rng, nocc) if orthonormalise else C
        case.C = np.stack([C, C2], axis=2)
        occ_b = np.ones(nocc)
        occ_b[nocc // 2:] = 0.0
        case.occ = np.stack([np.ones(nocc), occ_b], axis=1)
    return case


def molecule_set(n=256, seed=1004, functional=None, atoms=(3, 40)):
    """The batched workload: n seeded molecules of 3-40 C/H/O atoms (sizes drawn
    uniform; 40% C, 40% H, 20% O), each in a cube holding the 60-atom cluster's
    atom density, with the default basis (20-400 functions), 50-75 radial x
    194- or 302-class angular points per atom, and nocc = half the electron
    count.  The functional alternates VWN / PBE unless one is given; atoms is
    the inclusive range of molecule sizes.  C is
    scaled normal noise (not orthonormalised) to keep the set cheap to make."""
    rng = np.random.default_rng(seed)
    out = []
    for m in range(n):
        nat = int(rng.integers(atoms[0], atoms[1] + 1))
        kinds = rng.choice(["C", "H", "O"], size=nat, p=[0.4, 0.4, 0.2])
        counts = [(el, int(np.sum(kinds == el))) for el in ("C", "H", "O")]
        box = max(2.5, (nat / 0.035) ** (1.0 / 3.0))
        els, xyz = random_cluster(rng, counts, box, 1.0)
        nrad = int(rng.integers(50, 76))
        nang = 194 if rng.random() < 0.5 else 302
        xc = functional or ("VWN" if m % 2 == 0 else "PBE")
        nocc = max(1, sum(Z_OF[e] for e in els) // 2)
        out.append(build_case(f"mol{m}-{xc}", els, xyz, seed=seed * 1000 + m, exp_range=(0.1, 5e3), nrad=nrad,
                              nang=nang, functional=xc, nocc=nocc, orthonormalise=False))
    return out


def config(n, **kw):
    """The seeded workloads: 1 water VWN, 2 60-atom C/H PBE, 5 500-atom PBE."""
    if n == 1:
        els, xyz = water()
        return build_case("water-VWN", els, xyz, seed=1001, exp_range=(0.1, 5e3), nrad=50, nang=194,
                          functional="VWN", nocc=5, **kw)
    if n in (2, 3):
        rng = np.random.default_rng(1002)
        els, xyz = random_cluster(rng, [("C", 30), ("H", 30)], 12.0, 1.1)
        return build_case("CH60-PBE", els, xyz, seed=1002, exp_range=(0.05, 1e4), nrad=75, nang=302,
                          functional="PBE", nocc=210, **kw)
    if n == 5:
        # orthonormalising 1,700 orbitals of 5,800 functions against a quadrature
        # overlap needs tens of GB on the host: C is scaled normal noise instead
        kw.setdefault("orthonormalise", False)
        rng = np.random.default_rng(1005)
        els, xyz = random_cluster(rng, [("C", 150), ("H", 225), ("O", 75), ("N", 50)], 28.0, 1.0)
        return build_case("CHON500-PBE", els, xyz, seed=1005, exp_range=(0.05, 1e4), nrad=75, nang=302,
                          functional="PBE", nocc=1700, shells=SHELLS_F, **kw)
    raise ValueError(n)


def small_case(functional="PBE", seed=7, natoms=4, nrad=20, nang=50, nocc=6, ispin=1, lmax=2,
               exp_range=(0.1, 200.0)):
    """A few-atom case the oracle finishes in well under a second."""
    rng = np.random.default_rng(seed)
    els, xyz = random_cluster(rng, [("O", 1), ("C", max(natoms - 3, 0)), ("H", 2)], 3.5, 1.0)
    els, xyz = els[:natoms], xyz[:natoms]
    shells = {k: tuple(v[:lmax + 1]) for k, v in (SHELLS_F if lmax == 3 else SHELLS_DEFAULT).items()}
    if lmax == 3:
        shells = {"H": (2, 1), "C": (2, 2, 1, 1), "N": (2, 2, 1, 1), "O": (2, 2, 1, 1)}
    return build_case(f"small-{functional}-{seed}", els, xyz, seed=seed, exp_range=exp_range, nrad=nrad,
                      nang=nang, functional=functional, nocc=nocc, shells=shells, ispin=ispin)
