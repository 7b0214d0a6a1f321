"""ctypes mirrors of the plain-data structs in include/pgxc.h.

The same layouts describe a case to libpgxc (the product) and, in the tests,
to the CPU oracle, so one marshalling routine serves both.
"""
import ctypes as ct

import numpy as np

PGXC_OK = 0
PGXC_EINVAL = -1
PGXC_ENOTSUP = -2
PGXC_ENOMEM = -3
PGXC_ECUDA = -4
PGXC_ETIMEOUT = -5
PGXC_ENONFINITE = -6
PGXC_ENODEV = -7

XC_VWN = 1
XC_PBE = 2
XC_REVPBE = 3
XC_PBESOL = 4
XC_BP86 = 5
XC_PW91 = 6
XC_BPW91 = 7
XC_BLYP = 8
XC_XALPHA = 9
XC_B88 = 10
XC_PBEN = 11
XC_VMT = 12
XC_VT84 = 13
XC_VMTSOL = 14
XC_VT84SOL = 15
XC_HCTH = 16
XC_HCTH120 = 17
XC_HCTH147 = 18
XC_HCTH407 = 19
XC_NRECMV92 = 20
XC_PWLDA = 21
XC_B3LYP = 22
XC_PBE0 = 23
XC_LB94 = 24
XC_RVWN = 25
XC_RBP = 26
XC_ECMV92 = 27
XC_RPW91 = 28
XC_RVWN_ENGEL = 29
XC_TPSS = 30
XC_M06L = 31
XC_M06 = 32
XC_VSXC = 33
XC_IDS = {"VWN": XC_VWN, "PBE": XC_PBE, "revPBE": XC_REVPBE, "PBEsol": XC_PBESOL, "BP86": XC_BP86,
          "PW91": XC_PW91, "BPW91": XC_BPW91, "BLYP": XC_BLYP, "XALPHA": XC_XALPHA, "B88": XC_B88,
          "PBEN": XC_PBEN, "VMT": XC_VMT, "VT84": XC_VT84, "VMTsol": XC_VMTSOL, "VT84sol": XC_VT84SOL,
          "HCTH": XC_HCTH, "HCTH120": XC_HCTH120, "HCTH147": XC_HCTH147, "HCTH407": XC_HCTH407,
          "NRECMV92": XC_NRECMV92, "PWLDA": XC_PWLDA, "B3LYP": XC_B3LYP, "PBE0": XC_PBE0,
          "LB94": XC_LB94, "RVWN": XC_RVWN, "RBP": XC_RBP, "ECMV92": XC_ECMV92,
          "RPW91": XC_RPW91, "RVWN_ENGEL": XC_RVWN_ENGEL, "TPSS": XC_TPSS,
          "M06L": XC_M06L, "M06": XC_M06, "VSXC": XC_VSXC}
LDA_XC = ("VWN", "XALPHA", "PWLDA", "RVWN", "RVWN_ENGEL")
MGGA_XC = ("TPSS", "M06L", "M06", "VSXC")
# the keywords without tau (the point-functional API and every layout)
GGA_LDA_XC = tuple(k for k in XC_IDS if k not in MGGA_XC)


def is_gga(xc):
    """True for the GGA keywords (PGXC_XC_IS_GGA)."""
    return xc not in LDA_XC

PREC_FP64 = 0
PREC_MIXED_INT8 = 1
PREC_IDS = {"fp64": PREC_FP64, "mixed": PREC_MIXED_INT8}

_i32p = ct.POINTER(ct.c_int32)
_f64p = ct.POINTER(ct.c_double)


class Geometry(ct.Structure):
    _fields_ = [("natoms", ct.c_int32), ("coords", _f64p)]


class Basis(ct.Structure):
    _fields_ = [
        ("nshells", ct.c_int32),
        ("shell_atom", _i32p),
        ("shell_l", _i32p),
        ("shell_nexp", _i32p),
        ("shell_nunc", _i32p),
        ("shell_ncontr", _i32p),
        ("exponents", _f64p),
        ("norms", _f64p),
        ("contractions", _f64p),
        ("sa_coef", _f64p),
        ("sa_lmax", ct.c_int32),
    ]


class Grid(ct.Structure):
    _fields_ = [
        ("npts", ct.c_int64),
        ("grdpts", _f64p),
        ("weights_are_raw", ct.c_int32),
        ("point_atom", _i32p),
    ]


class GridSpec(ct.Structure):
    _fields_ = [
        ("nrad", _i32p),
        ("radius", _f64p),
        ("nang", ct.c_int32),
    ]


class MarshalledSpec:
    """pgxc_grid_spec of a case built on an atomic grid: its nrad, nang and the
    Pople radius of each element (pgxc/grid.py)."""

    def __init__(self, case):
        from . import grid as G
        self.nrad = np.full(len(case.coords), int(case.meta["nrad"]), dtype=np.int32)
        self.radius = np.array([G.POPLE_RADIUS[int(z)] for z in case.Z], dtype=np.float64)
        self.spec = GridSpec(i32p(self.nrad), f64p(self.radius), int(case.meta["nang"]))


class Options(ct.Structure):
    _fields_ = [
        ("functional", ct.c_int32),
        ("ispin", ct.c_int32),
        ("precision", ct.c_int32),
        ("batch_points", ct.c_int32),
        ("screen_threshold", ct.c_double),
        ("device", ct.c_int32),
        ("keep_orbitals", ct.c_int32),
        ("max_chunk_points", ct.c_int64),
    ]


class Symmetry(ct.Structure):
    _fields_ = [
        ("n_irrep", ct.c_int32),
        ("dims", _i32p),
        ("partners", _i32p),
        ("nnz", ct.c_int64),
        ("irrep", _i32p),
        ("partner", _i32p),
        ("fn", _i32p),
        ("ao", _i32p),
        ("coef", _f64p),
    ]


class MarshalledSymmetry:
    """pgxc_symmetry over an adaptation (pgxc.symmetry.Adaptation); keeps the arrays alive."""

    def __init__(self, ad):
        self.dims = np.ascontiguousarray(ad.dims, dtype=np.int32)
        self.partners = np.ascontiguousarray(ad.partners, dtype=np.int32)
        self.e = ad.entries()
        self.s = Symmetry(len(self.dims), i32p(self.dims), i32p(self.partners), len(self.e[0]), i32p(self.e[0]),
                          i32p(self.e[1]), i32p(self.e[2]), i32p(self.e[3]), f64p(self.e[4]))


class IrrepOrbitals:
    """Per-irrep C (dims, nocc, ispin) and occ (nocc, ispin) as the Fortran
    arrays, with the pointer arrays of pgxc_build_sym."""

    def __init__(self, Cs, occs):
        self.C = [np.ascontiguousarray(np.asarray(C, dtype=np.float64).transpose(2, 1, 0)).reshape(-1) for C in Cs]
        self.occ = [np.ascontiguousarray(np.asarray(o, dtype=np.float64).T).reshape(-1) for o in occs]
        self.nocc = np.array([np.asarray(o).shape[0] for o in occs], dtype=np.int32)
        n = len(Cs)
        self.pC = (_f64p * n)(*[f64p(c) for c in self.C])
        self.pocc = (_f64p * n)(*[f64p(o) for o in self.occ])


class Timings(ct.Structure):
    _fields_ = [
        ("h2d_ms", ct.c_double),
        ("basis_ms", ct.c_double),
        ("density_ms", ct.c_double),
        ("functional_ms", ct.c_double),
        ("potential_ms", ct.c_double),
        ("d2h_ms", ct.c_double),
        ("total_ms", ct.c_double),
        ("xgemm_ms", ct.c_double),
        ("vgemm_ms", ct.c_double),
        ("kernel_launches", ct.c_int64),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


def f64p(a):
    """Pointer to a C-contiguous float64 array (or NULL for None)."""
    if a is None:
        return ct.cast(None, _f64p)
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_f64p)


def i32p(a):
    if a is None:
        return ct.cast(None, _i32p)
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_i32p)


class Marshalled:
    """Keeps the numpy buffers alive while the C structs point into them."""

    def __init__(self, case, weighted=True):
        self._keep = []
        c = case
        coords = np.ascontiguousarray(c.coords, dtype=np.float64).reshape(-1)
        self._keep.append(coords)
        self.geometry = Geometry(len(c.coords), f64p(coords))
        arrs = [np.ascontiguousarray(a, dtype=np.int32) for a in
                (c.shell_atom, c.shell_l, c.shell_nexp, c.shell_nunc, c.shell_ncontr)]
        flt = [np.ascontiguousarray(a, dtype=np.float64) for a in
               (c.exponents, c.norms, c.contractions)]
        sa = None if c.sa_coef is None else np.ascontiguousarray(c.sa_coef, dtype=np.float64)
        self._keep += arrs + flt + [sa]
        self.basis = Basis(len(c.shell_l), *[i32p(a) for a in arrs], *[f64p(a) for a in flt],
                           f64p(sa), int(c.sa_lmax))
        w = c.grid_w if (weighted and c.grid_w is not None) else c.grid_wraw
        grd = np.concatenate([c.grid_xyz[:, 0], c.grid_xyz[:, 1], c.grid_xyz[:, 2], w])
        grd = np.ascontiguousarray(grd, dtype=np.float64)
        pa = np.ascontiguousarray(c.point_atom, dtype=np.int32)
        self._keep += [grd, pa]
        raw = 0 if (weighted and c.grid_w is not None) else 1
        self.grid = Grid(len(w), f64p(grd), raw, i32p(pa))
        self.weights_are_raw = raw
