"""ctypes binding of the FP64 CPU oracle (liboracle.so) -- TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module; the product (libpgxc) never does.
"""
import ctypes as ct
import glob
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "paragauss-gpl_b200"))
from pgxc import abi  # noqa: E402

_LIB = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _openblas_path():
    libs = os.path.join(os.path.dirname(np.__file__), os.pardir, "numpy.libs")
    hits = sorted(glob.glob(os.path.join(libs, "libscipy_openblas64_*.so")))
    return os.path.abspath(hits[0]) if hits else None


def lib():
    global _LIB
    if _LIB is not None:
        return _LIB
    path = os.path.join(HERE, "liboracle.so")
    if not os.path.exists(path):
        build()
    L = ct.CDLL(path)
    P = ct.POINTER
    L.oracle_set_blas.argtypes = [ct.c_char_p]
    L.oracle_max_threads.restype = ct.c_int
    L.oracle_nbas.argtypes = [P(abi.Geometry), P(abi.Basis)]
    L.oracle_nbas.restype = ct.c_int64
    L.oracle_orbitals.argtypes = [P(abi.Geometry), P(abi.Basis), ct.c_int64, abi._f64p, abi._f64p, abi._f64p]
    L.oracle_functionals.argtypes = [ct.c_int32, ct.c_int32, ct.c_int64, abi._f64p, abi._f64p, abi._f64p,
                                     abi._f64p, abi._f64p]
    L.oracle_functionals_mgga.argtypes = [ct.c_int32, ct.c_int32, ct.c_int64, abi._f64p, abi._f64p, abi._f64p,
                                          abi._f64p, abi._f64p, abi._f64p, abi._f64p]
    L.oracle_becke.argtypes = [P(abi.Geometry), ct.c_int64, abi._f64p, abi._i32p, abi._f64p, ct.c_int32]
    L.oracle_xc_build.argtypes = [P(abi.Geometry), P(abi.Basis), P(abi.Grid), ct.c_int32, ct.c_int32,
                                  abi._f64p, abi._f64p, ct.c_int32, ct.c_int32, abi._f64p, ct.c_int64,
                                  abi._f64p, abi._f64p, ct.c_int32, ct.c_int32, ct.c_int64, ct.c_int64]
    L.oracle_xc_build_sym.argtypes = [P(abi.Geometry), P(abi.Basis), P(abi.Grid), ct.c_int32, ct.c_int32,
                                      P(abi.Symmetry), P(abi._f64p), P(abi._f64p), abi._i32p, abi._f64p, ct.c_int64,
                                      P(ct.c_double), P(ct.c_double), ct.c_int32]
    L.oracle_xc_gradient.argtypes = [P(abi.Geometry), P(abi.Basis), P(abi.Grid), ct.c_int32, ct.c_int32,
                                     abi._f64p, abi._f64p, ct.c_int32, ct.c_int32, abi._f64p, P(ct.c_double)]
    L.oracle_overlap.argtypes = [P(abi.Geometry), P(abi.Basis), P(abi.Grid), abi._f64p, ct.c_int32]
    blas = _openblas_path()
    if blas:
        L.oracle_set_blas(blas.encode())
    _LIB = L
    return L


def max_threads():
    return lib().oracle_max_threads()


def orbitals(case, pts, grads=True):
    m = abi.Marshalled(case)
    pts = np.ascontiguousarray(np.asarray(pts, dtype=np.float64).T).reshape(-1)
    n = len(pts) // 3
    phi = np.zeros(n * case.nbas)
    gr = np.zeros(n * 3 * case.nbas) if grads else None
    st = lib().oracle_orbitals(ct.byref(m.geometry), ct.byref(m.basis), n, abi.f64p(pts), abi.f64p(phi),
                               abi.f64p(gr))
    assert st == 0, st
    phi = phi.reshape(case.nbas, n).T
    if grads:
        gr = gr.reshape(case.nbas, 3, n).transpose(2, 1, 0)
    return phi, gr


def functionals(xc, ispin, rho, gam=None):
    """rho (n, ispin), gam (n, 2ispin-1) -> f (n), fr (n, ispin), fg (n, 2ispin-1)."""
    xcid = abi.XC_IDS[xc] if isinstance(xc, str) else xc
    rho = np.asarray(rho, dtype=np.float64).reshape(len(rho), -1)
    n = rho.shape[0]
    ng = 2 * ispin - 1
    r = np.ascontiguousarray(rho.T).reshape(-1)
    g = np.ascontiguousarray(np.asarray(gam, dtype=np.float64).reshape(n, -1).T).reshape(-1) if gam is not None \
        else np.zeros(n * ng)
    f = np.zeros(n)
    fr = np.zeros(n * ispin)
    fg = np.zeros(n * ng)
    st = lib().oracle_functionals(xcid, ispin, n, abi.f64p(r), abi.f64p(g), abi.f64p(f), abi.f64p(fr),
                                  abi.f64p(fg))
    assert st == 0, st
    return f, fr.reshape(ispin, n).T, fg.reshape(ng, n).T


def functionals_mgga(xc, ispin, rho, gam, tau):
    """A meta-GGA: rho (n, ispin), gam (n, 2ispin-1), tau (n, ispin) ->
    f (n), fr (n, ispin), fg (n, 2ispin-1), ft (n, ispin)."""
    xcid = abi.XC_IDS[xc] if isinstance(xc, str) else xc
    rho = np.asarray(rho, dtype=np.float64).reshape(len(rho), -1)
    n = rho.shape[0]
    ng = 2 * ispin - 1
    col = lambda a, k: np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(n, k).T).reshape(-1)
    r, g, t = col(rho, ispin), col(gam, ng), col(tau, ispin)
    f, fr, fg, ft = np.zeros(n), np.zeros(n * ispin), np.zeros(n * ng), np.zeros(n * ispin)
    st = lib().oracle_functionals_mgga(xcid, ispin, n, abi.f64p(r), abi.f64p(g), abi.f64p(t), abi.f64p(f),
                                       abi.f64p(fr), abi.f64p(fg), abi.f64p(ft))
    assert st == 0, st
    return f, fr.reshape(ispin, n).T, fg.reshape(ng, n).T, ft.reshape(ispin, n).T


def becke(case, nthreads=0):
    m = abi.Marshalled(case, weighted=False)
    pts = np.ascontiguousarray(case.grid_xyz.T).reshape(-1)
    w = np.zeros(case.npts)
    st = lib().oracle_becke(ct.byref(m.geometry), case.npts, abi.f64p(pts), abi.i32p(m._keep[-1]), abi.f64p(w),
                            nthreads)
    assert st == 0, st
    return w


def weight_case(case, nthreads=0):
    """Fill case.grid_w = raw weight * Becke partition weight (mkgrid :3135)."""
    case.grid_w = case.grid_wraw * becke(case, nthreads)
    return case


def xc_build(case, vla=128, nthreads=0, pt_range=None):
    """Returns (ham_xc_arr, exc, nel) of one build on the weighted grid."""
    assert case.grid_w is not None
    m = abi.Marshalled(case)
    C = case.c_fortran()
    occ = case.occ_fortran()
    ham = np.zeros(case.xc_length)
    exc = ct.c_double(0.0)
    nel = ct.c_double(0.0)
    lo, hi = pt_range if pt_range else (0, case.npts)
    st = lib().oracle_xc_build(ct.byref(m.geometry), ct.byref(m.basis), ct.byref(m.grid),
                               abi.XC_IDS[case.functional], case.ispin, abi.f64p(C), abi.f64p(occ), case.nbas,
                               case.nocc, abi.f64p(ham), case.xc_length, ct.byref(exc), ct.byref(nel), vla,
                               nthreads, lo, hi)
    assert st == 0, st
    return ham, exc.value, nel.value


def xc_build_sym(case, ad, Cs, occs, nthreads=0):
    """Symmetry-adapted build (pgxc.symmetry.Adaptation, per-irrep C and occ);
    returns (ham_xc_arr, exc, nel)."""
    assert case.grid_w is not None
    m = abi.Marshalled(case)
    sy = abi.MarshalledSymmetry(ad)
    o = abi.IrrepOrbitals(Cs, occs)
    ham = np.zeros(ad.xc_length(case.ispin))
    exc = ct.c_double(0.0)
    nel = ct.c_double(0.0)
    st = lib().oracle_xc_build_sym(ct.byref(m.geometry), ct.byref(m.basis), ct.byref(m.grid),
                                   abi.XC_IDS[case.functional], case.ispin, ct.byref(sy.s), o.pC, o.pocc,
                                   abi.i32p(o.nocc), abi.f64p(ham), len(ham), ct.byref(exc), ct.byref(nel), nthreads)
    assert st == 0, st
    return ham, exc.value, nel.value


def xc_gradient(case):
    """dE_xc/dR (natoms, 3) on the raw grid moving with its atoms, and E_xc."""
    m = abi.Marshalled(case, weighted=False)
    g = np.zeros(3 * len(case.coords))
    e = ct.c_double(0.0)
    st = lib().oracle_xc_gradient(ct.byref(m.geometry), ct.byref(m.basis), ct.byref(m.grid),
                                  abi.XC_IDS[case.functional], case.ispin, abi.f64p(case.c_fortran()),
                                  abi.f64p(case.occ_fortran()), case.nbas, case.nocc, abi.f64p(g), ct.byref(e))
    assert st == 0, st
    return g.reshape(-1, 3), e.value


def overlap(case, nthreads=0):
    m = abi.Marshalled(case)
    S = np.zeros(case.nbas * case.nbas)
    st = lib().oracle_overlap(ct.byref(m.geometry), ct.byref(m.basis), ct.byref(m.grid), abi.f64p(S), nthreads)
    assert st == 0, st
    return S.reshape(case.nbas, case.nbas)


def unpack(ham, nbas, ispin=1, s=0):
    """Packed (j outer, k<=j inner, spin stride ispin) -> full symmetric matrix."""
    jj = np.repeat(np.arange(nbas), np.arange(1, nbas + 1))
    kk = np.concatenate([np.arange(j + 1) for j in range(nbas)])
    vals = ham[s::ispin][: len(jj)]
    V = np.zeros((nbas, nbas))
    V[kk, jj] = vals
    V[jj, kk] = vals
    return V


def pseudo2d_sym(ham, ispin, dims, nblocks, first, half):
    """xc_pseudo2d_sym (modules/xc_hamiltonian.f90:2637-2779) on a copy of the
    packed matrix of pgxc_build_sym's layout, with the reference's own 1-based
    packed positions and loop order.  Block b of irrep i: first function
    first[b] (0-based within the irrep: orbitalprojection_ob - ob - 1), the
    half size half[b] = n_exp * n_independent / 2.  Pure Python: small cases."""
    h = np.array(ham, dtype=np.float64, copy=True)
    offset = 0  # 0-based start of the irrep's packed block (times ispin)
    b0 = 0
    for i, dim in enumerate(dims):
        nb = int(nblocks[i])
        blk = [(int(first[b0 + b]) + 1, int(half[b0 + b])) for b in range(nb)]  # 1-based first function
        for x in range(nb):
            px, m1 = blk[x]
            for y in range(x + 1):
                py, m2 = blk[y]
                if x == y:
                    for s in range(ispin):
                        # diagonal blocks: A x A and B x B (:2686-2704)
                        c1 = (px * (px - 1)) // 2 + py
                        c2 = m2 + py + ((px + m1) * (px + m1 - 1)) // 2
                        stride = px * ispin - ispin
                        c1 = (c1 - 1) * ispin + s + 1 + offset
                        c2 = (c2 - 1) * ispin + s + 1 + offset
                        for im1 in range(1, m1 + 1):
                            for im2 in range(1, im1 + 1):
                                h[c1 - 1] = 0.5 * (h[c1 - 1] + h[c2 - 1])
                                h[c2 - 1] = h[c1 - 1]
                                c1 += ispin
                                c2 += ispin
                            c1 += stride
                            c2 += stride + m1 * ispin
                        # off diagonals: B x A (:2706-2721)
                        for i1 in range(1, m1 + 1):
                            c4 = ((px + m1 + i1 - 1) * (px + m1 + i1 - 2)) // 2 + py + i1 - 1
                            c4 = (c4 - 1) * ispin + s + 1 + offset
                            c3 = c4
                            st = (px + m1 + i1 - 1) * ispin
                            for i2 in range(i1, m1 + 1):
                                h[c4 - 1] = 0.5 * (h[c4 - 1] - h[c3 - 1])
                                h[c3 - 1] = -h[c4 - 1]
                                c4 += ispin
                                c3 += st
                                st += ispin
                else:
                    for s in range(ispin):
                        stride = (px - m2 + 1) * ispin - ispin
                        c1 = ((px * (px - 1)) // 2) + py
                        c2 = m2 + py + ((px + m1) * (px + m1 - 1)) // 2
                        c3 = ((px * (px - 1)) // 2) + py + m2
                        c4 = py + ((px + m1) * (px + m1 - 1)) // 2
                        c1 = (c1 - 1) * ispin + s + 1 + offset
                        c2 = (c2 - 1) * ispin + s + 1 + offset
                        c3 = (c3 - 1) * ispin + s + 1 + offset
                        c4 = (c4 - 1) * ispin + s + 1 + offset
                        for _ in range(m1):
                            for _ in range(m2):
                                h[c1 - 1] = 0.5 * (h[c1 - 1] + h[c2 - 1])
                                h[c2 - 1] = h[c1 - 1]
                                h[c3 - 1] = 0.5 * (h[c3 - 1] - h[c4 - 1])
                                h[c4 - 1] = -h[c3 - 1]
                                c1 += ispin
                                c2 += ispin
                                c3 += ispin
                                c4 += ispin
                            c1 += stride
                            c2 += stride + m1 * ispin
                            c3 += stride
                            c4 += stride + m1 * ispin
                            stride += ispin
        offset += dim * (dim + 1) // 2 * ispin
        b0 += nb
    return h
