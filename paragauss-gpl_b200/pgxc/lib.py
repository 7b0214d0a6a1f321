"""ctypes binding of libpgxc.so (the product).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""
import ctypes as ct
import os

import numpy as np

from . import abi

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG, "libpgxc.so")
_LIB = None


class PgxcError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"pgxc status {status}: {msg}")
        self.status = status


def lib():
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with __graft_entry__.build() "
                          "(nvcc, sm_100a); there is no CPU fallback")
    L = ct.CDLL(LIB_PATH)
    P = ct.POINTER
    vp = ct.c_void_p
    L.pgxc_default_options.argtypes = [P(abi.Options)]
    L.pgxc_create.argtypes = [P(abi.Geometry), P(abi.Basis), P(abi.Grid), P(abi.Options), P(vp)]
    L.pgxc_create_on_grid.argtypes = [P(abi.Geometry), P(abi.Basis), P(abi.GridSpec), P(abi.Options), P(vp)]
    L.pgxc_atomic_grid_size.argtypes = [P(abi.Geometry), P(abi.GridSpec), P(ct.c_int64)]
    L.pgxc_atomic_grid.argtypes = [P(abi.Geometry), P(abi.GridSpec), ct.c_int64, vp, vp, vp]
    L.pgxc_nbas.argtypes = [vp, P(ct.c_int32)]
    L.pgxc_screen_stats.argtypes = [vp, P(ct.c_int64), P(ct.c_int64), P(ct.c_int64), P(ct.c_double)]
    L.pgxc_build.argtypes = [vp, abi._f64p, abi._f64p, ct.c_int32, ct.c_int32, ct.c_int32, abi._f64p, ct.c_int64,
                             P(ct.c_double), P(ct.c_double), P(abi.Timings)]
    L.pgxc_build_device.argtypes = [vp, vp, vp, ct.c_int32, ct.c_int32, ct.c_int32, vp, ct.c_int64, vp,
                                    P(abi.Timings)]
    L.pgxc_build_density.argtypes = [vp, abi._f64p, ct.c_int32, ct.c_int32, abi._f64p, ct.c_int64, P(ct.c_double),
                                     P(ct.c_double), P(abi.Timings)]
    L.pgxc_grid_weights.argtypes = [vp, abi._f64p, ct.c_int64]
    L.pgxc_orbital_calculate.argtypes = [vp, ct.c_int64, abi._f64p, abi._f64p, abi._f64p]
    L.pgxc_xc_functionals_mgga.argtypes = [ct.c_int32, ct.c_int32, ct.c_int64, abi._f64p, abi._f64p, abi._f64p,
                                           abi._f64p, abi._f64p, abi._f64p, abi._f64p]
    L.pgxc_xc_functionals.argtypes = [ct.c_int32, ct.c_int32, ct.c_int64, abi._f64p, abi._f64p, abi._f64p,
                                      abi._f64p, abi._f64p]
    L.pgxc_becke_weights.argtypes = [P(abi.Geometry), ct.c_int64, abi._f64p, abi._i32p, abi._f64p]
    L.pgxc_last_error.argtypes = [vp]
    L.pgxc_last_error.restype = ct.c_char_p
    L.pgxc_strerror.argtypes = [ct.c_int]
    L.pgxc_strerror.restype = ct.c_char_p
    L.pgxc_destroy.argtypes = [vp]
    L.pgxc_batch_create.argtypes = [P(vp), ct.c_int32, P(vp), P(vp), P(ct.c_int32), P(vp), P(vp), P(vp)]
    L.pgxc_batch_create_chunked.argtypes = [P(vp), ct.c_int32, P(vp), P(vp), P(ct.c_int32), P(vp), P(vp),
                                            ct.c_int64, P(vp)]
    L.pgxc_batch_is_set.argtypes = [vp, P(ct.c_int32)]
    L.pgxc_batch_run.argtypes = [vp, P(ct.c_double)]
    L.pgxc_batch_destroy.argtypes = [vp]
    L.pgxc_batch_stats.argtypes = [vp, P(ct.c_int64), P(ct.c_int64)]
    L.pgxc_xc_gradient.argtypes = [vp, abi._f64p, abi._f64p, ct.c_int32, ct.c_int32, ct.c_int32, abi._f64p,
                                   P(ct.c_double)]
    L.pgxc_xc_energies.argtypes = [vp, abi._f64p, abi._f64p, ct.c_int32, ct.c_int32, ct.c_int32, ct.c_int32,
                                   abi._i32p, abi._f64p, P(ct.c_double)]
    L.pgxc_set_symmetry.argtypes = [vp, P(abi.Symmetry)]
    L.pgxc_set_pseudo2d.argtypes = [vp, abi._i32p, abi._i32p, abi._i32p]
    L.pgxc_sym_xc_length.argtypes = [vp, P(ct.c_int64)]
    L.pgxc_build_sym.argtypes = [vp, P(abi._f64p), P(abi._f64p), abi._i32p, ct.c_int32, abi._f64p, ct.c_int64,
                                 P(ct.c_double), P(ct.c_double), P(abi.Timings)]
    L.pgxc_xc_gradient_sym.argtypes = [vp, P(abi._f64p), P(abi._f64p), abi._i32p, ct.c_int32, abi._f64p,
                                       P(ct.c_double)]
    _LIB = L
    return L


def _check(st, ctx=None):
    if st != 0:
        msg = lib().pgxc_last_error(ctx)
        raise PgxcError(st, (msg or b"").decode())


class Context:
    """One geometry: pgxc_create ... pgxc_destroy."""

    def __init__(self, case, precision="fp64", weighted=True, device=-1, max_chunk_points=0,
                 screen_threshold=0.0, batch_points=128, keep_orbitals=False, on_grid=False):
        """on_grid: build the case's atomic grid and its Becke weights on the
        device (pgxc_create_on_grid) instead of passing the host grid."""
        L = lib()
        self.case = case
        self._m = abi.Marshalled(case, weighted=weighted)
        o = abi.Options()
        L.pgxc_default_options(ct.byref(o))
        o.functional = abi.XC_IDS[case.functional]
        o.ispin = case.ispin
        o.precision = abi.PREC_IDS[precision]
        o.device = device
        o.max_chunk_points = max_chunk_points
        o.screen_threshold = screen_threshold
        o.batch_points = batch_points
        o.keep_orbitals = int(bool(keep_orbitals))
        self.opt = o
        h = ct.c_void_p()
        if on_grid:
            self._spec = abi.MarshalledSpec(case)
            st = L.pgxc_create_on_grid(ct.byref(self._m.geometry), ct.byref(self._m.basis),
                                       ct.byref(self._spec.spec), ct.byref(o), ct.byref(h))
        else:
            st = L.pgxc_create(ct.byref(self._m.geometry), ct.byref(self._m.basis), ct.byref(self._m.grid),
                               ct.byref(o), ct.byref(h))
        _check(st)
        self.h = h
        nb = ct.c_int32()
        _check(L.pgxc_nbas(h, ct.byref(nb)), h)
        self.nbas = nb.value

    def build(self, C=None, occ=None, ham=None, timings=False):
        """Returns (ham_xc_arr, exc, nel[, timings dict]); ham is accumulated into when given."""
        c = self.case
        Cf = c.c_fortran() if C is None else np.ascontiguousarray(C, dtype=np.float64).reshape(-1)
        of = c.occ_fortran() if occ is None else np.ascontiguousarray(occ, dtype=np.float64).reshape(-1)
        if ham is None:
            ham = np.zeros(c.xc_length)
        exc = ct.c_double(0.0)
        nel = ct.c_double(0.0)
        tm = abi.Timings()
        st = lib().pgxc_build(self.h, abi.f64p(Cf), abi.f64p(of), c.nbas, c.nocc, c.ispin, abi.f64p(ham),
                              c.xc_length, ct.byref(exc), ct.byref(nel), ct.byref(tm))
        _check(st, self.h)
        if timings:
            return ham, exc.value, nel.value, tm.as_dict()
        return ham, exc.value, nel.value

    def xc_gradient(self, C=None, occ=None):
        """dE_xc/dR (natoms, 3) with the grid moving with its atoms, and E_xc
        (a context created with weighted=False: raw weights and point_atom)."""
        c = self.case
        Cf = c.c_fortran() if C is None else np.ascontiguousarray(C, dtype=np.float64).reshape(-1)
        of = c.occ_fortran() if occ is None else np.ascontiguousarray(occ, dtype=np.float64).reshape(-1)
        g = np.zeros(3 * len(c.coords))
        e = ct.c_double(0.0)
        _check(lib().pgxc_xc_gradient(self.h, abi.f64p(Cf), abi.f64p(of), c.nbas, c.nocc, c.ispin, abi.f64p(g),
                                      ct.byref(e)), self.h)
        return g.reshape(-1, 3), e.value

    def xc_energies(self, functionals, C=None, occ=None):
        """E_xc of each keyword in functionals on this context's density
        (post-SCF energies); returns (list of E_xc, N_el)."""
        c = self.case
        Cf = c.c_fortran() if C is None else np.ascontiguousarray(C, dtype=np.float64).reshape(-1)
        of = c.occ_fortran() if occ is None else np.ascontiguousarray(occ, dtype=np.float64).reshape(-1)
        ids = np.array([abi.XC_IDS[f] for f in functionals], dtype=np.int32)
        out = np.zeros(len(ids))
        nel = ct.c_double(0.0)
        _check(lib().pgxc_xc_energies(self.h, abi.f64p(Cf), abi.f64p(of), c.nbas, c.nocc, c.ispin, len(ids),
                                      abi.i32p(ids), abi.f64p(out), ct.byref(nel)), self.h)
        return list(out), nel.value

    def set_symmetry(self, ad):
        """Attach a symmetry adaptation (pgxc.symmetry.Adaptation)."""
        self._sym = abi.MarshalledSymmetry(ad)
        _check(lib().pgxc_set_symmetry(self.h, ct.byref(self._sym.s)), self.h)
        n = ct.c_int64()
        _check(lib().pgxc_sym_xc_length(self.h, ct.byref(n)), self.h)
        self.sym_xc_length = n.value

    def set_pseudo2d(self, nblocks, first=(), half=()):
        """Pseudo-2D irreps (pgxc_set_pseudo2d): per irrep its (atom, l) blocks'
        first functions and half sizes; None removes it."""
        if nblocks is None:
            _check(lib().pgxc_set_pseudo2d(self.h, None, None, None), self.h)
            return
        self._p2 = [np.ascontiguousarray(x, dtype=np.int32) for x in (nblocks, first, half)]
        _check(lib().pgxc_set_pseudo2d(self.h, *[abi.i32p(x) for x in self._p2]), self.h)

    def build_sym(self, Cs, occs, ham=None, timings=False):
        """Symmetry-adapted build from per-irrep C (dims, nocc, ispin) and occ
        (nocc, ispin); returns (ham_xc_arr, exc, nel[, timings])."""
        o = abi.IrrepOrbitals(Cs, occs)
        n = getattr(self, "sym_xc_length", 0)   # 0 before set_symmetry: the library reports the error
        if ham is None:
            ham = np.zeros(n)
        exc = ct.c_double(0.0)
        nel = ct.c_double(0.0)
        tm = abi.Timings()
        _check(lib().pgxc_build_sym(self.h, o.pC, o.pocc, abi.i32p(o.nocc), self.case.ispin, abi.f64p(ham),
                                    n, ct.byref(exc), ct.byref(nel), ct.byref(tm)), self.h)
        if timings:
            return ham, exc.value, nel.value, tm.as_dict()
        return ham, exc.value, nel.value

    def xc_gradient_sym(self, Cs, occs):
        """XC nuclear gradient of a symmetry-adapted context from per-irrep C
        and occ (as build_sym); returns (grad (natoms, 3), E_xc)."""
        o = abi.IrrepOrbitals(Cs, occs)
        g = np.zeros(3 * len(self.case.coords))
        e = ct.c_double(0.0)
        _check(lib().pgxc_xc_gradient_sym(self.h, o.pC, o.pocc, abi.i32p(o.nocc), self.case.ispin, abi.f64p(g),
                                          ct.byref(e)), self.h)
        return g.reshape(-1, 3), e.value

    def build_density(self, P, ham=None):
        """Build from density matrices P (ispin, nbas, nbas); returns (ham_xc_arr, exc, nel)."""
        c = self.case
        Pf = np.ascontiguousarray(np.asarray(P, dtype=np.float64).reshape(c.ispin, c.nbas, c.nbas)).reshape(-1)
        if ham is None:
            ham = np.zeros(c.xc_length)
        exc = ct.c_double(0.0)
        nel = ct.c_double(0.0)
        tm = abi.Timings()
        _check(lib().pgxc_build_density(self.h, abi.f64p(Pf), c.nbas, c.ispin, abi.f64p(ham), c.xc_length,
                                        ct.byref(exc), ct.byref(nel), ct.byref(tm)), self.h)
        return ham, exc.value, nel.value

    def build_device(self, d_C, d_occ, d_ham, d_exc_nel):
        """Device-pointer build (ints); returns the timings dict."""
        c = self.case
        tm = abi.Timings()
        st = lib().pgxc_build_device(self.h, d_C, d_occ, c.nbas, c.nocc, c.ispin, d_ham, c.xc_length, d_exc_nel,
                                     ct.byref(tm))
        _check(st, self.h)
        return tm.as_dict()

    def screen_stats(self):
        """{ntiles, nslots, nlisted, sum_n2} of a screened context."""
        v = [ct.c_int64(), ct.c_int64(), ct.c_int64(), ct.c_double()]
        _check(lib().pgxc_screen_stats(self.h, *[ct.byref(x) for x in v]), self.h)
        return dict(ntiles=v[0].value, nslots=v[1].value, nlisted=v[2].value, sum_n2=v[3].value)

    def grid_weights(self):
        w = np.zeros(self.case.npts)
        _check(lib().pgxc_grid_weights(self.h, abi.f64p(w), len(w)), self.h)
        return w

    def orbitals(self, pts, grads=True):
        pts = np.asarray(pts, dtype=np.float64)
        n = len(pts)
        p = np.ascontiguousarray(pts.T).reshape(-1)
        phi = np.zeros(n * self.nbas)
        gr = np.zeros(n * 3 * self.nbas) if grads else None
        _check(lib().pgxc_orbital_calculate(self.h, n, abi.f64p(p), abi.f64p(phi), abi.f64p(gr)), self.h)
        phi = phi.reshape(self.nbas, n).T
        if grads:
            gr = gr.reshape(self.nbas, 3, n).transpose(2, 1, 0)
        return phi, gr

    def close(self):
        if getattr(self, "h", None):
            lib().pgxc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Batch:
    """Device builds of many screened contexts replayed as one CUDA graph
    (pgxc_batch_create / pgxc_batch_run).  Per context the operands are device
    pointers (ints): C and occ in the pgxc_build_device layout, the packed V
    and {E_xc, N_el} outputs (overwritten by every run)."""

    def __init__(self, contexts, d_C, d_occ, d_ham, d_exc_nel, max_chunk_points=0):
        """max_chunk_points: the chunk of a set of INT8 contexts (0: from free memory)."""
        n = len(contexts)
        arr = lambda xs: (ct.c_void_p * n)(*[ct.c_void_p(int(x)) for x in xs])
        self.contexts = list(contexts)  # kept alive while the batch exists
        self._args = (arr([c.h.value for c in contexts]), arr(d_C), arr(d_occ),
                      (ct.c_int32 * n)(*[c.case.nocc for c in contexts]), arr(d_ham), arr(d_exc_nel))
        h = ct.c_void_p()
        a = self._args
        _check(lib().pgxc_batch_create_chunked(a[0], n, a[1], a[2], a[3], a[4], a[5], int(max_chunk_points),
                                               ct.byref(h)))
        self.h = h

    def is_set(self):
        """Whether the batch runs as one set (one launch per kernel over all contexts' tiles)."""
        v = ct.c_int32()
        _check(lib().pgxc_batch_is_set(self.h, ct.byref(v)))
        return bool(v.value)

    def run(self):
        """One replay of every build; returns its device time in ms."""
        ms = ct.c_double()
        _check(lib().pgxc_batch_run(self.h, ct.byref(ms)))
        return ms.value

    def stats(self):
        """{kernel_nodes, nodes} of the batch's CUDA graph."""
        k, n = ct.c_int64(), ct.c_int64()
        _check(lib().pgxc_batch_stats(self.h, ct.byref(k), ct.byref(n)))
        return dict(kernel_nodes=k.value, nodes=n.value)

    def close(self):
        if self.h:
            lib().pgxc_batch_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def xc_functionals(xc, rho, gam=None):
    """Point functional on the device.  Closed shell: rho (n,), gam (n,) or
    None -> f, fr, fg of shape (n,).  Open shell: rho (n, 2), gam (n, 3) =
    (aa, bb, ab) or None -> f (n,), fr (n, 2), fg (n, 3)."""
    rho = np.asarray(rho, dtype=np.float64)
    ispin = 2 if rho.ndim == 2 else 1
    n = len(rho)
    ng = 2 * ispin - 1
    r = np.ascontiguousarray(rho.reshape(n, ispin).T).reshape(-1)
    g = None if gam is None else np.ascontiguousarray(np.asarray(gam, dtype=np.float64).reshape(n, ng).T).reshape(-1)
    f = np.zeros(n)
    fr = np.zeros(n * ispin)
    fg = np.zeros(n * ng) if g is not None else None
    _check(lib().pgxc_xc_functionals(abi.XC_IDS[xc], ispin, n, abi.f64p(r), abi.f64p(g), abi.f64p(f), abi.f64p(fr),
                                     abi.f64p(fg)))
    if ispin == 1:
        return f, fr, fg
    return f, fr.reshape(ispin, n).T, None if fg is None else fg.reshape(ng, n).T


def becke_weights(case):
    m = abi.Marshalled(case, weighted=False)
    pts = np.ascontiguousarray(case.grid_xyz.T).reshape(-1)
    owner = np.ascontiguousarray(case.point_atom, dtype=np.int32)
    w = np.zeros(case.npts)
    _check(lib().pgxc_becke_weights(ct.byref(m.geometry), case.npts, abi.f64p(pts), abi.i32p(owner), abi.f64p(w)))
    return w


def xc_functionals_mgga(xc, rho, gam, tau):
    """Meta-GGA point functional on the device: rho, gam, tau as the oracle's
    functionals_mgga ((n, ispin), (n, 2 ispin - 1), (n, ispin)) -> f (n,),
    fr (n, ispin), fg (n, 2 ispin - 1), ft (n, ispin)."""
    rho = np.asarray(rho, dtype=np.float64)
    n = rho.shape[0]
    rho = rho.reshape(n, -1)
    ispin = rho.shape[1]
    ng = 2 * ispin - 1
    col = lambda a, k: np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(n, k).T).reshape(-1)
    r, g, t = col(rho, ispin), col(gam, ng), col(tau, ispin)
    f, fr, fg, ft = np.zeros(n), np.zeros(n * ispin), np.zeros(n * ng), np.zeros(n * ispin)
    _check(lib().pgxc_xc_functionals_mgga(abi.XC_IDS[xc], ispin, n, abi.f64p(r), abi.f64p(g), abi.f64p(t),
                                          abi.f64p(f), abi.f64p(fr), abi.f64p(fg), abi.f64p(ft)))
    return f, fr.reshape(ispin, n).T, fg.reshape(ng, n).T, ft.reshape(ispin, n).T
