"""Basis values kept on the device across builds (keep_orbitals, the
reference's orbitals_in_memory): the first build of a context evaluates and
stores phi, grad phi (and the INT8 point digits) of every slot of the grid;
later builds of the same geometry skip that evaluation.  The results must not
change, whatever the orbitals of the later builds.
"""
import numpy as np
import pytest

import oracle as O
from pgxc import cases, lib

pytestmark = pytest.mark.gpu

BUILDS = pytest.mark.parametrize("precision,thr,tol", [("fp64", 0.0, 1e-10), ("mixed", 1e-10, 1e-7)],
                                 ids=["fp64", "int8"])


def _other_orbitals(c, seed):
    rng = np.random.default_rng(seed)
    C = c.C * (1.0 + 0.2 * rng.standard_normal(c.C.shape))
    return np.ascontiguousarray(C.transpose(2, 1, 0)).reshape(-1)


@BUILDS
@pytest.mark.parametrize("xc", ["VWN", "PBE"])
def test_kept_basis_gives_the_same_builds(xc, precision, thr, tol):
    c = cases.small_case(functional=xc, seed=41, lmax=3, natoms=5, nocc=7)
    O.weight_case(c)
    kw = dict(precision=precision, screen_threshold=thr, max_chunk_points=1024)
    C2 = _other_orbitals(c, 3)
    with lib.Context(c, **kw) as plain:
        ref1 = plain.build()
        ref2 = plain.build(C=C2)
    with lib.Context(c, keep_orbitals=True, **kw) as ctx:
        r1 = ctx.build(timings=True)
        r2 = ctx.build(timings=True)
        r3 = ctx.build(C=C2)
    for got, ref in ((r1, ref1), (r2, ref1), (r3, ref2)):
        # the same kernels on the same values: E and N exactly, V up to the order of its atomics
        assert got[1] == ref[1] and got[2] == ref[2]
        np.testing.assert_allclose(got[0], ref[0], rtol=0, atol=1e-12)
    # the second build skipped the basis evaluation
    assert r2[3]["basis_ms"] < 0.5 * r1[3]["basis_ms"], (r1[3]["basis_ms"], r2[3]["basis_ms"])
    ref_ham, ref_exc, ref_nel = O.xc_build(c)
    assert abs(r2[1] - ref_exc) < tol and abs(r2[2] - ref_nel) < tol
    assert float(np.max(np.abs(r2[0] - ref_ham))) < tol


def test_kept_basis_open_shell():
    c = cases.small_case(functional="PBE", seed=42, ispin=2, nocc=7)
    O.weight_case(c)
    with lib.Context(c, screen_threshold=0.0, max_chunk_points=2048) as plain:
        ref = plain.build()
    with lib.Context(c, screen_threshold=0.0, max_chunk_points=2048, keep_orbitals=True) as ctx:
        ctx.build()
        got = ctx.build()
    assert got[1] == ref[1] and got[2] == ref[2]
    np.testing.assert_allclose(got[0], ref[0], rtol=0, atol=1e-12)


def test_kept_basis_in_a_batch():
    """A batch captured after a first build replays builds that reuse the stored values."""
    torch = pytest.importorskip("torch")
    mols = cases.molecule_set(4, seed=9, atoms=(3, 8))
    for m in mols:
        O.weight_case(m)
    ctxs = [lib.Context(m, precision="mixed", screen_threshold=1e-10, keep_orbitals=True) for m in mols]
    try:
        ops = [[torch.from_numpy(m.c_fortran()).cuda() for m in mols],
               [torch.from_numpy(m.occ_fortran()).cuda() for m in mols],
               [torch.zeros(m.xc_length, dtype=torch.float64, device="cuda") for m in mols],
               [torch.zeros(2, dtype=torch.float64, device="cuda") for m in mols]]
        for c, a, o, h, s in zip(ctxs, *ops):
            c.build_device(a.data_ptr(), o.data_ptr(), h.data_ptr(), s.data_ptr())
        first = [(h.clone(), s.clone()) for h, s in zip(ops[2], ops[3])]
        with lib.Batch(ctxs, *[[t.data_ptr() for t in x] for x in ops]) as b:
            b.run()
            b.run()
        for (h1, s1), h, s in zip(first, ops[2], ops[3]):
            assert torch.equal(s, s1)
            assert torch.allclose(h, h1, rtol=0, atol=1e-10)
    finally:
        for c in ctxs:
            c.close()
