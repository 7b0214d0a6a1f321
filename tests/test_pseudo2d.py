"""Pseudo-2D irrep symmetrisation (xc_pseudo2d_sym, modules/xc_hamiltonian.f90
:2637-2779): the oracle's restatement of the reference's packed-index loops
against the rule it implements, written here directly on full matrices."""
import numpy as np
import pytest

import oracle as O


def unpack_irreps(h, ispin, dims):
    """Packed (k <= j column order, spin stride, irreps one after the other) ->
    full symmetric matrices [irrep][spin]."""
    out, off = [], 0
    for d in dims:
        mats = []
        for s in range(ispin):
            m = np.zeros((d, d))
            for j in range(d):
                for k in range(j + 1):
                    m[k, j] = m[j, k] = h[s + ispin * (off + j * (j + 1) // 2 + k)]
            mats.append(m)
        out.append(mats)
        off += d * (d + 1) // 2
    return out


def rule(h, ispin, dims, nblocks, first, half):
    """H(X_A, Y_A) = H(X_B, Y_B) = their mean; H(X_A, Y_B) = -H(X_B, Y_A) =
    half their difference; block pairs X >= Y, element (r, c) of X x Y with
    r in X, c in Y, and for X == Y only r >= c (A x A, B x B) / the cross
    pairs (B_c, A_r), (B_r, A_c) with c <= r."""
    mats = unpack_irreps(h, ispin, dims)
    b0 = 0
    for i, d in enumerate(dims):
        blk = [(first[b0 + b], half[b0 + b]) for b in range(nblocks[i])]
        for s in range(ispin):
            m = mats[i][s]
            for x, (px, hx) in enumerate(blk):
                for y in range(x + 1):
                    py, hy = blk[y]
                    for r in range(hx):
                        for c in range(hy if x != y else r + 1):
                            aa, bb = (px + r, py + c), (px + hx + r, py + hy + c)
                            v = 0.5 * (m[aa] + m[bb])
                            m[aa] = m[aa[::-1]] = m[bb] = m[bb[::-1]] = v
                            if x != y:
                                ab, ba = (px + r, py + hy + c), (px + hx + r, py + c)
                            else:
                                ab, ba = (px + hx + c, px + r), (px + hx + r, px + c)
                            v = 0.5 * (m[ab] - m[ba])
                            m[ab] = m[ab[::-1]] = v
                            m[ba] = m[ba[::-1]] = -v
        b0 += nblocks[i]
    out, off = np.zeros_like(h), 0
    for i, d in enumerate(dims):
        for s in range(ispin):
            m = mats[i][s]
            for j in range(d):
                for k in range(j + 1):
                    out[s + ispin * (off + j * (j + 1) // 2 + k)] = m[k, j]
        off += d * (d + 1) // 2
    return out


def layout(rng):
    """Two irreps, the second pseudo-2D with three (atom, l) blocks."""
    halves = [2, 3, 1]
    gaps = [1, 0, 2]
    first, pos = [], 0
    for g, hh in zip(gaps, halves):
        pos += g
        first.append(pos)
        pos += 2 * hh
    dims = [5, pos + 1]
    return dims, [0, 3], first, halves


@pytest.mark.parametrize("ispin", [1, 2])
def test_oracle_restatement_is_the_rule(ispin):
    rng = np.random.default_rng(7 + ispin)
    dims, nblocks, first, half = layout(rng)
    n = ispin * sum(d * (d + 1) // 2 for d in dims)
    h = rng.normal(size=n)
    got = O.pseudo2d_sym(h, ispin, dims, nblocks, first, half)
    want = rule(h, ispin, dims, nblocks, first, half)
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-15)
    # the first irrep is not pseudo-2D: untouched
    n0 = ispin * dims[0] * (dims[0] + 1) // 2
    assert np.array_equal(got[:n0], h[:n0])
    # idempotent: a symmetrised matrix is a fixed point
    np.testing.assert_allclose(O.pseudo2d_sym(got, ispin, dims, nblocks, first, half), got, rtol=0, atol=1e-15)
