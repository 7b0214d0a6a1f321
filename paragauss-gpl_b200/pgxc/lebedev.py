"""Lebedev-McLaren angular quadratures on the unit sphere, as ParaGauss uses them.

ParaGauss builds its angular grids in INIGRD (modules/grid_module.f90:1359-2100)
from octahedrally symmetric point orbits (A. D. McLaren, Math. Comp. 17, 361
(1963); V. I. Lebedev's rules up to degree 29).  The rule parameters below are
the published constants exactly as that routine holds them (a table of
published numbers has to be alike); the orbit generators are written here from
the orbits' definitions and emit the points in the order INIGRD emits them, so
the grids are point-for-point the reference's.

Orbits (all with the full octahedral sign/permutation symmetry):
  a1  6 points  (+-1, 0, 0) and permutations
  a2 12 points  (+-1/sqrt2, +-1/sqrt2, 0) and permutations
  a3  8 points  (+-1/sqrt3, +-1/sqrt3, +-1/sqrt3)
  b  24 points  (+-l, +-l, +-m), l = sqrt((1 - m^2)/2), and permutations
  c  24 points  (+-p, +-q, 0), p, q = sqrt((1 +- sqrt(1 - 4v))/2), and permutations
  d  48 points  (+-u, +-w, +-r), r = sqrt(1 - u^2 - w^2), all permutations

Weights sum to one (the 4 pi of the one-centre weight is applied by the grid
builder, grid_main_calc :425-432).  Where INIGRD writes a weight to 12 digits
the rule integrates constants to about 1e-11, as the reference's does.

The reference's grid code selects a rule by its order code ICGRD (31, 32, 33,
51, 71, ..., 291); NANG_TO_POINTS maps those codes to point counts
(grid_main_calc :371-372).
"""
import math

import numpy as np

# ICGRD order code -> number of points (grid_main_calc nang_par, plus the two
# McLaren rules 32 and 33 that INIGRD also holds)
NANG_TO_POINTS = {31: 6, 32: 8, 33: 12, 51: 14, 71: 26, 91: 38, 111: 50, 131: 78, 151: 86, 171: 110,
                  191: 146, 231: 194, 291: 302}

# points -> list of (orbit, parameters, weight)
RULES = {
    6: [("a1", (), 1.0 / 6.0)],
    8: [("a3", (), 1.0 / 8.0)],
    12: [("a2", (), 1.0 / 12.0)],
    14: [("a1", (), 8.0 / 120.0), ("a3", (), 9.0 / 120.0)],
    26: [("a1", (), 40.0 / 840.0), ("a2", (), 32.0 / 840.0), ("a3", (), 27.0 / 840.0)],
    38: [("a1", (), 1.0 / 105.0), ("a3", (), 9.0 / 280.0), ("c", (1.0 / 6.0,), 1.0 / 35.0)],
    50: [("a1", (), 4.0 / 315.0), ("a2", (), 64.0 / 2835.0), ("a3", (), 27.0 / 1280.0),
         ("b", (3.0 / math.sqrt(11.0),), 14641.0 / 725760.0)],
    78: [("a1", (), 0.0138665921047), ("b", (0.914152532416,), 0.0130509318626),
         ("b", (0.359236381200,), 0.0132064232231), ("c", (0.206339716383,), 0.0119426635549)],
    86: [("a1", (), 8.0 / 693.0), ("a3", (), 0.0119439090859), ("b", (0.852518311701,), 0.0111105557106),
         ("b", (0.189063552885,), 0.0118765012945), ("c", (0.120441650315,), 0.0118123037469)],
    110: [("a1", (), 0.00382827049494), ("a3", (), 0.00979373751249),
          ("b", (0.965124035087,), 0.00821173728319), ("b", (0.828769981253,), 0.00959547133607),
          ("b", (0.215957291846,), 0.00994281489118), ("c", (3.0 / 17.0,), 19652.0 / 2027025.0)],
    146: [("a1", (), 1856.0 / 3095235.0), ("a2", (), 606208.0 / 82219995.0),
          ("a3", (), 6490935.0 / 900204032.0), ("b", (0.974888643677,), 7.57439415905e-03),
          ("b", (0.807089818360,), 6.75382948631e-03), ("b", (0.291298882210,), 7.11635549312e-03),
          ("d", (0.140355381171, 0.449332832327), 1773593.0 / 253693440.0)],
    194: [("a1", (), 1.78234044724e-03), ("a2", (), 5.71690594998e-03), ("a3", (), 5.57338317884e-03),
          ("b", (0.777493219315,), 5.51877146727e-03), ("b", (0.912509096867,), 5.15823771181e-03),
          ("b", (0.314196994183,), 5.60870408259e-03), ("b", (0.982972302707,), 4.10677702817e-03),
          ("c", (2.0 / 19.0,), 5.05184606462e-03), ("d", (0.159041710538, 0.525118572443), 5.53024891623e-03)],
    302: [("a1", (), 8.54591172878e-04), ("a3", (), 3.59911928502e-03),
          ("b", (0.129238672710,), 3.65004580768e-03), ("b", (0.371034178385,), 3.60482260142e-03),
          ("b", (0.743452042987,), 3.57672966173e-03), ("b", (0.867643624544,), 3.44978842429e-03),
          ("b", (0.949454317226,), 3.10895312238e-03), ("b", (0.990705621379,), 2.35210141366e-03),
          ("c", (0.220093335298,), 3.60082093222e-03), ("c", (0.650272754659e-01,), 2.98234496317e-03),
          ("d", (0.800072749407, 0.544867737258), 3.57154055427e-03),
          ("d", (0.902442529533, 0.412772408317), 3.39231220501e-03)],
}

_SIGNS = [(i, j, k) for i in (-1.0, 1.0) for j in (-1.0, 1.0) for k in (-1.0, 1.0)]
_AXIS_PAIRS = ((0, 1), (0, 2), (1, 2))
_SIGN_PAIRS = ((1.0, 1.0), (1.0, -1.0), (-1.0, 1.0), (-1.0, -1.0))


def _two_axis(a, b):
    """12 points with a, b on two axes (pairs xy, xz, yz; signs ++, +-, -+, --), third 0."""
    out = []
    for ax, bx in _AXIS_PAIRS:
        for sa, sb in _SIGN_PAIRS:
            v = [0.0, 0.0, 0.0]
            v[ax] = sa * a
            v[bx] = sb * b
            out.append(v)
    return out


def _three_types(t1, t2, t3):
    """24 points: the 8 sign triples applied to t1, then to t2, then to t3."""
    return [[s[0] * t[0], s[1] * t[1], s[2] * t[2]] for t in (t1, t2, t3) for s in _SIGNS]


def orbit(kind, params=()):
    """Points of one orbit, (n, 3), in INIGRD's order."""
    if kind == "a1":
        pts = [[0, 0, 1], [0, 0, -1], [0, 1, 0], [0, -1, 0], [1, 0, 0], [-1, 0, 0]]
    elif kind == "a2":
        pts = _two_axis(1.0 / math.sqrt(2.0), 1.0 / math.sqrt(2.0))
    elif kind == "a3":
        r = 1.0 / math.sqrt(3.0)
        pts = [[s[0] * r, s[1] * r, s[2] * r] for s in _SIGNS]
    elif kind == "b":
        (m,) = params
        lk = math.sqrt((1.0 - m * m) / 2.0)
        pts = _three_types((lk, lk, m), (lk, m, lk), (m, lk, lk))
    elif kind == "c":
        (v,) = params
        d = math.sqrt(1.0 - 4.0 * v)
        p, q = math.sqrt((1.0 + d) / 2.0), math.sqrt((1.0 - d) / 2.0)
        pts = _two_axis(p, q) + _two_axis(q, p)
    elif kind == "d":
        u, w = params
        r = math.sqrt(1.0 - u * u - w * w)
        first = _three_types((u, w, r), (w, r, u), (r, u, w))
        pts = first + [[x, z, y] for x, y, z in first]
    else:
        raise ValueError(kind)
    return np.asarray(pts, dtype=np.float64)


def rule(npts):
    """(points (n, 3), weights (n,)) of the rule with npts points."""
    if npts not in RULES:
        raise ValueError(f"no Lebedev-McLaren rule with {npts} points; have {sorted(RULES)}")
    ps, ws = [], []
    for kind, params, w in RULES[npts]:
        o = orbit(kind, params)
        ps.append(o)
        ws.append(np.full(len(o), w))
    pts, wts = np.concatenate(ps), np.concatenate(ws)
    assert len(pts) == npts
    return pts, wts
