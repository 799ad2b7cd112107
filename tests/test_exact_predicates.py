"""Known-answer tests of the exact predicates (nif_exact.h, through the CPU
oracle library) and of their static filters.

Every sign is checked against two independent answers: exact rational
arithmetic (Python fractions; a double is a dyadic rational, so the
determinants are exact), and Shewchuk's adaptive robust predicates as
natinterp3d ships them in predicates.c (compiled in oracle/_ref, where
natinterp3d's sources are available).  Inputs: random points, near-coplanar and
near-cospherical points a few ulps off, exactly degenerate lattice points,
translated and widely scaled coordinates."""
from fractions import Fraction

import numpy as np
import pytest

from oracle import oracle


def _sgn(x):
    return (x > 0) - (x < 0)


def _det3(m):
    return (m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1])
            - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0])
            + m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]))


def _det4(m):
    total = 0
    for j in range(4):
        minor = [[m[i][k] for k in range(4) if k != j] for i in range(1, 4)]
        total += (-1) ** j * m[0][j] * _det3(minor)
    return total


def orient_rational(a, b, c, d):
    F = [[Fraction(float(p[k])) - Fraction(float(d[k])) for k in range(3)] for p in (a, b, c)]
    return _sgn(_det3(F))


def insphere_rational(a, b, c, d, e):
    rows = []
    for p in (a, b, c, d):
        r = [Fraction(float(p[k])) - Fraction(float(e[k])) for k in range(3)]
        rows.append(r + [r[0] * r[0] + r[1] * r[1] + r[2] * r[2]])
    return _sgn(_det4(rows))


def _cases(rng, n):
    """(orient quadruples, insphere quintuples) covering the hard regimes"""
    o, s = [], []
    for _ in range(n):
        a, b, c = rng.uniform(-1, 1, (3, 3))
        # random
        o.append((a, b, c, rng.uniform(-1, 1, 3)))
        s.append((a, b, c, rng.uniform(-1, 1, 3), rng.uniform(-1, 1, 3)))
        # near-coplanar: d on the plane of a, b, c, rounded, then nudged a few ulps
        u, v = rng.uniform(-2, 2, 2)
        d = a + u * (b - a) + v * (c - a)
        d = d + rng.integers(-3, 4, 3) * np.spacing(d)
        o.append((a, b, c, d))
        # near-cospherical: five points on one sphere, rounded, nudged
        cen = rng.uniform(-1, 1, 3)
        rad = rng.uniform(0.1, 2)
        dirs = rng.standard_normal((5, 3))
        pts = cen + rad * dirs / np.linalg.norm(dirs, axis=1, keepdims=True)
        pts[4] = pts[4] + rng.integers(-2, 3, 3) * np.spacing(pts[4])
        s.append(tuple(pts))
        # far from the origin, tiny extent (translated data)
        off = np.full(3, 1e6)
        loc = rng.uniform(-1e-3, 1e-3, (5, 3)) + off
        o.append(tuple(loc[:4]))
        s.append(tuple(loc))
    # exact degeneracies on a lattice: coplanar and cospherical points
    lat = rng.integers(-4, 5, (4 * n, 5, 3)).astype(np.float64)
    for p in lat:
        p2 = p.copy()
        p2[3, 2] = p2[0, 2]
        p2[3, :2] = p2[0, :2] + (p2[1, :2] - p2[0, :2])  # frequently coplanar
        o.append(tuple(p[:4]))
        o.append(tuple(p2[:4]))
        s.append(tuple(p))
    sph = np.array([[3, 4, 0], [0, 3, 4], [4, 0, 3], [-5, 0, 0], [0, 0, 5], [0, -4, 3],
                    [5, 0, 0], [0, 5, 0]], np.float64)
    for k in range(n):
        idx = rng.choice(len(sph), 5, replace=False)
        pts = sph[idx] * (2.0 ** rng.integers(-30, 30)) + rng.integers(-3, 4) * 0.5
        s.append(tuple(pts))                                        # exactly cospherical
        q = pts.copy()
        q[4] = q[4] + np.spacing(q[4]) * rng.choice([-1.0, 1.0], 3)
        s.append(tuple(q))                                          # one ulp off
    # widely different magnitudes
    for _ in range(n):
        scale = 10.0 ** rng.integers(-12, 12, (5, 1))
        p = rng.uniform(-1, 1, (5, 3)) * scale
        o.append(tuple(p[:4]))
        s.append(tuple(p))
    return o, s


@pytest.fixture(scope='module')
def cases():
    return _cases(np.random.default_rng(7), 60)


def test_orient_exact_sign_matches_rational_arithmetic(cases):
    o, _ = cases
    zeros = 0
    for args in o:
        want = orient_rational(*args)
        zeros += want == 0
        assert oracle.orient_exact_sign(*args) == want, args
    assert zeros > 10  # the lattice cases produce true zeros


def test_insphere_exact_sign_matches_rational_arithmetic(cases):
    _, s = cases
    zeros = 0
    for args in s:
        want = insphere_rational(*args)
        zeros += want == 0
        assert oracle.insphere_exact_sign(*args) == want, args
    assert zeros > 10


def test_filters_only_certify_correct_signs(cases):
    o, s = cases
    unc_o = unc_s = 0
    for args in o:
        if oracle.orient_uncertain(*args):
            unc_o += 1
        else:
            assert _sgn(oracle.orient(*args)) == orient_rational(*args)
    for args in s:
        if oracle.insphere_uncertain(*args):
            unc_s += 1
        else:
            assert _sgn(oracle.insphere(*args)) == insphere_rational(*args)
    # the near-degenerate families reach inside the bounds, the random ones do not
    assert unc_o > 20 and unc_s > 20
    assert unc_o < len(o) and unc_s < len(s)


def test_fast_signs_are_wrong_somewhere_inside_the_bound(cases):
    """The point of the exact path: the non-robust sign does flip on these inputs."""
    o, s = cases
    flips = sum(_sgn(oracle.orient(*a)) != orient_rational(*a) for a in o)
    flips += sum(_sgn(oracle.insphere(*a)) != insphere_rational(*a) for a in s)
    assert flips > 0


@pytest.mark.skipif(not oracle.ref_available(), reason='natinterp3d reference library not built')
def test_exact_signs_match_shewchuks_robust_predicates(cases):
    o, s = cases
    for args in o:
        assert oracle.orient_exact_sign(*args) == _sgn(oracle.ref_orient3d_robust(*args)), args
    for args in s:
        assert oracle.insphere_exact_sign(*args) == _sgn(oracle.ref_insphere_robust(*args)), args
