"""CPU tests of the decision-exact predicates (PAC_PRED_EXACT's checker).

The restatement's exact predicates (oracle/exact_oracle.cpp: an
extended-precision filter, then arbitrary-precision integers over the
multiplied-out polynomials) are pinned here against a third formulation:
rational arithmetic (fractions.Fraction) on the geometric definitions --
the radical foot of an edge and the orthocentres of triangles and
tetrahedra solved as linear systems, powers compared at those points, and
the orientation/insphere determinants expanded by cofactors."""
from fractions import Fraction as F

import numpy as np
import pytest

from conftest import canonical


def _q(b):
    """Ball (x, y, z, r) as exact rationals, weight r^2."""
    x, y, z, r = (F(float(v)) for v in b)
    return (x, y, z), r * r


def _sub(a, b):
    return tuple(p - q for p, q in zip(a, b))


def _dot(a, b):
    return sum(p * q for p, q in zip(a, b))


def _cross(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


def _det3(a, b, c):
    return _dot(a, _cross(b, c))


def _solve3(M, rhs):
    """Cramer's rule over rationals; None when singular."""
    d = _det3(*M)
    if d == 0:
        return None
    cols = list(zip(*M))
    out = []
    for k in range(3):
        c = [list(col) for col in cols]
        c[k] = list(rhs)
        out.append(_det3(*zip(*c)) / d)
    return tuple(out)


def _power(x, p, w):
    return _dot(_sub(x, p), _sub(x, p)) - w


def _centre(balls):
    """Point of equal power to all balls in their affine hull (radical
    centre): None when degenerate."""
    P = [_q(b) for b in balls]
    p1, w1 = P[0]
    rows, rhs = [], []
    for p, w in P[1:]:
        d = _sub(p, p1)
        rows.append(d)
        rhs.append((_dot(d, d) + w1 - w) / 2)  # d . y = B/2 with y = x - p1
    if len(rows) == 1:
        d = rows[0]
        dd = _dot(d, d)
        if dd == 0:
            return None
        t = rhs[0] / dd
        y = tuple(t * c for c in d)
    elif len(rows) == 2:
        n = _cross(rows[0], rows[1])
        if _dot(n, n) == 0:
            return None
        y = _solve3([rows[0], rows[1], n], [rhs[0], rhs[1], F(0)])
    else:
        y = _solve3(rows, rhs)
        if y is None:
            return None
    return tuple(a + b for a, b in zip(p1, y))


def _frac_pred(kind, balls, alpha):
    a = F(float(np.float32(alpha)))
    if kind in (0, 1, 2):
        k = kind + 2
        c = _centre(balls[:k])
        if c is None:
            return 2 if kind == 2 else 0
        p1, w1 = _q(balls[0])
        return int(_power(c, p1, w1) <= a)
    if kind == 3:
        P = [_q(b)[0] for b in balls[:4]]
        v = _det3(_sub(P[0], P[3]), _sub(P[1], P[3]), _sub(P[2], P[3]))
        return (v > 0) - (v < 0)
    if kind == 4:
        Q = [_q(b) for b in balls[:5]]
        pe, we = Q[4]
        rows = []
        for p, w in Q[:4]:
            d = _sub(p, pe)
            rows.append(list(d) + [_dot(d, d) - (w - we)])
        v = 0
        for j in range(4):  # Laplace along the lifted column
            minor = [r[:3] for i, r in enumerate(rows) if i != j]
            v += (-1) ** (j + 3) * rows[j][3] * _det3(*minor)
        return (v > 0) - (v < 0)
    # attachment: ball q at least as close (power) to the simplex's centre
    k = 2 if kind == 5 else 3
    c = _centre(balls[:k])
    p1, w1 = _q(balls[0])
    pq, wq = _q(balls[k])
    return int(_power(c, pq, wq) <= _power(c, p1, w1))


def _cases(rng, n, lattice):
    for _ in range(n):
        if lattice:
            P = rng.integers(-3, 4, size=(5, 3)) * 0.5 + 20.0
            R = rng.choice([1.5, 1.55, 1.7, 2.9, 3.1], 5)
        else:
            P = rng.normal(size=(5, 3)) * 2.5 + 30.0
            R = rng.uniform(1.4, 3.2, 5)
        yield np.concatenate([P, R[:, None]], 1).astype(np.float32)


@pytest.mark.parametrize("lattice", [False, True])
def test_exact_predicates_match_rationals(orc, lattice):
    rng = np.random.default_rng(21 + lattice)
    seen = {}
    for b in _cases(rng, 250, lattice):
        alpha = float(rng.choice([0.0, 0.5, 1.0, 2.25]))
        for kind in range(7):
            if kind in (5, 6) and _centre(b[:2 if kind == 5 else 3]) is None:
                continue  # attachment is only asked of simplices with a centre
            want = _frac_pred(kind, b, alpha)
            got = orc.exact_pred(kind, b[:[2, 3, 4, 4, 5, 3, 4][kind]], alpha)
            assert got == want, (kind, b.tolist(), alpha, got, want)
            seen.setdefault(kind, set()).add(want)
    # every predicate took more than one value; on the lattice the
    # degenerate answers (flat tetrahedra, zero determinants) occurred
    assert all(len(v) >= 2 for v in seen.values()), seen
    if lattice:
        assert 2 in seen[2] and 0 in seen[3] and 0 in seen[4]


def test_exact_mode_equals_reference_arithmetic_away_from_ties(pac, orc):
    """On a generic globule the single-precision decisions are all correct,
    so the exact mode gives the reference's complex."""
    balls = pac.globule(1500, seed=pac.SEED_BASE + 51)
    a = orc.alpha_complex(balls, 1.4, 1.0, exact=True)
    b = orc.alpha_complex(balls, 1.4, 1.0)
    for x, y in zip(a[:3], b[:3]):
        np.testing.assert_array_equal(x, y)


def test_exact_mode_differs_on_lattice_ties(pac, orc):
    """Centres on a 0.25 A lattice and radii on a 0.05 A grid: co-spherical
    and co-planar sets are common and the single-precision tests flip some
    ties; the exact mode decides them exactly (and needs its integer path)."""
    balls = pac.snapped_globule(1500, seed=pac.SEED_BASE + 52)
    import ctypes
    fb = ctypes.c_uint64.in_dll(orc.lib(), "oex_fallbacks")
    fb.value = 0
    a = orc.alpha_complex(balls, 1.4, 1.0, exact=True)
    assert fb.value > 0
    b = orc.alpha_complex(balls, 1.4, 1.0)
    d = [len(set(map(tuple, canonical(x))) ^ set(map(tuple, canonical(y))))
         for x, y in zip(a[:3], b[:3])]
    assert 0 < sum(d) < 0.01 * sum(len(x) for x in a[:3])
