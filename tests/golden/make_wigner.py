"""Exact Wigner 3j/6j/9j values from sympy.physics.wigner for tests/test_math.py.

    python tests/golden/make_wigner.py      (writes tests/golden/wigner.npz)
"""
import os

import numpy as np
from sympy import Rational
from sympy.physics.wigner import wigner_3j, wigner_6j, wigner_9j

HERE = os.path.dirname(os.path.abspath(__file__))
rng = np.random.default_rng(20261203)


def h(x):
    return Rational(int(x), 2)


def tri(a, b, c):
    return (a + b + c) % 2 == 0 and abs(a - b) <= c <= a + b


def valid6(a):
    return tri(a[0], a[1], a[2]) and tri(a[0], a[4], a[5]) and tri(a[3], a[1], a[5]) and tri(a[3], a[4], a[2])


def valid9(a):
    return (tri(a[0], a[1], a[2]) and tri(a[3], a[4], a[5]) and tri(a[6], a[7], a[8]) and tri(a[0], a[3], a[6])
            and tri(a[1], a[4], a[7]) and tri(a[2], a[5], a[8]))


def tri_pick(a, b):
    """A doubled j3 coupling a and b (triangle and parity), or None."""
    lo, hi = abs(a - b), a + b
    if hi < lo:
        return None
    return int(lo + 2 * rng.integers(0, (hi - lo) // 2 + 1))


def large_9j(count, top):
    """Valid 9j symbols with doubled arguments up to `top`: the recoupling
    coefficients of two-body j <= 4 and three-body J <= 9/2 reach about 18."""
    t, v = [], []
    while len(t) < count:
        a = [0] * 9
        a[0], a[1] = (int(x) for x in rng.integers(0, top + 1, 2))
        a[3], a[4] = (int(x) for x in rng.integers(0, top + 1, 2))
        a[2], a[5] = tri_pick(a[0], a[1]), tri_pick(a[3], a[4])
        a[6], a[7] = tri_pick(a[0], a[3]), tri_pick(a[1], a[4])
        if None in a[:8] or max(a[:8]) > top:
            continue
        lo = max(abs(a[6] - a[7]), abs(a[2] - a[5]))
        hi = min(a[6] + a[7], a[2] + a[5], top)
        cands = [x for x in range(lo, hi + 1) if (a[6] + a[7] + x) % 2 == 0 and (a[2] + a[5] + x) % 2 == 0]
        if not cands:
            continue
        a[8] = int(cands[rng.integers(0, len(cands))])
        if not valid9(a):
            continue
        t.append(tuple(a))
        v.append(float(wigner_9j(*[h(x) for x in a])))
    return t, v


def main():
    t3, v3 = [], []
    while len(t3) < 400:
        j1, j2 = rng.integers(0, 13, 2)
        j3 = rng.integers(abs(j1 - j2), j1 + j2 + 1)
        if (j1 + j2 + j3) % 2:
            j3 = j3 + 1 if j3 + 1 <= j1 + j2 else j3 - 1
        m1 = rng.integers(-j1, j1 + 1)
        m1 -= (m1 - j1) % 2
        m2 = rng.integers(-j2, j2 + 1)
        m2 -= (m2 - j2) % 2
        m3 = -m1 - m2
        if abs(m3) > j3 or (j3 + m3) % 2 or (j1 + j2 + j3) % 2 or not (abs(j1 - j2) <= j3 <= j1 + j2):
            continue
        t3.append((j1, j2, j3, m1, m2, m3))
        v3.append(float(wigner_3j(h(j1), h(j2), h(j3), h(m1), h(m2), h(m3))))
    t6, v6 = [], []
    n_invalid = 0
    while len(t6) < 400:
        a = rng.integers(0, 17, 6)
        if not valid6(a):
            if n_invalid >= 60:
                continue
            n_invalid += 1
        try:
            val = wigner_6j(*[h(x) for x in a])
        except ValueError:  # sympy rejects triangle/parity violations; the symbol is 0
            val = 0
        t6.append(tuple(a))
        v6.append(float(val))
    t9, v9 = [], []
    n_invalid = 0
    while len(t9) < 200:
        a = rng.integers(0, 9, 9)
        a[4] = 1 if rng.random() < 0.5 else a[4]  # the reference's spin-1/2 slot
        if not valid9(a):
            if n_invalid >= 30:
                continue
            n_invalid += 1
        t9.append(tuple(a))
        try:
            val = wigner_9j(*[h(x) for x in a], prec=None)
        except ValueError:
            val = 0
        v9.append(float(val))
    t9b, v9b = large_9j(120, 18)
    np.savez_compressed(os.path.join(HERE, "wigner.npz"), t9b=np.array(t9b), v9b=np.array(v9b), t3=np.array(t3),
                        v3=np.array(v3), t6=np.array(t6),
                        v6=np.array(v6), t9=np.array(t9), v9=np.array(v9))


if __name__ == "__main__":
    main()
