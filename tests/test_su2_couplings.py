"""SU(2) recoupling coefficients of the SU2U1 builder against sympy's exact
Wigner symbols (independent implementation of the same published formulas)."""
import itertools
import math

import pytest
from sympy import Rational
from sympy.physics.wigner import wigner_6j, wigner_9j

from dmrgb200 import _capi as capi

H = Rational(1, 2)


def tri(a, b, c):
    return abs(a - b) <= c <= a + b and (a + b + c) % 2 == 0


def test_wigner6j_grid():
    vals = range(0, 7)
    n = 0
    for args in itertools.product(vals, repeat=6):
        a, b, c, d, e, f = args
        if not (tri(a, b, c) and tri(a, e, f) and tri(d, b, f) and tri(d, e, c)):
            continue
        exact = float(wigner_6j(*[x * H for x in args]))
        got = capi.lib.dmrgb200_wigner6j(*args)
        assert abs(got - exact) <= 1e-13 * max(1.0, abs(exact)), args
        n += 1
    assert n > 500


@pytest.mark.parametrize("seed", range(4))
def test_wigner9j_random(seed):
    import random
    rng = random.Random(seed)
    n = 0
    while n < 150:
        a, b = rng.randint(0, 6), rng.randint(0, 6)
        c = rng.choice([x for x in range(abs(a - b), a + b + 1, 2)])
        d, e = rng.randint(0, 6), rng.randint(0, 6)
        f = rng.choice([x for x in range(abs(d - e), d + e + 1, 2)])
        g = rng.choice([x for x in range(abs(a - d), a + d + 1, 2)])
        h = rng.choice([x for x in range(abs(b - e), b + e + 1, 2)])
        opts = [x for x in range(abs(c - f), c + f + 1, 2) if tri(g, h, x)]
        if not opts:
            continue
        i = rng.choice(opts)
        args = (a, b, c, d, e, f, g, h, i)
        exact = float(wigner_9j(*[x * H for x in args]))
        got = capi.lib.dmrgb200_wigner9j(*args)
        assert abs(got - exact) <= 1e-12 * max(1.0, abs(exact)), args
        n += 1


def test_set_coupling_cases():
    """Four couplings: (row, col) spin cases of op_iterate (op_iterate.hpp:56-63)."""
    import ctypes as C
    out = (C.c_double * 4)()
    for args in [(1, 1, 2, 1, 1, 0, 2, 1, 1), (0, 1, 1, 2, 2, 2, 2, 1, 1), (2, 0, 2, 1, 0, 1, 1, 1, 2)]:
        a, b, c, d, e, f, g, h, i = args
        capi.lib.dmrgb200_set_coupling(*args, 0.5, out)
        pre = math.sqrt((i + 1) * (a + 1) / ((g + 1) * (c + 1))) * 0.5

        def mod(a_, b_, c_, d_, e_, f_, g_, h_, i_):
            try:
                w = float(wigner_9j(*[x * H for x in (a_, b_, c_, d_, e_, f_, g_, h_, i_)]))
            except ValueError:  # sympy rejects non-integer perimeters: the symbol vanishes
                w = 0.0
            return math.sqrt((g_ + 1) * (h_ + 1) * (c_ + 1) * (f_ + 1)) * w
        exp = [0.0] * 4
        if abs(a - b) <= c <= a + b:
            exp[0] = pre * mod(a, b, c, d, e, f, g, h, i)
            exp[2] = pre * mod(a, b, c, d, e, f, g, 2, i)
        if abs(a - 2) <= c <= a + 2:
            exp[1] = pre * mod(a, 2, c, d, e, f, g, h, i)
            exp[3] = pre * mod(a, 2, c, d, e, f, g, 2, i)
        for k in range(4):
            assert abs(out[k] - exp[k]) <= 1e-13, (args, k)
