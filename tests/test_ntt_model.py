"""The engine's own transform arithmetic (tests/ntt_model.py, bit-exact to the
CUDA passes) gives exact cyclic and negacyclic convolutions for every class of
the reference (K = 2..5 reference primes -> K + 1 transform primes below
2^30), with coefficients at the size of the normal form; and the transform
primes cover the reference's CRT range."""
import math
import random

import pytest

import ntt_model as M

REF_PRIMES = [(125 << 25) + 1, (243 << 24) + 1, (235 << 24) + 1, (29 << 27) + 1, (13 << 28) + 1]


def test_transform_primes():
    from sympy import isprime
    for p in M.TPRIMES:
        assert isprime(p) and p < (1 << 30) and p > (1 << 29) and (p - 1) % (1 << 23) == 0
    for p, g in zip(M.TPRIMES, M.TGEN):
        # g generates: g^((p-1)/q) != 1 for every prime q | p - 1
        from sympy import factorint
        assert all(pow(g, (p - 1) // q, p) != 1 for q in factorint(p - 1))
    for K in range(2, 6):
        assert math.prod(M.TPRIMES[:K + 1]) > math.prod(REF_PRIMES[:K])


@pytest.mark.parametrize("K,bits,ln", [(5, 72, 5), (5, 72, 7), (4, 62, 6), (3, 44, 6), (2, 31, 6)])
def test_model_products_are_exact(K, bits, ln):
    rng = random.Random(K * 100 + ln)
    n = 1 << ln
    for q in (False, True):
        x = [rng.randrange(-(1 << (bits - 1)), 1 << (bits - 1)) for _ in range(n)]
        y = [rng.randrange(-(1 << (bits - 1)), 1 << (bits - 1)) for _ in range(n)]
        # extreme values too: the lazy bounds must hold for every input
        x[0], x[1], y[0] = (1 << (bits - 1)) - 1, -(1 << (bits - 1)), -(1 << (bits - 1))
        for yy in (None, y):
            got = M.product(x, yy, ln, K, q)
            exp = M.exact_product(x, yy, ln, q)
            wrap = 1 << (32 * K)
            exp = [((e + wrap // 2) % wrap) - wrap // 2 for e in exp]
            assert got == exp, "K=%d ln=%d %s %s" % (K, ln, "Q" if q else "R", "square" if yy is None else "mul")


def test_row_twiddles_factor_into_row_constant_and_shared_table():
    # the twiddle of row r (of HR = 2^a rows) at row level t and index m is
    # w[(HR + r) 2^t] * beta_t[m], beta_t the row-independent domain-R table of
    # the level with 2^t polynomials (positions 2^t + m of a longer transform):
    # the structure a twisted row transform with one shared table relies on
    ln, a = 17, 5
    HR = 1 << a
    for k in (0, 5):
        p = M.TPRIMES[k]
        beta = M.tables(14, k, False)[0].astype(object)
        for q in (False, True):
            w = M.tables(ln, k, q)[0].astype(object)
            for r in (0, 3, HR - 1):
                for t in range(ln - 1 - a):
                    base = (HR + r) << t
                    for m in range(0, 1 << t, max(1, (1 << t) // 5)):
                        assert w[base + m] == w[base] * beta[(1 << t) + m] % p
