"""Shared helpers for the tests: seeded N, random normal-form registers."""
import numpy as np

import annie_b200 as A
from annie_b200.synth import Xoshiro256ss

PRIMES = [(125 << 25) + 1, (243 << 24) + 1, (235 << 24) + 1, (29 << 27) + 1, (13 << 28) + 1]


def pick_N(bits, seed, a=3, rule_cpu_too=False, oracle=None):
    """Random odd N (top bit set) with gcd(N, R) = 1 for the factory rule
    (and for transformCPU's rule when rule_cpu_too)."""
    rng = Xoshiro256ss(seed)
    for _ in range(100):
        N = rng.random_odd(bits)
        params, failed = A.probe(N, a)
        if failed:
            continue
        if rule_cpu_too:
            cp = oracle.select_params(N, a, 1)
            _, f2 = A.probe(N, a, forced=cp)
            if f2:
                continue
        return N
    raise RuntimeError("no N found")


def random_digits_register(K, pck, ln, lbase, seed, with_exact=False):
    """Normal-form register of random digits: coefficient i holds the residues
    of D_i = sum_l d_l 2^(l lbase), d_l uniform in [0, 2^lbase) (and, with
    with_exact, the D_i)."""
    rng = np.random.default_rng(seed)
    n = 1 << ln
    d = [rng.integers(0, 1 << lbase, size=n, dtype=np.uint64) for _ in range(pck)]
    v = np.zeros(n, dtype=object)
    for l in reversed(range(pck)):
        v = v * (1 << lbase) + d[l].astype(object)
    out = np.zeros(K * n, dtype=np.uint32)
    for k in range(K):
        out[k * n:(k + 1) * n] = np.array([int(x) % PRIMES[k] for x in v], dtype=np.uint32)
    return (out, list(v)) if with_exact else out


def random_residues(K, ln, seed):
    rng = np.random.default_rng(seed)
    n = 1 << ln
    return np.concatenate([rng.integers(0, PRIMES[k], size=n, dtype=np.uint64).astype(np.uint32) for k in range(K)])


SMALL_PRIMES = [p for p in range(3, 2000) if all(p % q for q in range(2, int(p ** 0.5) + 1))]


def coprime_to_small(N):
    return all(N % p for p in SMALL_PRIMES)


def random_N(bits, seed):
    """First draw of the seeded generator with no prime factor below 2000
    (the rule of tests/golden/make_golden.py)."""
    rng = Xoshiro256ss(seed)
    while True:
        N = rng.random_odd(bits)
        if coprime_to_small(N):
            return N


def proth_N(n, seed):
    """k*2^n + 1 with k odd in [2^19, 2^20) from the seeded generator, no prime factor below 2000."""
    from annie_b200.synth import proth
    rng = Xoshiro256ss(seed)
    while True:
        k = rng.uniform(1 << 19, 1 << 20) | 1
        N = proth(k, n)
        if coprime_to_small(N):
            return k, N
