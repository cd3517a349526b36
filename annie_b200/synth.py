"""Seeded synthetic inputs: xoshiro256** (Blackman & Vigna) seeded by splitmix64.

Random odd b-bit N: b bits drawn little-endian from the generator, then the
top bit and bit 0 are set.  Proth numbers k*2^n + 1 use k odd drawn from the
same generator.
"""

MASK64 = (1 << 64) - 1


def splitmix64(state):
    state = (state + 0x9E3779B97F4A7C15) & MASK64
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
    return state, z ^ (z >> 31)


def _rotl(x, k):
    return ((x << k) | (x >> (64 - k))) & MASK64


class Xoshiro256ss:
    def __init__(self, seed):
        st = seed & MASK64
        self.s = []
        for _ in range(4):
            st, z = splitmix64(st)
            self.s.append(z)

    def next(self):
        s = self.s
        result = (_rotl((s[1] * 5) & MASK64, 7) * 9) & MASK64
        t = (s[1] << 17) & MASK64
        s[2] ^= s[0]
        s[3] ^= s[1]
        s[1] ^= s[2]
        s[0] ^= s[3]
        s[2] ^= t
        s[3] = _rotl(s[3], 45)
        return result

    def uniform(self, lo, hi):
        """Uniform integer in [lo, hi) (rejection sampling on 64-bit draws)."""
        span = hi - lo
        lim = (1 << 64) - ((1 << 64) % span)
        while True:
            x = self.next()
            if x < lim:
                return lo + x % span

    def random_odd(self, bits):
        words = (bits + 63) // 64
        buf = bytearray(8 * words)
        for i in range(words):
            buf[8 * i:8 * i + 8] = self.next().to_bytes(8, "little")
        x = int.from_bytes(bytes(buf), "little")
        x &= (1 << bits) - 1
        return x | (1 << (bits - 1)) | 1

    def random(self):
        return (self.next() >> 11) * (1.0 / (1 << 53))


def random_odd(bits, seed):
    return Xoshiro256ss(seed).random_odd(bits)


def proth(k, n):
    return k * (1 << n) + 1


def jacobi(a, n):
    """Jacobi symbol (a/n), n odd positive."""
    a %= n
    r = 1
    while a:
        while a % 2 == 0:
            a //= 2
            if n % 8 in (3, 5):
                r = -r
        a, n = n, a
        if a % 4 == 3 and n % 4 == 3:
            r = -r
        a %= n
    return r if n == 1 else 0


def euler_base(N):
    """Smallest non-square a >= 2 with (a/N) = -1: the Euler-test base rule of the
    reference driver (src/annie.h:250-253)."""
    import math
    a = 2
    while jacobi(a, N) != -1:
        a += 1
        s = math.isqrt(a)
        if s * s == a:
            a += 1
    return a


# The workloads the benchmarks and the parity tests share.
FERMAT_33M_BITS, FERMAT_33M_SEED = 33219281, 2


def fermat_33m():
    """The 33,219,281-bit random odd N (about 10 M digits) tested with base 3."""
    return random_odd(FERMAT_33M_BITS, FERMAT_33M_SEED)


def proth_2m(n=2000000, seed=11, usable=None):
    """Proth number k*2^n + 1, k odd in [2^19, 2^20) drawn from seed `seed`, and its
    Euler base; `usable(N, a)` (optional) rejects draws, e.g. those whose N shares
    a factor with the transform's R."""
    rng = Xoshiro256ss(seed)
    while True:
        k = rng.uniform(1 << 19, 1 << 20) | 1
        N = proth(k, n)
        a = euler_base(N)
        if usable is None or usable(N, a):
            return k, N, a
