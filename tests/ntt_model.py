"""Bit-exact numpy model of the engine's own transform arithmetic (not the
reference's): the transform primes, the Shoup twiddle tables, the lazily
reduced butterflies, the Montgomery pointwise product and the CRT with its
fixed-point quotient estimate, level by level.  Every element goes through the
same operations in the same order as in the CUDA passes (only the grouping of
butterflies into passes differs), so the model reproduces the device's lazy
words; it is the reference for the forward-transform kernel test and, on the
CPU, checks the design against exact big-integer convolutions.
"""
import numpy as np

TPRIMES = [119 * (1 << 23) + 1, 107 * (1 << 23) + 1, 105 * (1 << 23) + 1,
           90 * (1 << 23) + 1, 77 * (1 << 23) + 1, 71 * (1 << 23) + 1]
TGEN = [3, 3, 26, 11, 3, 3]
U32 = np.uint32
M32 = (1 << 32) - 1


def bitrev(i, s):
    r = 0
    while s > 1:
        r = 2 * r | (i & 1)
        i >>= 1
        s >>= 1
    return r


def shoup_const(w, p):
    return (w << 32) // p


def _bitrev_array(s):
    """bitrev(j, s) for j < s (s a power of two)."""
    j = np.arange(s, dtype=np.int64)
    r = np.zeros(s, dtype=np.int64)
    b = s.bit_length() - 1
    for i in range(b):
        r |= ((j >> i) & 1) << (b - 1 - i)
    return r


def _powers(x, s, p):
    """x^j mod p for j < s (numpy, p < 2^30)."""
    out = np.ones(s, dtype=np.uint64)
    j = np.arange(s, dtype=np.int64)
    sq = np.uint64(x % p)
    for i in range(max(1, s.bit_length())):
        sel = ((j >> i) & 1) == 1
        out[sel] = out[sel] * sq % np.uint64(p)
        sq = sq * sq % np.uint64(p)
    return out


def tables(ln, k, domain_q):
    """(w, ws), and for domain R (wi, wis) = -w^-1, at positions s + bitrev(j, s)."""
    p, g = TPRIMES[k], TGEN[k]
    n = 1 << ln
    w = np.zeros(n // 2, dtype=np.uint64)
    wi = np.zeros(n // 2, dtype=np.uint64)
    lvl = ln - 1
    s = n // 4
    while s >= 1:
        rho = pow(g, (p - 1) >> lvl, p)
        rhoi = pow(rho, p - 2, p)
        t0 = pow(g, (p - 1) >> (lvl + 1), p) if domain_q else 1
        pos = s + _bitrev_array(s)
        w[pos] = _powers(rho, s, p) * np.uint64(t0) % np.uint64(p)
        wi[pos] = (np.uint64(p) - _powers(rhoi, s, p)) % np.uint64(p)
        s //= 2
        lvl -= 1
    ws = (w << np.uint64(32)) // np.uint64(p)
    wis = (wi << np.uint64(32)) // np.uint64(p)
    if domain_q:
        return w, ws, None, None
    return w, ws, wi, wis


def _u(x):
    return (np.asarray(x, dtype=np.uint64) & np.uint64(M32))


def shoup(x, w, ws, p):
    x = _u(x)
    q = (x * _u(ws)) >> np.uint64(32)
    return _u(x * _u(w) - q * np.uint64(p))


def mont(a, b, p):
    pinv = pow(p, -1, 1 << 32)
    t = _u(a) * _u(b)
    lo, hi = t & np.uint64(M32), t >> np.uint64(32)
    m = _u(lo * np.uint64(pinv))
    return _u(hi - ((m * np.uint64(p)) >> np.uint64(32)) + np.uint64(p))


def red2(x, p):
    x = _u(x)
    y = _u(x - np.uint64(2 * p))
    return np.minimum(x, y)


def exact_limbs(exact):
    """Three 32-bit limbs (two's complement, 96 bits) of python-int exact values."""
    d = [int(v) & ((1 << 96) - 1) for v in exact]
    d0 = np.array([x & M32 for x in d], dtype=np.uint64)
    d1 = np.array([(x >> 32) & M32 for x in d], dtype=np.uint64)
    d2 = np.array([(x >> 64) & M32 for x in d], dtype=np.uint64)
    return d0, d1, d2


def encode(exact, k, limbs=None):
    """Residues in [0, 3p) of exact values (python ints, |v| < 2^95), as the column pass."""
    p = TPRIMES[k]
    d0, d1, d2 = exact_limbs(exact) if limbs is None else limbs
    d2u = d2 ^ np.uint64(0x80000000)
    one_s = (1 << 32) // p
    a = _u(d0 - ((d0 * np.uint64(one_s)) >> np.uint64(32)) * np.uint64(p))
    c32 = (1 << 32) % p
    c64 = c32 * c32 % p
    b = shoup(d1, c32, shoup_const(c32, p), p)
    e = shoup(d2u, c64, shoup_const(c64, p), p)
    s = red2(a + b, p)
    s = red2(s + e, p)
    k95 = (p - (c64 * ((1 << 31) % p)) % p) % p
    return _u(s + np.uint64(k95))


def forward(x, ln, k, domain_q, reduce_out=False):
    """All ln-1 forward levels (index bit ln-1-l at level l), lazy [0, 4p)."""
    p = TPRIMES[k]
    w, ws, _, _ = tables(ln, k, domain_q)
    x = _u(x).copy()
    n = 1 << ln
    for l in range(ln - 1):
        half = n >> (l + 1)
        i = np.arange(n)
        i0 = i[(i & half) == 0]
        i1 = i0 + half
        j = i0 >> (ln - l)
        tw, tws = w[(1 << l) + j], ws[(1 << l) + j]
        a = red2(x[i0], p)
        t = shoup(x[i1], tw, tws, p)
        x[i0] = _u(a + t)
        x[i1] = _u(a - t + np.uint64(2 * p))
    return red2(x, p) if reduce_out else x


def pointwise(x, ln, k, domain_q, y=None):
    """Degree-1 products mod (x^2 -+ c), c = w[n/4 + m/2] (Montgomery, outputs [0, 2p))."""
    p = TPRIMES[k]
    w, ws, _, _ = tables(ln, k, domain_q)
    n = 1 << ln
    m = np.arange(n // 2)
    c, cs = w[n // 4 + (m >> 1)], ws[n // 4 + (m >> 1)]
    x0, x1 = red2(x[0::2], p), red2(x[1::2], p)
    if y is None:
        t = shoup(mont(x1, x1, p), c, cs, p)
        y1 = mont(red2(x0 + x0, p), x1, p)
        y0 = mont(x0, x0, p)
    else:
        p0, p1 = _u(y[0::2]), _u(y[1::2])
        t = shoup(mont(x1, p1, p), c, cs, p)
        y1 = red2(mont(x0, p1, p) + mont(x1, p0, p), p)
        y0 = mont(x0, p0, p)
    y0 = np.where((m & 1) == 0, red2(y0 + t, p), red2(y0 - t + np.uint64(2 * p), p))
    out = np.empty(n, dtype=np.uint64)
    out[0::2], out[1::2] = y0, y1
    return out


def inverse(x, ln, k, domain_q):
    """All inverse levels, with -w^-1 (R: its table; Q: w at the mirrored position)."""
    p = TPRIMES[k]
    w, ws, wi, wis = tables(ln, k, domain_q)
    x = _u(x).copy()
    n = 1 << ln
    for l in reversed(range(ln - 1)):
        half = n >> (l + 1)
        i = np.arange(n)
        i0 = i[(i & half) == 0]
        i1 = i0 + half
        j = i0 >> (ln - l)
        idx = (1 << l) + j
        if domain_q:
            mi = 3 * (1 << l) - 1 - idx
            v, vs = w[mi], ws[mi]
        else:
            v, vs = wi[idx], wis[idx]
        s = _u(x[i0] + x[i1])
        d = _u(x[i1] - x[i0] + np.uint64(2 * p))
        x[i0] = red2(s, p)
        x[i1] = shoup(d, v, vs, p)
    return x


def crt(res, ln, K):
    """Exact signed values from the K+1 planes (each [0, 2p), holding (n/2) 2^-32 V)."""
    KP = K + 1
    M = 1
    for p in TPRIMES[:KP]:
        M *= p
    n = 1 << ln
    L = 32 * K
    out = []
    ys = []
    for k in range(KP):
        p = TPRIMES[k]
        Mk = M // p
        c = pow(n // 2, -1, p) * ((1 << 32) % p) % p * pow(Mk % p, -1, p) % p
        y = shoup(res[k], c, shoup_const(c, p), p)
        ys.append(np.where(y >= p, y - np.uint64(p), y))
    fl = [(1 << 60) // p for p in TPRIMES[:KP]]
    for i in range(len(ys[0])):
        est = sum(int(ys[k][i]) * fl[k] for k in range(KP)) & ((1 << 64) - 1)
        t = (est + (1 << 59)) >> 60
        v = (sum(int(ys[k][i]) * (M // TPRIMES[k]) for k in range(KP)) - t * M) % (1 << L)
        if v >> (L - 1):
            v -= 1 << L
        out.append(v)
    return out


def product(xe, ye, ln, K, domain_q):
    """Exact coefficients of x*y mod (x^n -+ 1) (ye None: x^2) through the model."""
    res = []
    for k in range(K + 1):
        fx = forward(encode(xe, k), ln, k, domain_q)
        fy = None if ye is None else forward(encode(ye, k), ln, k, domain_q, reduce_out=True)
        res.append(inverse(pointwise(fx, ln, k, domain_q, fy), ln, k, domain_q))
    return crt(res, ln, K)


def exact_product(xe, ye, ln, domain_q):
    """Cyclic (R) or negacyclic (Q) convolution with python ints."""
    n = 1 << ln
    ye = xe if ye is None else ye
    out = [0] * n
    for i in range(n):
        xi = int(xe[i])
        if xi == 0:
            continue
        for j in range(n):
            t = i + j
            if t >= n:
                t -= n
                out[t] += -xi * int(ye[j]) if domain_q else xi * int(ye[j])
            else:
                out[t] += xi * int(ye[j])
    return out
