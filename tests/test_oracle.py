"""CPU tests of the oracle (C restatement of the reference transform) against
the reference's own transformCPU / transformGMP (compiled from the reference
sources when available) and against the committed golden fixtures."""
import glob
import math
import os

import numpy as np
import pytest

import annie_b200 as A
from annie_b200.synth import Xoshiro256ss
from helpers import random_N

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def coprime_N(bits, seed, oracle_mod, a=3):
    rng = Xoshiro256ss(seed)
    while True:
        N = rng.random_odd(bits)
        o = oracle_mod.Oracle(N, a, rule=1)
        if not o.init_failed():
            return N


@pytest.mark.parametrize("bits,seed", [(20000, 1), (70000, 2)])
def test_oracle_registers_equal_reference_transformCPU(oracle_mod, bits, seed, tmp_path):
    if not oracle_mod.ref_available():
        pytest.skip("reference sources not built here")
    N = coprime_N(bits, seed, oracle_mod)
    o = oracle_mod.Oracle(N, 3, rule=1)
    r = oracle_mod.RefTransform(N, 3, 0)
    o.set1(); r.set1(); o.copy(1, 0); r.copy(1, 0)
    K, n = o.K, o.n
    path = str(tmp_path / "ck.bin")
    for i, a in enumerate([3, 1, 3, 3, 1]):
        o.square_mul(a); r.square_mul(a)
        w = r.checkpoint_words(path)
        assert np.array_equal(o.read_reg(0), w[:K * n]), "Reg0 after square_mul %d" % i
    o.mul(1, 0); r.mul(1, 0)
    w = r.checkpoint_words(path)
    assert np.array_equal(o.read_reg(1), w[K * n:])
    assert o.get(0) == r.get(0) and o.get(1) == r.get(1)


@pytest.mark.parametrize("bits,rule", [(5000, 0), (30000, 0), (30000, 1), (100000, 0)])
def test_oracle_get_equals_pow_and_transformGMP(oracle_mod, bits, rule):
    rng = Xoshiro256ss(bits + rule)
    while True:
        N = rng.random_odd(bits)
        o = oracle_mod.Oracle(N, 3, rule=rule)
        if not o.init_failed():
            break
    o.set1(); o.copy(1, 0)
    e = 0
    for a in [3, 3, 1, 3, 1, 1, 3, 3, 1, 3, 1, 3]:
        o.square_mul(a)
        e = 2 * e + (a == 3)
    o.mul(1, 0)
    assert o.get(0) == pow(3, e, N) and o.get(1) == pow(3, e, N)
    if oracle_mod.ref_available():
        g = oracle_mod.RefTransform(N, 3, 1)
        if not g.init_failed():
            g.set1()
            for a in [3, 3, 1, 3, 1, 1, 3, 3, 1, 3, 1, 3]:
                g.square_mul(a)
            assert g.get(0) == o.get(0)


def test_oracle_reproduces_golden_registers(oracle_mod):
    files = sorted(glob.glob(os.path.join(GOLDEN, "regs_*.npz")))
    assert files, "golden register fixtures missing"
    for f in files:
        bits, seed = [int(x) for x in os.path.basename(f)[5:-4].replace("s", "").split("_")]
        N = random_N(bits, seed)
        d = np.load(f)
        o = oracle_mod.Oracle(N, 3, rule=1)
        o.set1(); o.copy(1, 0)
        for i, a in enumerate(d["pattern"]):
            o.square_mul(int(a))
            assert np.array_equal(o.read_reg(0), d["reg0"][i]), "%s step %d" % (f, i)
        o.mul(1, 0)
        assert np.array_equal(o.read_reg(1), d["reg1"])


def test_parameter_rules(oracle_mod):
    # factory rule (transformGPU.h:822-857) of the product equals the oracle's;
    # at K=5 the CPU rule equals the reference's own get_n_base
    rng = Xoshiro256ss(99)
    for bits in (3000, 20000, 262144, 700000, 2000020, 3000000):
        N = rng.random_odd(bits)
        assert A.probe(N, 3)[0] == oracle_mod.select_params(N, 3, 0)
    if oracle_mod.ref_available():
        import ctypes as C
        L = oracle_mod.lib_ref()
        for bits in (20000, 262144, 2000020):
            N = rng.random_odd(bits)
            K, pck, ln, lbase = oracle_mod.select_params(N, 3, 1)
            lnr, lbr = C.c_int(), C.c_int()
            # log2(16 a N) and log2(prod P / 2a) as transformCPU computes them
            # (mpz_get_d_2exp truncates N to its top 53 bits)
            top = N >> (N.bit_length() - 53)
            log2_16aN = math.log2(48.0) + math.log2(top / (1 << 53)) + N.bit_length()
            P = [(125 << 25) + 1, (243 << 24) + 1, (235 << 24) + 1, (29 << 27) + 1, (13 << 28) + 1]
            l = math.log2(P[0]) + math.log2(P[1]) + math.log2(P[2]) + math.log2(P[3]) - math.log2(6.0)
            l += math.log2(P[4])
            L.ref_cpu_get_n_base(C.byref(lnr), C.byref(lbr), 4, log2_16aN, l)
            assert (ln, lbase) == (lnr.value, lbr.value)


def test_init_failed_reports_gcd(oracle_mod):
    rng = Xoshiro256ss(5)
    while True:
        N = rng.random_odd(30000)
        if N % 3 == 0:
            break
    o = oracle_mod.Oracle(N, 3)
    assert o.init_failed()
    f = o.get_factor()
    assert f > 1 and N % f == 0 and A.probe(N, 3)[1]


def _carry_model(V, pck, lb, a, nega, K):
    """Python model of the reference carry (kernel.cl:1561-1649) on exact
    coefficient values V_i: returns the re-encoded digit values D_i."""
    mask = (1 << (32 * K)) - 1

    def wrap(x):
        x &= mask
        return x - (1 << (32 * K)) if x >> (32 * K - 1) else x
    n = len(V)
    G = n // 4
    B = 1 << (pck * lb)
    digits, cout = [0] * n, [0] * G
    for g in range(G):
        f = 0
        for j in range(4):
            f = wrap(f + V[4 * g + j] * a)
            digits[4 * g + j] = f & (B - 1)
            f >>= pck * lb
        cout[g] = f
    D = [0] * n
    for g in range(G):
        f = cout[g - 1] if g > 0 else (wrap(-cout[G - 1]) if nega else cout[G - 1])
        for j in range(3):
            f = wrap(f + digits[4 * g + j])
            low = f & (B - 1)
            top = low >> ((pck - 1) * lb)
            f >>= pck * lb
            if top >= (1 << lb) // 2:
                top -= 1 << lb
                f = wrap(f + 1)
            D[4 * g + j] = (low & ((1 << ((pck - 1) * lb)) - 1)) + top * (1 << ((pck - 1) * lb))
        f = wrap(f + digits[4 * g + 3])
        D[4 * g + 3] = f   # small: the last digit absorbs the carry
    return D


@pytest.mark.parametrize("K,ln,lbase", [(5, 6, 18), (3, 6, 22), (2, 7, 14)])
def test_oracle_carry_matches_python_model(oracle_mod, K, ln, lbase):
    pck = {2: 1, 3: 2, 4: 2, 5: 4}[K]
    P = [(125 << 25) + 1, (243 << 24) + 1, (235 << 24) + 1, (29 << 27) + 1, (13 << 28) + 1][:K]
    n = 1 << ln
    N = Xoshiro256ss(K).random_odd(64)
    o = oracle_mod.Oracle(N, 3, params=(K, pck, ln, lbase))
    M = math.prod(P)
    rng = np.random.default_rng(K + ln)
    bound = 1 << (2 * pck * lbase + ln)
    V = [int(x) for x in rng.integers(-(1 << 62), 1 << 62, size=n)]
    V = [v * (bound >> 62) // 4 for v in V]
    norm = [pow(2, -(ln - 1), p) for p in P]
    # the carry input is V in the Montgomery domain scaled by 2^(ln-1): x = V * 2^32 * 2^(ln-1)
    x = np.zeros(K * n, dtype=np.uint32)
    for k, p in enumerate(P):
        for i, v in enumerate(V):
            x[k * n + i] = (v * pow(2, 32, p) * pow(2, ln - 1, p)) % p
    for nega in (0, 1):
        got = o.carry(x, 3, nega)
        D = _carry_model(V, pck, lbase, 3, nega, K)
        for k, p in enumerate(P):
            assert all(int(got[k * n + i]) == D[i] % p for i in range(n)), (nega, k)
    assert norm  # computed for documentation of the scaling
