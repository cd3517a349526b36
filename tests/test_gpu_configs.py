"""Parity on the exact numbers the benchmarks time, and determinism of the schedule.

* The 33,219,281-bit Fermat number (base 3) and the Proth number k*2^2000000+1
  (Euler base) are the benchmark workloads.  After a window of test-loop
  iterations from set1 and the Gerbicz-Li product Reg1 *= Reg0, the raw
  register words of Reg0 and Reg1 must equal those of the reference's own
  transformCPU (src/transformCPU.h, compiled from the reference sources) on
  the same N -- the factory and transformCPU choose the same K, n and digit
  size at both sizes.  Where the reference is not built, the oracle (the C
  restatement) is the checker.
* The registers after 512 squarings do not depend on the schedule: the
  overlapped two-stream schedule, a single stream, every row/column split,
  and repeated runs all give the same words.
"""
import os
import tempfile

import numpy as np
import pytest

import annie_b200 as A
from annie_b200.synth import fermat_33m, proth_2m
from helpers import pick_N

pytestmark = pytest.mark.gpu


def _checker(oracle_mod, N, a, params):
    """(square_mul, mul, registers) of the reference transformCPU, or of the oracle."""
    if oracle_mod.ref_available():
        r = oracle_mod.RefTransform(N, a, 0)
        assert not r.init_failed()
        fd, path = tempfile.mkstemp()
        os.close(fd)

        def regs():
            w = r.checkpoint_words(path)
            return w

        return r, regs, path
    o = oracle_mod.Oracle(N, a, params=params)
    return o, (lambda: np.concatenate([o.read_reg(0), o.read_reg(1)])), None


def _window(oracle_mod, N, a, E, count):
    t = A.Transform(N, a)
    assert not t.init_failed()
    params = (t.K, t.pck, t.ln, t.lbase)
    ref, regs, path = _checker(oracle_mod, N, a, params)
    try:
        top = E.bit_length() - 1
        mults = [a if (E >> (top - i)) & 1 else 1 for i in range(count)]
        for x in (t, ref):
            x.set1()
            x.copy(1, 0)
        for m in mults:
            t.square_mul(m)
        if hasattr(ref, "square_mul_seq"):
            ref.square_mul_seq(mults)
        else:
            for m in mults:
                ref.square_mul(m)
        t.mul(1, 0)
        ref.mul(1, 0)
        w = np.asarray(regs(), dtype=np.uint32)
        K, n = t.K, t.n
        assert len(w) >= 2 * K * n
        got0, got1 = t.read_register(0), t.read_register(1)
        d0 = int(np.count_nonzero(got0 != w[:K * n]))
        d1 = int(np.count_nonzero(got1 != w[K * n:2 * K * n]))
        assert d0 == 0 and d1 == 0, "Reg0: %d words differ, Reg1: %d words differ" % (d0, d1)
        return t, params
    finally:
        if path:
            os.unlink(path)


def test_fermat_33m_window_equals_reference(oracle_mod):
    N = fermat_33m()
    t, params = _window(oracle_mod, N, 3, N - 1, 8)
    assert params == (5, 4, 19, 17)


def test_proth_2m_window_equals_reference(oracle_mod):
    k, N, a = proth_2m(usable=lambda N, a: not A.probe(N, a)[1])
    t, params = _window(oracle_mod, N, a, (N - 1) >> 1, 64)
    assert params == (5, 4, 15, 17)


@pytest.mark.parametrize("bits", [500000, 2000000, 8000000])
def test_registers_do_not_depend_on_the_schedule(bits):
    N = pick_N(bits, seed=bits + 1)
    t = A.Transform(N, 3)
    t.set1()
    t.copy(1, 0)
    t.square_mul_bits(0x5A5A5A5A5A5A5A5A, 64, 3)
    start = t.save_checkpoint()
    bits_word = (0x3C3C3C3C3C3C3C3C << 64) | 0x0F0F0F0F0F0F0F0F
    pattern = bits_word | (bits_word << 128) | (bits_word << 256) | (bits_word << 384)

    def run():
        assert t.read_checkpoint(start)
        t.square_mul_bits(pattern, 512, 3)
        t.mul(1, 0)
        return np.concatenate([t.read_register(0), t.read_register(1)])

    ref = run()
    default_split = t.geometry()[0]
    L = t.ln - 1
    for overlap in (True, False):
        t.set_overlap(overlap)
        for lb in range(max(4, L - 6), min(13, L - 1) + 1):
            t.set_geometry(lb)
            for rep in range(3):
                got = run()
                assert np.array_equal(got, ref), "overlap=%s row levels %d repeat %d: %d words differ" % (
                    overlap, lb, rep, int(np.count_nonzero(got != ref)))
    t.set_overlap(True)
    t.set_geometry(default_split)
    for rep in range(10):
        assert np.array_equal(run(), ref), "repeat %d" % rep


def test_multiplier_below_one_is_rejected():
    N = pick_N(20000, seed=3)
    t = A.Transform(N, 3)
    t.set1()
    for a in (0, -3):
        with pytest.raises(A.EngineError) as e:
            t.square_mul(a)
        assert e.value.code == A.AB_E_ARG


def test_noalloc_multiplier_below_one_is_rejected():
    import torch
    N = pick_N(20000, seed=3)
    t = A.Transform(N, 3)
    dev = torch.zeros(t.K * t.n, dtype=torch.int32, device="cuda:0")
    with pytest.raises(A.EngineError) as e:
        t.square_mul_noalloc(dev.data_ptr(), 0)
    assert e.value.code == A.AB_E_ARG
