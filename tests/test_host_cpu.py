"""Host-side logic on CPU: the number theory and bit handling that bench.py's
Proth workload shares with the PRP driver (Jacobi symbol and Euler base,
Gerbicz-Li block size and chunk sums, exponent bit packing), and the periodic
Gerbicz-Li check with an injected error and rollback, run on an exact
integer stand-in for the transform (no GPU)."""
import math
import os
import sys
import types


ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402
from annie_b200.synth import Xoshiro256ss, proth  # noqa: E402


def test_jacobi_matches_sympy():
    from sympy import jacobi_symbol
    rng = Xoshiro256ss(3)
    for _ in range(300):
        n = rng.random_odd(rng.uniform(8, 200))
        a = rng.uniform(0, 1 << 40)
        assert bench._jacobi(a, n) == jacobi_symbol(a, n)


def test_euler_base_rule():
    # smallest a >= 2, not a square, with (a/N) = -1 (src/annie.h:249-254)
    from sympy import jacobi_symbol
    rng = Xoshiro256ss(4)
    for _ in range(50):
        N = proth(rng.uniform(3, 1 << 20) | 1, rng.uniform(100, 400))
        a = bench._euler_base(N)
        assert jacobi_symbol(a, N) == -1 and math.isqrt(a) ** 2 != a
        assert all(jacobi_symbol(b, N) != -1 or math.isqrt(b) ** 2 == b for b in range(2, a))


def test_gl_block_size():
    # B = (size - 1) / L + 1 with L = 2 << (floor(log2 size) / 2) (src/annie.h:97-101)
    for size in [2, 3, 17, 1000, 262143, 1999999, 2000020, 33219280]:
        L = 2 << ((size.bit_length() - 1) // 2)
        assert bench._gl_block(size) == (size - 1) // L + 1
    assert bench._gl_block(262144) == 256          # E = N - 1 of the 262,144-bit Fermat test


def test_chunk_sum_and_bit_packing():
    rng = Xoshiro256ss(5)
    e = rng.random_odd(3000)
    B = 37
    assert bench._chunk_sum(e, B) == sum((e >> (B * i)) & ((1 << B) - 1) for i in range(e.bit_length() // B + 1))
    top, count = 2999, 70
    w = bench._pack_bits(e, top, count)
    assert all(((w >> s) & 1) == ((e >> (top - s)) & 1) for s in range(count))
    w = bench._pack_bits(e, 5, 10)                 # runs past bit 0: missing bits read 0
    assert all(((w >> s) & 1) == (((e >> (5 - s)) & 1) if s <= 5 else 0) for s in range(10))


class _ExactTransform:
    """Registers as integers mod N: the arithmetic the CUDA transform must match."""

    def __init__(self, N, a):
        self.N, self.r = N, [1, 1, 1]
        self.ln = self.K = self.lbase = 0

    def set1(self): self.r[0] = 1
    def copy(self, d, s): self.r[d] = self.r[s]
    def mul(self, d, s): self.r[d] = self.r[d] * self.r[s] % self.N
    def get(self, i): return self.r[i]
    def save_checkpoint(self): return (self.r[0], self.r[1])
    def read_checkpoint(self, p): self.r[0], self.r[1] = p; return True
    def inject_word(self, i, index, delta=-1): self.r[i] = (self.r[i] + 1) % self.N    # one word moved
    def synchronize(self): pass
    def flush_l2(self, n): pass
    def timer_start(self): pass
    def timer_stop(self): return 1.0

    def square_mul_bits(self, bits, count, a):
        for i in range(count):
            self.r[0] = self.r[0] * self.r[0] * (a if (bits >> i) & 1 else 1) % self.N


def test_periodic_gerbicz_li_check_detects_and_rolls_back(monkeypatch):
    import annie_b200 as A
    monkeypatch.setattr(A, "Transform", _ExactTransform)
    monkeypatch.setattr(A, "probe", lambda N, a, **kw: ((5, 4, 10, 17), False))
    args = types.SimpleNamespace(proth_n=3000, proth_squarings=700, warmup=1)
    res = bench.run_proth2m_workload(args)
    assert res["gl_check"]["passed"]
    assert res["injected_error"]["detected"] and res["injected_error"]["rolled_back_and_verified"]


def test_issue_bound_of_the_bench_line():
    # the bench's issue bound: warp instructions / (SMs x 4 schedulers x clock)
    names = ["a", "b", "c", "r0", "r1", "r2", "r3", "r4", "r5"]
    per = [0.01, 0.02, 0.02, 0.03, 0.03, 0.03, 0.03, 0.03, 0.04]
    instr = {nm: 1_000_000 for nm in names[3:]}
    out = bench.issue_bound(names, per, 8, instr, 200.0, 100, 1000.0)
    rate = 100 * 4 * 1000.0e6
    assert out["dominant"]["bound_us"] == round(1e6 / rate * 1e6, 2)
    assert out["critical_path"]["warp_instructions"] == 6_000_000
    assert out["critical_path"]["frac_of_squaring"] == round(6e6 / rate / 200e-6, 3)
    assert bench.issue_bound(names, per, 8, {"r0": 1}, 200.0, 100, 1000.0) is None
