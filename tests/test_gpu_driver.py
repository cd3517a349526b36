"""GPU tests of the PRP driver and of the engine against the reference's own
results (golden fixtures made by tests/golden/make_golden.py from the
reference driver and transformCPU), the reference's Fibonacci known answers,
periodic Gerbicz-Li checking with an injected fault, and checkpoint
abort/resume."""
import glob
import json
import os
import threading
import time

import numpy as np
import pytest

import annie_b200 as A
from helpers import proth_N, random_N

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def _vectors():
    path = os.path.join(GOLDEN, "prp_vectors.json")
    with open(path) as f:
        return json.load(f)


def _N_of(v):
    if v["form"] == "random_odd":
        return random_N(v["bits"], v["seed"])
    k, N = proth_N(v["n"], v["seed"])
    assert k == v["k"]
    return N


@pytest.mark.parametrize("v", _vectors(), ids=lambda v: "%s-%s" % (v["form"], v.get("bits", v.get("n"))))
def test_prp_matches_reference_driver(v):
    N = _N_of(v)
    r = A.prp_check(N, euler=bool(v["euler"]), base=v["base"], gl_check_blocks=4)
    assert r["status"] == v["status"] == 0, r["message"]
    assert bool(r["is_prp"]) == v["is_prp"]
    if v["res64"] is not None:
        assert "%016X" % r["res64"] == v["res64"], r["message"]
    assert r["gl_failures"] == 0


def test_engine_registers_equal_reference_golden(oracle_mod):
    for f in sorted(glob.glob(os.path.join(GOLDEN, "regs_*.npz"))):
        bits, seed = [int(x) for x in os.path.basename(f)[5:-4].replace("s", "").split("_")]
        N = random_N(bits, seed)
        d = np.load(f)
        params = oracle_mod.select_params(N, 3, 1)       # transformCPU's parameter rule
        t = A.Transform(N, 3, params=params)
        t.set1()
        t.copy(1, 0)
        for i, a in enumerate(d["pattern"]):
            t.square_mul(int(a))
            assert np.array_equal(t.read_register(0), d["reg0"][i]), "%s: Reg0 after step %d" % (f, i)
        t.mul(1, 0)
        assert np.array_equal(t.read_register(1), d["reg1"])


def _fib(n):
    a, b = 0, 1
    for bit in bin(n)[2:]:
        a, b = a * (2 * b - a), a * a + b * b
        if bit == "1":
            a, b = b, a + b
    return a


# Fibonacci probable primes the reference's QUICK_TEST checks (src/main.cpp:163):
# each must be reported a Fermat probable prime to base 2.
@pytest.mark.parametrize("index", [25561, 35999, 81839, 148091])
def test_fibonacci_known_answers(index):
    r = A.prp_check(_fib(index))
    assert r["status"] == 0 and r["is_prp"] == 1, r["message"]
    assert r["base"] == 2


def test_injected_fault_is_detected_and_rolled_back():
    N = random_N(100000, 3)
    clean = A.prp_check(N, base=3, gl_check_blocks=2)
    assert clean["status"] == 0 and clean["gl_checks"] > 0 and clean["rollbacks"] == 0
    bad = A.prp_check(N, base=3, gl_check_blocks=2, inject_iteration=N.bit_length() // 2, inject_word=12345)
    assert bad["status"] == 0, bad["message"]
    assert bad["gl_failures"] >= 1 and bad["rollbacks"] >= 1
    assert bad["res64"] == clean["res64"] and bad["is_prp"] == clean["is_prp"]


def test_fault_without_periodic_check_fails_final_validation():
    N = random_N(60000, 2)
    r = A.prp_check(N, base=3, gl_check_blocks=0, inject_iteration=N.bit_length() // 3, inject_word=7)
    assert r["status"] == 1 and "Validation failed" in r["message"]


def test_euler_proth_with_fault_rollback():
    k, N = proth_N(200000, 31)
    clean = A.prp_check(N, euler=True, gl_check_blocks=8)
    bad = A.prp_check(N, euler=True, gl_check_blocks=8, inject_iteration=150000, inject_word=99)
    assert clean["status"] == 0 and bad["status"] == 0
    assert bad["rollbacks"] >= 1
    assert (bad["res64"], bad["is_prp"]) == (clean["res64"], clean["is_prp"])
    # Euler base: smallest non-square a with Jacobi(a, N) = -1 (annie.h:250-253)
    from sympy import jacobi_symbol
    a = clean["base"]
    assert jacobi_symbol(a, N) == -1
    assert all(jacobi_symbol(b, N) != -1 or int(b ** 0.5) ** 2 == b for b in range(2, a))


def test_checkpoint_abort_and_resume(tmp_path):
    N = random_N(262144, 4)
    ref = A.prp_check(N, base=3)
    path = str(tmp_path / "a.chk")
    A.lib().ab_prp_reset_quit()
    box = {}
    th = threading.Thread(target=lambda: box.update(A.prp_check(N, base=3, checkpoint_path=path, checkpoint_seconds=0.2)))
    th.start()
    time.sleep(2.0)
    A.lib().ab_prp_quit()
    th.join()
    A.lib().ab_prp_reset_quit()
    if box["status"] == 0:
        pytest.skip("test finished before the abort request")
    assert box["status"] == 2
    assert os.path.exists(path)
    res = A.prp_check(N, base=3, checkpoint_path=path)
    assert res["resumed"] == 1 and res["status"] == 0
    assert res["res64"] == ref["res64"] and res["is_prp"] == ref["is_prp"]
    assert not os.path.exists(path)      # cleared on completion (annie.h:428)


def test_bench_table_rows_validate():
    # the reference's -h mode (src/annie.h:432-556) on its first sizes: the
    # Gerbicz-Li check of the 6^50 exponentiation holds on each transform
    rows = A.bench_table(A.BENCH_TABLE_E[:4], seconds=0.2)
    assert len(rows) == 4
    for r in rows:
        assert r["validated"] == 1, r
        assert r["squarings"] > 0 and r["ms_per_bit"] > 0
        N = 3 * (1 << r["e"]) + 1
        assert (r["K"], r["pck"], r["ln"], r["lbase"]) == A.probe(N, 3)[0]
