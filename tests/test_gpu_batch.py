"""GPU tests of batches (many candidates squared together from a captured
CUDA graph) and of the continuous-batching runner: every candidate's result
must be the same in the mix as alone, bit for bit."""
import json
import os

import numpy as np
import pytest

import annie_b200 as A
from annie_b200.synth import Xoshiro256ss
from helpers import proth_N, random_N

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _same_class_numbers(cls, count, lo, hi, seed):
    rng = Xoshiro256ss(seed)
    out = []
    while len(out) < count:
        bits = rng.uniform(lo, hi)
        N = rng.random_odd(bits)
        p, failed = A.probe(N, 3)
        if not failed and p[:3] == cls:
            out.append((N, p))
    return out


def test_batch_slots_equal_single_transforms():
    cls = (5, 4, 12)
    nums = _same_class_numbers(cls, 5, 200000, 280000, 1)
    assert len({p[3] for _, p in nums}) >= 1
    b = A.Batch(cls + (0,), capacity=6, max_steps=16)
    singles = []
    for s, (N, p) in enumerate(nums):
        assert not b.load(s, N, 3)
        v = b.slot(s)
        v.set1(); v.copy(1, 0)
        t = A.Transform(N, 3)
        t.set1(); t.copy(1, 0)
        singles.append(t)
    rng = np.random.default_rng(7)
    for rnd in range(3):
        steps = 16
        mult = rng.choice([1, 3], size=(steps, 6)).astype(np.uint32)
        mult[:, 5] = 0                      # slot 5 is empty
        mult[steps - 3:, 2] = 0             # slot 2 sits the last steps out
        snap = np.zeros((steps, 6), dtype=np.uint8)
        snap[5, 1] = 1
        b.steps(mult, snap)
        b.gl_mul(1)
        for s, t in enumerate(singles):
            for i in range(steps):
                if mult[i, s]:
                    t.square_mul(int(mult[i, s]))
                    if s == 1 and i == 5:
                        t.copy(2, 0)
            if s == 1:
                t.mul(1, 2)
        for s, t in enumerate(singles):
            v = b.slot(s)
            assert np.array_equal(v.read_register(0), t.read_register(0)), "slot %d Reg0, round %d" % (s, rnd)
            assert np.array_equal(v.read_register(1), t.read_register(1)), "slot %d Reg1, round %d" % (s, rnd)
    for s, t in enumerate(singles):
        assert b.slot(s).get(0) == t.get(0)


def _run_all(runner, limit=200000):
    results = {}
    for _ in range(limit):
        active, queued = runner.advance()
        for tag, r in runner.poll():
            results[tag] = r
        if active == 0 and queued == 0:
            break
    for tag, r in runner.poll():
        results[tag] = r
    return results


@pytest.mark.parametrize("latency_ln", [0, 10])
def test_runner_matches_reference_golden_and_solo(latency_ln):
    # latency_ln 10: the smaller classes and the larger ones take turns (1 ms epochs)
    with open(os.path.join(HERE, "golden", "prp_vectors.json")) as f:
        vec = [v for v in json.load(f) if not v.get("big")]
    jobs = {}
    for tag, v in enumerate(vec):
        N = random_N(v["bits"], v["seed"]) if v["form"] == "random_odd" else proth_N(v["n"], v["seed"])[1]
        jobs[tag] = (N, v)
    r = A.Runner(chunk=32, max_slots_per_class=8, latency_ln=latency_ln, epoch_us=1000)
    if latency_ln:
        lns = {A.probe(N, v["base"] or 2)[0][2] for N, v in jobs.values()}
        assert min(lns) <= latency_ln < max(lns)                 # both groups present
    for tag, (N, v) in jobs.items():
        r.submit(N, euler=bool(v["euler"]), base=v["base"], tag=tag)
    res = _run_all(r)
    assert set(res) == set(jobs)
    for tag, (N, v) in jobs.items():
        got = res[tag]
        assert got["status"] == 0, got["message"]
        assert bool(got["is_prp"]) == v["is_prp"]
        if v["res64"] is not None:
            assert "%016X" % got["res64"] == v["res64"]
        solo = A.prp_check(N, euler=bool(v["euler"]), base=v["base"])
        assert (solo["res64"], solo["is_prp"]) == (got["res64"], got["is_prp"])


def test_runner_periodic_check_detects_and_rolls_back():
    # every test checked every 2 Gerbicz-Li blocks; one test gets a word of
    # Reg0 changed mid-run: its next check fails, it rolls back to the last
    # verified state and still ends with the reference's RES64
    with open(os.path.join(HERE, "golden", "prp_vectors.json")) as f:
        vec = [v for v in json.load(f) if not v.get("big")]
    jobs = {}
    for tag, v in enumerate(vec):
        N = random_N(v["bits"], v["seed"]) if v["form"] == "random_odd" else proth_N(v["n"], v["seed"])[1]
        jobs[tag] = (N, v)
    victim = max(jobs, key=lambda t: jobs[t][0].bit_length())
    bits = jobs[victim][0].bit_length()
    r = A.Runner(chunk=32, max_slots_per_class=8, gl_check_blocks=2, inject_tag=victim, inject_bit=bits // 2, inject_word=777)
    for tag, (N, v) in jobs.items():
        r.submit(N, euler=bool(v["euler"]), base=v["base"], tag=tag)
    res = _run_all(r)
    assert set(res) == set(jobs)
    for tag, (N, v) in jobs.items():
        got = res[tag]
        assert got["status"] == 0, got["message"]
        assert got["gl_checks"] > 0
        if v["res64"] is not None:
            assert "%016X" % got["res64"] == v["res64"]
    assert res[victim]["gl_failures"] >= 1 and res[victim]["rollbacks"] >= 1
    assert all(res[t]["gl_failures"] == 0 for t in jobs if t != victim)


def test_runner_continuous_admission_under_budget():
    # room for 2 slots of the class at a time: the rest wait and are admitted as slots free up
    nums = _same_class_numbers((5, 4, 10), 5, 50000, 70000, 3)
    per = A.lib().ab_batch_slot_bytes(A.Params(5, 4, 10, 0))
    r = A.Runner(chunk=64, max_slots_per_class=2, hbm_budget_bytes=2 * per)
    for tag, (N, p) in enumerate(nums):
        r.submit(N, base=3, tag=tag)
    a, q = r.advance()
    assert a == 2 and q == 3
    res = _run_all(r)
    assert len(res) == 5
    for tag, (N, p) in enumerate(nums):
        solo = A.prp_check(N, base=3)
        assert res[tag]["res64"] == solo["res64"] and res[tag]["status"] == 0


def test_runner_decides_trivial_cases():
    r = A.Runner(chunk=16)
    r.submit(1000003, tag=1)              # <= 15 digits: GMP decides (annie.h:222-237)
    r.submit((1 << 4000) + 2, tag=2)      # even
    res = _run_all(r, limit=10)
    assert res[1]["decided_early"] == 1 and res[1]["is_prp"] == 1
    assert res[2]["decided_early"] == 1 and "even" in res[2]["message"]


def test_autotune_keeps_loaded_slots_and_results():
    cls = (5, 4, 12)
    nums = _same_class_numbers(cls, 3, 200000, 280000, 6)
    b = A.Batch(cls + (0,), capacity=4, max_steps=8)
    singles = []

    def load(s, N):
        assert not b.load(s, N, 3)
        v = b.slot(s)
        v.set1(); v.copy(1, 0)
        v.square_mul(3)
        t = A.Transform(N, 3)
        t.set1(); t.copy(1, 0); t.square_mul(3)
        singles.append(t)

    for s in range(2):
        load(s, nums[s][0])
    before = [b.slot(s).read_register(0) for s in range(2)]
    lb = b.autotune(0, 8)
    L = cls[2] - 1
    assert 4 <= lb <= min(13, L - 1) and L - lb <= 6
    assert b.slot(2) is None and b.slot(3) is None          # the copies are gone
    for s in range(2):
        assert np.array_equal(b.slot(s).read_register(0), before[s])
    load(2, nums[2][0])                                     # a slot loaded under the tuned split
    mult = np.array([[3, 1, 3, 0]] * 8, dtype=np.uint32)
    b.steps(mult)
    for s, t in enumerate(singles):
        for i in range(8):
            t.square_mul(int(mult[i, s]))
        assert np.array_equal(b.slot(s).read_register(0), t.read_register(0)), "slot %d" % s
    b.slot(2).mul(1, 0); singles[2].mul(1, 0)
    assert b.slot(2).get(1) == singles[2].get(1)
    assert b.autotune(1, 8) == lb                           # remembered for the class


def test_load_many_equals_single_loads():
    cls = (5, 4, 12)
    nums = _same_class_numbers(cls, 3, 200000, 280000, 9)
    rng = Xoshiro256ss(10)
    while True:                                  # a class member that shares the factor 3 with R
        N3 = rng.random_odd(240000)
        if N3 % 3 == 0 and A.probe(N3, 3)[0][:3] == cls:
            break
    b = A.Batch(cls + (0,), capacity=5, max_steps=8)
    failed = b.load_many([(4, nums[0][0], 3), (1, nums[1][0], 3), (2, N3, 3), (0, nums[2][0], 3)])
    assert failed == [False, False, True, False]
    assert b.slot(2).get_factor() % 3 == 0
    b.release(2)
    order = [(4, nums[0][0], 3), (1, nums[1][0], 3), (0, nums[2][0], 3)]
    singles = []
    for s, N, a in order:
        v = b.slot(s)
        v.set1()
        t = A.Transform(N, a)
        t.set1()
        singles.append(t)
    mult = np.zeros((8, 5), dtype=np.uint32)
    mult[:, 4] = 3; mult[:, 1] = 1; mult[:, 0] = 3
    b.steps(mult)
    for (s, N, a), t in zip(order, singles):
        for i in range(8):
            t.square_mul(int(mult[i, s]))
        assert np.array_equal(b.slot(s).read_register(0), t.read_register(0)), "slot %d" % s
        assert b.slot(s).get(0) == pow(int(mult[0, s]), 255, N)       # 8 steps of r = m r^2 from r = 1


def test_runner_frees_idle_batches_for_other_sizes():
    # a budget that holds one batch of one slot: the second size class can only
    # be admitted once the first test is done and its idle batch freed
    small = random_N(20000, 1)
    big = random_N(60000, 2)
    pb, _ = A.probe(big, 3)
    ps, _ = A.probe(small, 3)
    assert pb[:3] != ps[:3]
    budget = max(A.lib().ab_batch_slot_bytes(A.Params(*pb[:3], 0)), A.lib().ab_batch_slot_bytes(A.Params(*ps[:3], 0)))
    r = A.Runner(chunk=32, max_slots_per_class=4, hbm_budget_bytes=budget)
    r.submit(small, base=3, tag=1)
    r.submit(big, base=3, tag=2)
    a, q = r.advance()
    assert a == 1 and q == 1
    res = _run_all(r)
    assert set(res) == {1, 2}
    for tag, N in ((1, small), (2, big)):
        solo = A.prp_check(N, base=3)
        assert res[tag]["status"] == 0 and res[tag]["res64"] == solo["res64"]


def test_prepare_then_install_equals_load():
    # the two halves of ab_batch_load, the host half on another thread
    import ctypes as C
    import threading
    cls = (5, 4, 12)
    (N, _), = _same_class_numbers(cls, 1, 200000, 280000, 12)
    L = A.lib()
    limbs = A.int_to_limbs(N)
    out = {}

    def host_half():
        p, prm, failed = C.c_void_p(), A.Params(), C.c_int()
        out["rc"] = L.ab_batch_prepare(limbs.ctypes.data_as(A._u64p), len(limbs), 3, C.byref(p), C.byref(prm), C.byref(failed))
        out["p"], out["cls"], out["failed"] = p, (prm.K, prm.pck, prm.ln), failed.value
    th = threading.Thread(target=host_half)
    th.start()
    th.join()
    assert out["rc"] == A.AB_OK and out["cls"] == cls and out["failed"] == 0
    b = A.Batch(cls + (0,), capacity=2, max_steps=8)
    assert L.ab_batch_ready(b.h) == 2                        # idle
    A._check(L.ab_batch_install(b.h, 1, out["p"]))           # takes ownership
    b.Ns[1], b.bases[1] = N, 3                                # what the Python wrapper keeps for get()
    b.load(0, N, 3)
    for s in (0, 1):
        b.slot(s).set1()
    mult = np.full((8, 2), 3, dtype=np.uint32)
    b.steps(mult)
    assert np.array_equal(b.slot(0).read_register(0), b.slot(1).read_register(0))
    assert b.slot(1).get(0) == pow(3, 255, N)
    b.synchronize()
    assert L.ab_batch_ready(b.h) == 2


def test_mixed_group_equals_single_transforms():
    # three size classes (three row lengths, K = 3, 4, 5) in one group: every
    # pass is one launch over all of them; slots must equal single transforms
    specs = [((5, 4, 12), 200000, 280000), ((4, 2, 11), 90000, 110000), ((3, 2, 9), 15000, 25000)]
    batches, singles, caps = [], [], [3, 4, 2]
    for ci, (cls, lo, hi) in enumerate(specs):
        nums = _same_class_numbers(cls, 2, lo, hi, 30 + ci)
        b = A.Batch(cls + (0,), capacity=caps[ci], max_steps=16)
        row = []
        for s, (N, _) in zip((0, caps[ci] - 1), nums):        # a gap between the loaded slots
            assert not b.load(s, N, 3)
            v = b.slot(s)
            v.set1(); v.copy(1, 0)
            t = A.Transform(N, 3)
            t.set1(); t.copy(1, 0)
            row.append((s, t))
        batches.append(b)
        singles.append(row)
    m = A.Mixed(batches, max_steps=16)
    rng = np.random.default_rng(11)
    for rnd in range(3):
        steps = 16 if rnd != 1 else 12                      # a second graph for a shorter chunk
        mults, snaps = [], []
        for ci, b in enumerate(batches):
            mult = rng.choice([1, 3], size=(steps, caps[ci])).astype(np.uint32)
            loaded = {s for s, _ in singles[ci]}
            for s in range(caps[ci]):
                if s not in loaded:
                    mult[:, s] = 0
            if ci == 1 and rnd == 2:
                mult[steps - 4:, caps[ci] - 1] = 0             # sits the last steps out
            snap = np.zeros((steps, caps[ci]), dtype=np.uint8)
            snap[5, 0] = 1
            mults.append(mult); snaps.append(snap)
        m.steps(mults, snaps)
        for ci, b in enumerate(batches):
            b.gl_mul(0)
            for s, t in singles[ci]:
                for i in range(steps):
                    if mults[ci][i, s]:
                        t.square_mul(int(mults[ci][i, s]))
                        if s == 0 and i == 5:
                            t.copy(2, 0)
                if s == 0:
                    t.mul(1, 2)
                v = b.slot(s)
                assert np.array_equal(v.read_register(0), t.read_register(0)), "class %d slot %d Reg0, round %d" % (ci, s, rnd)
                assert np.array_equal(v.read_register(1), t.read_register(1)), "class %d slot %d Reg1, round %d" % (ci, s, rnd)
    assert m.launch_count() > 0
    m.synchronize()
    assert m.ready() == 2
    for ci, b in enumerate(batches):
        for s, t in singles[ci]:
            assert b.slot(s).get(0) == t.get(0)
    m.close()
