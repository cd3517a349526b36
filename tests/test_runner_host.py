"""Host half of admission, on CPU (no CUDA call is made on these paths):

* ab_batch_prepare gives the size class of ab_probe and, when gcd(N, R) != 1,
  the gcd, as the reference's factory reports it (src/transformGPU.h:822-850);
* the runner's set-up threads decide the trivial cases of src/annie.h:222-237
  and finish a test whose N has no supported length with status -1, without a
  transform or a GPU.
"""
import ctypes as C
import time

import numpy as np
import pytest

import annie_b200 as A
from helpers import random_N


def _lib():
    try:
        return A.lib()
    except A.EngineUnavailable as e:
        pytest.skip(str(e))


def _prepare(L, N, a):
    limbs = A.int_to_limbs(N)
    p, prm, failed = C.c_void_p(), A.Params(), C.c_int()
    rc = L.ab_batch_prepare(limbs.ctypes.data_as(A._u64p), len(limbs), a, C.byref(p), C.byref(prm), C.byref(failed))
    assert rc == A.AB_OK, L.ab_last_error()
    return p, (prm.K, prm.pck, prm.ln, prm.lbase), failed.value


def test_prepare_matches_probe():
    L = _lib()
    for bits, seed in ((60000, 2), (250000, 3)):
        N = random_N(bits, seed)
        p, params, failed = _prepare(L, N, 3)
        try:
            assert (params, bool(failed)) == A.probe(N, 3)
            assert failed == 0
            n = 1 << params[2]
            assert L.ab_prepared_bytes(p) == 3 * 3 * n * 4          # N, N^-1 mod R and 1 in normal form
        finally:
            L.ab_prepared_destroy(p)


def test_prepare_reports_the_gcd():
    L = _lib()
    N = 3 * (1 << 664381) + 1                                  # gcd(N, R) = 7 for this class
    p, params, failed = _prepare(L, N, 3)
    try:
        assert failed == 1 and A.probe(N, 3) == (params, True)
        out, cnt = np.zeros(4, dtype=np.uint64), C.c_size_t()
        assert L.ab_prepared_factor(p, out.ctypes.data_as(A._u64p), 4, C.byref(cnt)) == A.AB_OK
        assert [int(x) for x in out[:cnt.value]] == [7]
    finally:
        L.ab_prepared_destroy(p)


def _drain(r, want, seconds=60):
    got, t0 = {}, time.time()
    while len(got) < want and time.time() - t0 < seconds:
        r.advance()
        got.update(dict(r.poll()))
    return got


def test_runner_decides_without_a_transform():
    _lib()
    r = A.Runner(chunk=16)
    try:
        r.submit(1000003, tag=1)                     # <= 15 digits: decided by GMP
        r.submit(999999999999999, tag=2)             # composite, 15 digits
        r.submit((1 << 4000) + 2, tag=3)             # even
        r.submit(3 * (1 << 664381) + 1, euler=True, tag=4)   # gcd(N, R) = 7
        r.submit((1 << 400_000_000) + 1, tag=5)     # beyond the longest transform
        res = _drain(r, 5)
        assert res[1]["decided_early"] == 1 and res[1]["is_prp"] == 1
        assert res[2]["decided_early"] == 1 and res[2]["is_prp"] == 0
        assert "even" in res[3]["message"]
        assert res[4]["decided_early"] == 1 and res[4]["message"].startswith("7 divides N")
        assert res[5]["status"] == -1 and "set up" in res[5]["message"]
        assert r.advance() == (0, 0)
        assert r.stats()["batches"] == 0                 # no batch was created
    finally:
        r.close()


def test_runner_rejects_bad_epoch_options():
    _lib()
    with pytest.raises(A.EngineError):
        A.Runner(latency_ln=-1)
    with pytest.raises(A.EngineError):
        A.Runner(latency_ln=12, epoch_us=0)
    r = A.Runner(latency_ln=12, epoch_us=5000)          # host only until a test needs a transform
    r.submit(1000003, tag=7)
    res = _drain(r, 1)
    assert res[7]["decided_early"] == 1
    r.close()
