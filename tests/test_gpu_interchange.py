"""Checkpoint interchange with the reference (src/annie.h:140-190 for the file,
src/transformGPU.h:608-641 for the GPU payload, src/file.h for the CRC seal).

* A file written by the reference's own file class, holding a GPU-layout
  payload built from the reference transformCPU's registers in the middle of
  a test, is resumed by this engine's PRP driver, which then finishes the test
  with the RES64 and Gerbicz-Li validation of the uninterrupted reference run.
* A file this driver wrote when the test was aborted is read and seal-checked
  by the reference's file class, its registers go into transformCPU, and the
  reference finishes the test loop with the same RES64.

N is the 60,000-bit golden number (tests/golden/prp_vectors.json), for which
the GPU factory and transformCPU choose the same K, n and digit size.
"""
import json
import os
import threading
import time

import numpy as np
import pytest

import annie_b200 as A
from helpers import random_N

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
BITS, SEED, BASE = 60000, 2, 3


def _golden_res64():
    with open(os.path.join(HERE, "golden", "prp_vectors.json")) as f:
        v = [x for x in json.load(f) if x["form"] == "random_odd" and x["bits"] == BITS and x["seed"] == SEED]
    return v[0]["res64"]


def _gl_block(size):
    L = 2 << ((size.bit_length() - 1) // 2)
    return (size - 1) // L + 1


def _ref_loop(r, E, a, i_from, i_end, B):
    """annie::check's loop (src/annie.h:319-341) on the reference transform over
    the bits i_from, i_from - 1, ..., i_end of E, with the Gerbicz-Li product."""
    i = i_from
    while i >= i_end:
        stop = max(i_end, (i // B) * B)
        r.square_mul_seq([a if (E >> j) & 1 else 1 for j in range(i, stop - 1, -1)])
        if stop % B == 0 and stop // B != 0:
            r.mul(1, 0)
        i = stop - 1


def _setup(oracle_mod):
    if not oracle_mod.ref_available():
        pytest.skip("the reference's transformCPU is not built here")
    N = random_N(BITS, SEED)
    params, failed = A.probe(N, BASE)
    assert not failed and params == oracle_mod.select_params(N, BASE, 1)
    return N, params[0], 1 << params[2]


def test_reference_checkpoint_resumes_here(oracle_mod, tmp_path):
    N, K, n = _setup(oracle_mod)
    E = N - 1
    B = _gl_block(E.bit_length())
    i0 = E.bit_length() - 1
    i_ck = i0 - 3 * B - 17                     # inside a Gerbicz-Li block
    r = oracle_mod.RefTransform(N, BASE, 0)
    r.set1()
    r.copy(1, 0)
    _ref_loop(r, E, BASE, i0, i_ck + 1, B)
    w = r.checkpoint_words(str(tmp_path / "cpu.bin"))
    payload = np.empty(2 + 2 * K * n, dtype=np.uint32)
    payload[0], payload[1] = K, n
    for k in range(K):                         # per prime: Reg0 then Reg1 (transformGPU.h:626-641)
        payload[2 + 2 * k * n:2 + 2 * k * n + n] = w[k * n:(k + 1) * n]
        payload[2 + 2 * k * n + n:2 + 2 * (k + 1) * n] = w[K * n + k * n:K * n + (k + 1) * n]
    path = str(tmp_path / "interchange.chk")
    assert oracle_mod.ref_file_write_checkpoint(path, i_ck, 12.5, payload.tobytes()) == 0
    res = A.prp_check(N, base=BASE, checkpoint_path=path)
    assert res["resumed"] == 1, res["message"]
    assert res["status"] == 0, res["message"]            # final Gerbicz-Li validation passed
    assert "%016X" % res["res64"] == _golden_res64()


def test_checkpoint_written_here_finishes_in_reference(oracle_mod, tmp_path):
    N, K, n = _setup(oracle_mod)
    E = N - 1
    B = _gl_block(E.bit_length())
    path = str(tmp_path / "aborted.chk")
    L = A.lib()
    out = {}
    # checkpoints after every run of squarings; abort once the first file exists
    th = threading.Thread(target=lambda: out.update(A.prp_check(N, base=BASE, checkpoint_path=path, checkpoint_seconds=1e-9)))
    L.ab_prp_reset_quit()
    th.start()
    t0 = time.time()
    while not os.path.exists(path) and time.time() - t0 < 60:
        time.sleep(0.001)
    L.ab_prp_quit()
    th.join()
    L.ab_prp_reset_quit()
    assert out["status"] == 2, "the test was not aborted: %s" % out["message"]
    st, i, elapsed, payload = oracle_mod.ref_file_read_checkpoint(path, 8 + 8 * K * n)
    assert st == 0, "the reference's file class rejects the file (%d)" % st
    assert 0 <= i < E.bit_length() - 1
    p = np.frombuffer(payload, dtype=np.uint32)
    assert p[0] == K and p[1] == n
    planes = p[2:].reshape(K, 2, n)
    words = np.concatenate([planes[:, 0, :].reshape(-1), planes[:, 1, :].reshape(-1)])
    r = oracle_mod.RefTransform(N, BASE, 0)
    r.load_checkpoint_words(words, str(tmp_path / "cpu.bin"))
    _ref_loop(r, E, BASE, i, 0, B)
    assert "%016X" % (r.get(0) & ((1 << 64) - 1)) == _golden_res64()
