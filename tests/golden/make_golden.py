"""Generates the golden fixtures of tests/golden from the reference's own code.

Run where the reference sources are available (they are compiled into
oracle/_ref/libannie_ref.so by oracle/Makefile):

    python tests/golden/make_golden.py [--big]

* prp_vectors.json -- full PRP tests through the reference driver annie::check
  (src/annie.h:217-430, built with CPU_TRANSFORM: transformGMP below 10^4
  digits, transformCPU above): verdict and RES64 for seeded random odd N
  (Fermat base 3) and Proth numbers k*2^n+1 (Euler, base from the Jacobi
  rule).  --big appends the 262,144-bit Fermat case and a Proth number
  k*2^100000+1 (about 30 CPU minutes).
* regs_*.npz -- raw register words of the reference transformCPU
  (src/transformCPU.h) after each of a fixed list of square_mul calls, and of
  Reg1 after mul(Reg1, Reg0), for seeded N.

N is reproduced from (form, bits/k/n, seed) by annie_b200.synth, so the
fixtures stay small.
"""
import json
import math
import os
import re
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

sys.path.insert(0, os.path.dirname(HERE))
import pyoracle  # noqa: E402
from helpers import proth_N, random_N  # noqa: E402

SQ_PATTERN = [3, 1, 3, 3, 1, 1, 3, 1]


def ref_check(N, euler, base):
    """annie::check through the reference driver; returns (status, is_prp, res64 or None, line)."""
    L = pyoracle.lib_ref()
    limbs = pyoracle.int_to_limbs(N)
    with tempfile.TemporaryDirectory() as d:
        st = L.ref_check(pyoracle._ptr64(limbs), len(limbs), int(euler), base, d.encode())
        text = open(os.path.join(d, "results.txt")).read() if os.path.exists(os.path.join(d, "results.txt")) else ""
    line = text.strip().splitlines()[-1] if text.strip() else ""
    m = re.search(r"res64 = ([0-9A-F]{16})", line)
    return st, ("probable prime" in line), (m.group(1) if m else None), line


def prp_vectors(big):
    out = []
    for bits, seed in ([(20000, 1), (60000, 2), (100000, 3)] if not big else [(262144, 4)]):
        N = random_N(bits, seed)
        st, prp, res, line = ref_check(N, False, 3)
        out.append({"form": "random_odd", "bits": bits, "seed": seed, "euler": 0, "base": 3,
                    "status": st, "is_prp": prp, "res64": res})
        print(out[-1], flush=True)
    for n, seed in ([(20000, 5), (40000, 6)] if not big else [(100000, 7)]):
        k, N = proth_N(n, seed)
        st, prp, res, line = ref_check(N, True, 0)
        out.append({"form": "proth", "k": k, "n": n, "seed": seed, "euler": 1, "base": 0,
                    "status": st, "is_prp": prp, "res64": res})
        print(out[-1], flush=True)
    return out


def register_vectors():
    for bits, seed in [(20000, 11), (70000, 12)]:
        N = random_N(bits, seed)
        t = pyoracle.RefTransform(N, 3, 0)
        assert not t.init_failed()
        path = tempfile.mktemp()
        t.set1()
        t.copy(1, 0)
        regs = []
        for a in SQ_PATTERN:
            t.square_mul(a)
            w = t.checkpoint_words(path)
            regs.append(w[: len(w) // 2])
        t.mul(1, 0)
        w = t.checkpoint_words(path)
        os.unlink(path)
        np.savez_compressed(os.path.join(HERE, "regs_%d_s%d.npz" % (bits, seed)),
                            reg0=np.array(regs, dtype=np.uint32), reg1=w[len(w) // 2:].astype(np.uint32),
                            pattern=np.array(SQ_PATTERN, dtype=np.int32), get0=np.frombuffer(
                                t.get(0).to_bytes((N.bit_length() + 7) // 8 + 8, "little"), dtype=np.uint8))
        print("regs", bits, seed, flush=True)


if __name__ == "__main__":
    pyoracle.build()
    big = "--big" in sys.argv
    path = os.path.join(HERE, "prp_vectors.json")
    if not big:
        register_vectors()
        vec = prp_vectors(False)
    else:
        # appends the long cases to the existing file
        with open(path) as f:
            vec = [v for v in json.load(f) if not v.get("big")]
        for v in prp_vectors(True):
            v["big"] = 1
            vec.append(v)
    with open(path, "w") as f:
        json.dump(vec, f, indent=1)
