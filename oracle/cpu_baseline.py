"""TEST/BENCH INFRASTRUCTURE ONLY: times the reference's own CPU transform.

The reference's transformCPU (src/transformCPU.h, single-threaded by design)
is compiled from the reference sources into _ref/libannie_ref.so (Makefile
here).  To use every host core, P independent processes each build the
transform for the same N and time `squarings` square_mul calls; throughput is
the total number of squarings over the slowest process's time.  Set-up
(N^-1 mod R, NTT of N) is not timed.
"""
import multiprocessing as mp
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))


def _worker(args):
    bits, seed, a, squarings = args
    sys.path.insert(0, HERE)
    sys.path.insert(0, os.path.dirname(HERE))
    import pyoracle
    from annie_b200.synth import Xoshiro256ss
    N = Xoshiro256ss(seed).random_odd(bits)
    t = pyoracle.RefTransform(N, a, 0)
    t.set1()
    t.square_mul(a)   # first touch of the arrays, not timed
    t0 = time.perf_counter()
    pattern = [a if (i % 2 == 0) else 1 for i in range(squarings)]
    t.square_mul_seq(pattern)
    dt = time.perf_counter() - t0
    t.close()
    return dt


def run(bits, seed, a=3, squarings=2, procs=None):
    """Returns dict(value_us=aggregate microseconds per squaring, single_us=one
    core's microseconds per squaring, cores=P, squarings=total)."""
    import pyoracle
    if not pyoracle.ref_available():
        pyoracle.build()
    if procs is None:
        procs = max(1, min(os.cpu_count() or 1, 64))
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        times = pool.map(_worker, [(bits, seed, a, squarings)] * procs)
    total = procs * squarings
    slowest = max(times)
    return {
        "value_us": slowest / total * 1e6,
        "single_us": sum(times) / len(times) / squarings * 1e6,
        "cores": procs,
        "squarings": total,
        "seconds": slowest,
    }


if __name__ == "__main__":
    print(run(int(sys.argv[1]), int(sys.argv[2]), squarings=int(sys.argv[3]) if len(sys.argv) > 3 else 2))
