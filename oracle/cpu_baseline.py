"""TEST/BENCH INFRASTRUCTURE ONLY: times the reference's own CPU transform.

The reference's transformCPU (src/transformCPU.h, single-threaded by design)
is compiled from the reference sources into _ref/libannie_ref.so (Makefile
here).  To use every host core, P independent processes each build the
transform for the same N and time `squarings` square_mul calls -- the first
iterations of the Fermat test loop; throughput is the total number of
squarings over the slowest process's time.  Set-up (N^-1 mod R, NTT of N) is
not timed.  One process also returns its registers after the window, which
checks the GPU engine on the same window.
"""
import multiprocessing as mp
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))


def window_multipliers(N, a, count):
    """Multipliers of the first `count` iterations of the Fermat test loop on
    E = N - 1 (src/annie.h:319-341): a where the bit of E is set, else 1, from
    the top bit down."""
    E = N - 1
    top = E.bit_length() - 1
    return [a if (E >> (top - i)) & 1 else 1 for i in range(count)]


def _worker(args):
    bits, seed, a, squarings, keep = args
    sys.path.insert(0, HERE)
    sys.path.insert(0, os.path.dirname(HERE))
    import tempfile
    import pyoracle
    from annie_b200.synth import Xoshiro256ss
    N = Xoshiro256ss(seed).random_odd(bits)
    t = pyoracle.RefTransform(N, a, 0)
    # the window: Reg0 = 1, Reg1 = Reg0, `squarings` iterations of the test
    # loop, then the Gerbicz-Li product Reg1 *= Reg0 (untimed)
    t.set1()
    t.copy(1, 0)
    pattern = window_multipliers(N, a, squarings)
    t0 = time.perf_counter()
    t.square_mul_seq(pattern)
    dt = time.perf_counter() - t0
    regs = None
    if keep:
        t.mul(1, 0)
        fd, path = tempfile.mkstemp()
        os.close(fd)
        try:
            regs = t.checkpoint_words(path)
        finally:
            os.unlink(path)
    t.close()
    return dt, regs


def _registers_worker(args):
    limbs, a, mults = args
    sys.path.insert(0, HERE)
    import tempfile
    import pyoracle
    N = int.from_bytes(bytes(limbs), "little")
    t = pyoracle.RefTransform(N, a, 0)
    t.set1()
    t.copy(1, 0)
    t.square_mul_seq(mults)
    t.mul(1, 0)
    fd, path = tempfile.mkstemp()
    os.close(fd)
    try:
        return t.checkpoint_words(path)
    finally:
        os.unlink(path)
        t.close()


def reference_registers(N, a, mults):
    """Reg0 || Reg1 of the reference's transformCPU after set1, Reg1 = Reg0, the
    square_mul calls with multipliers `mults`, and Reg1 *= Reg0 (in a spawned
    process)."""
    import pyoracle
    if not pyoracle.ref_available():
        pyoracle.build()
    if not pyoracle.ref_available():
        raise RuntimeError("the reference's transformCPU is not built (oracle/_ref/libannie_ref.so)")
    ctx = mp.get_context("spawn")
    with ctx.Pool(1) as pool:
        return pool.map(_registers_worker, [(list(N.to_bytes((N.bit_length() + 7) // 8, "little")), a, list(mults))])[0]


def run(bits, seed, a=3, squarings=2, procs=None):
    """Returns dict(value_us=aggregate microseconds per squaring, single_us=one
    core's microseconds per squaring, cores=P, squarings=total, seconds=the
    slowest process's timed seconds, regs=Reg0 || Reg1 words of the reference
    after the window and the product, as written by its save_checkpoint)."""
    import pyoracle
    if not pyoracle.ref_available():
        pyoracle.build()
    if not pyoracle.ref_available():
        raise RuntimeError("the reference's transformCPU is not built (oracle/_ref/libannie_ref.so)")
    if procs is None:
        procs = max(1, min(os.cpu_count() or 1, 64))
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.map(_worker, [(bits, seed, a, squarings, i == 0) for i in range(procs)])
    times = [r[0] for r in res]
    total = procs * squarings
    slowest = max(times)
    return {
        "value_us": slowest / total * 1e6,
        "single_us": sum(times) / len(times) / squarings * 1e6,
        "cores": procs,
        "squarings": total,
        "seconds": slowest,
        "regs": res[0][1],
    }


if __name__ == "__main__":
    r = run(int(sys.argv[1]), int(sys.argv[2]), squarings=int(sys.argv[3]) if len(sys.argv) > 3 else 2)
    r.pop("regs")
    print(r)
