"""Builds the CUDA engine in-tree: annie_b200/lib/libannie_b200.so (sm_100a).

    python -m annie_b200.build [--verbose-ptxas]

nvcc compiles every .cu under annie_b200/csrc for sm_100a only and links the
system GMP runtime (libgmp.so.10) used for the integer set-up (N^-1 mod R, gcd,
mod N), as the reference does.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libannie_b200.so")
GMP_SO = "/usr/lib/x86_64-linux-gnu/libgmp.so.10"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


HOST = os.path.join(HERE, "host")


def sources():
    return (sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu")) +
            sorted(os.path.join(HOST, f) for f in os.listdir(HOST) if f.endswith(".cpp")))


def deps():
    inc = os.path.join(HERE, "..", "include")
    return (sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC)) + sorted(os.path.join(HOST, f) for f in os.listdir(HOST)) +
            sorted(os.path.join(inc, f) for f in os.listdir(inc)) + [os.path.join(HERE, "gmp", "gmp.h")])


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in deps())


def build(force=False, ptxas_verbose=False, jobs=None):
    if not force and up_to_date():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    objs = []
    procs = []
    for src in sources():
        obj = os.path.join(LIBDIR, os.path.basename(src).rsplit(".", 1)[0] + ".o")
        cmd = [NVCC, "-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC", "-c",
               "-I" + os.path.join(HERE, "gmp"), "-I" + CSRC, "-I" + HOST, src, "-o", obj]
        if ptxas_verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    failed = False
    for src, p in procs:
        out = p.communicate()[0].decode()
        if p.returncode != 0:
            failed = True
            sys.stderr.write(out)
        elif ptxas_verbose:
            sys.stdout.write(out)
    if failed:
        raise RuntimeError("nvcc failed")
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-L" + os.path.dirname(GMP_SO), "-l:" + os.path.basename(GMP_SO), "-cudart=static"]
    subprocess.run(cmd, check=True)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    build(force=True, ptxas_verbose="--verbose-ptxas" in sys.argv)
    print(LIB)
