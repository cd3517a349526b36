#!/usr/bin/env python
"""Benchmark of the modular-squaring engine at the headline size.

Workload: Fermat PRP base 3 of a random odd 33,219,281-bit N (about 10 M
digits; xoshiro256** seed 2, top bit and bit 0 set), NTT of 2^19 words over
K = 5 primes, digits of 4 x 17 bits -- the reference's own parameter choice
(transformGPU.h:822-857).  One step = 512 consecutive square_mul calls of the
exponentiation loop (annie.h:319-341) on E = N - 1.

Metric: microseconds per squaring (lower is better), whole job: the timed
device time divided by the squarings of all ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU: one process per GPU (torchrun); every rank runs an independent
test (replicas, weak scaling) -- a single test does not shard.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BITS = 33219281
SEED = 2
BASE = 3
SQ_PER_STEP = 512
METRIC = "us_per_squaring_33.2Mbit"
UNIT = "us/squaring"
WORKLOAD = "Fermat PRP base 3, random odd 33,219,281-bit N (xoshiro256** seed 2), NTT 2^19 x 5 primes, 4x17-bit digits"


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def barrier(pg):
    if pg is not None:
        import torch
        t = torch.ones(1, device="cuda")
        pg.all_reduce(t)
        torch.cuda.synchronize()


def allmax(pg, value):
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def allsum(pg, value):
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    pg.all_reduce(t)
    return float(t.item())


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().strip().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def exponent_bits(N, start, count):
    """Bits E_start, E_(start-1), ... of E = N - 1, packed LSB-first for square_mul_bits."""
    E = N - 1
    lo = start - count + 1
    window = (E >> lo) & ((1 << count) - 1) if lo >= 0 else (E & ((1 << (start + 1)) - 1)) << (-lo)
    return int(format(window, "0%db" % count)[::-1], 2)


def run_ours(args, world, rank, local, pg):
    import annie_b200 as A
    from annie_b200.synth import Xoshiro256ss

    N = Xoshiro256ss(SEED).random_odd(BITS)
    t = A.Transform(N, BASE, device=local)
    if t.init_failed():
        raise SystemExit("N shares a factor with R; choose another seed")
    S = SQ_PER_STEP
    top = N.bit_length() - 1
    pos = top
    steps_bits = []
    for _ in range(args.warmup + args.steps + args.e2e_steps):
        steps_bits.append(exponent_bits(N, pos, S))
        pos -= S
    t.set1()
    t.copy(1, 0)
    si = 0
    for _ in range(args.warmup):
        t.square_mul_bits(steps_bits[si], S, BASE)
        si += 1
    t.synchronize()

    # ---- device-timed region: K steps, L2 flushed between steps (not timed)
    clocks = Clocks(local)
    launches0 = t.launch_count()
    barrier(pg)
    clocks.start()
    wall0 = time.perf_counter()
    dev_ms = 0.0
    for _ in range(args.steps):
        t.flush_l2(256 << 20)
        t.timer_start()
        t.square_mul_bits(steps_bits[si], S, BASE)
        dev_ms += t.timer_stop()
        si += 1
    t.synchronize()
    wall_ms = (time.perf_counter() - wall0) * 1e3
    clk = clocks.stop()
    barrier(pg)
    launches = t.launch_count() - launches0 - args.steps * 0
    dev_ms_max = allmax(pg, dev_ms)
    total_sq = S * args.steps * world
    value = dev_ms_max * 1e3 / total_sq

    # ---- end to end through the C ABI with host buffers: per step, load the
    # checkpoint (Reg0, Reg1) from pinned host memory, S squarings, the
    # Gerbicz-Li product, save the checkpoint back to host memory.
    size = 8 + 8 * t.K * t.n
    arr, ptr = t.pinned(size)
    t.save_checkpoint_into(ptr, size)
    barrier(pg)
    e0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        t.read_checkpoint_from(ptr, size)
        t.square_mul_bits(steps_bits[si], S, BASE)
        t.mul(1, 0)
        t.save_checkpoint_into(ptr, size)
        si += 1
    e2e_ms = (time.perf_counter() - e0) * 1e3
    barrier(pg)
    e2e_ms = allmax(pg, e2e_ms)
    t.free_pinned(ptr)
    e2e_value = e2e_ms * 1e3 / (S * args.e2e_steps * world)

    # ---- roofline of the dominant kernel: per-launch device times of one squaring
    prof = [t.profile_square(BASE) for _ in range(5)][1:]
    per = [statistics.median(x[i] for x in prof) for i in range(len(prof[0]))]
    A_bytes = t.K * t.n * 4
    # launches of one squaring and their algorithmic bytes (reads + writes of
    # registers and operands, twiddle tables excluded), in units of A = K n 4
    names = ["rowpass square Q+R", "colpass carry Q->TQ, R->fwdR", "rowpass mul Ninv (R)",
             "colpass carry R+2 -> fwdQ", "rowpass mul N (Q)", "colpass carry-sub Q -> Reg0, fwdQ+R"]
    units = [4, 4, 3, 2, 3, 5]
    peak, peak_kind = measured_peak()
    kernels = []
    for nm, u, ms in zip(names, units, per):
        gbs = u * A_bytes / (ms * 1e-3) / 1e9
        kernels.append({"name": nm, "ms": round(ms, 5), "alg_bytes": u * A_bytes, "GBps": round(gbs, 1)})
    dom = max(range(len(per)), key=lambda i: per[i])
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            traffic = json.load(f).get(names[dom])
    sq_ms = sum(per)
    roof = {
        "bound": "hbm", "kernel": names[dom],
        "achieved": kernels[dom]["GBps"], "peak": peak, "unit": "GB/s",
        "frac": round(kernels[dom]["GBps"] / peak, 4), "peak_source": peak_kind,
        "traffic": traffic,
        "per_squaring": {"alg_bytes": 21 * A_bytes, "ms": round(sq_ms, 5),
                         "GBps": round(21 * A_bytes / (sq_ms * 1e-3) / 1e9, 1),
                         "frac": round(21 * A_bytes / (sq_ms * 1e-3) / 1e9 / peak, 4),
                         "GBps_27A_model": round(27 * A_bytes / (sq_ms * 1e-3) / 1e9, 1)},
        "kernels": kernels,
    }

    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dev_ms_max / args.steps, 4),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded random N)",
        "config": {"workload": WORKLOAD, "squarings_per_step": S, "ln": t.ln, "K": t.K, "pck": t.pck, "lbase": t.lbase,
                   "l2": "256 MiB write between steps, outside the timed region",
                   "parallelism": "replicas (one independent test per GPU)"},
        "wall_ms_timed_region": round(wall_ms, 2),
        "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "h2d_bytes_per_step": size, "d2h_bytes_per_step": size,
                "note": "checkpoint load + %d squarings + Gerbicz-Li mul + checkpoint save per step, pinned host buffers" % S},
        "gpu_launches": int(allsum(pg, launches)),
        "clocks": clk,
        "roofline": roof,
    }
    return line


def cpu_baseline_line(args, steps):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import cpu_baseline
    res = cpu_baseline.run(BITS, SEED, BASE, squarings=steps)
    return res


def run_reference(args, world, rank, pg):
    if rank != 0:
        return None
    res = cpu_baseline_line(args, max(1, args.steps // 5))
    v = res["value_us"]
    return {
        "metric": METRIC, "value": round(v, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(v * SQ_PER_STEP / 1e3, 3), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded random N)",
        "impl": "reference",
        "config": {"workload": WORKLOAD, "squarings_per_step": SQ_PER_STEP},
        "cpu_baseline": {"value": round(v, 3), "unit": UNIT, "cores": res["cores"], "kind": "reference",
                         "sample": "reference transformCPU (src/transformCPU.h) compiled from the reference sources, "
                                   "%d processes x %d squarings at 33.2M bits, set-up untimed; one core: %.0f us/squaring"
                                   % (res["cores"], res["squarings"] // res["cores"], res["single_us"])},
        "e2e": {"value": round(v, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    world, rank, local, pg = dist_setup()
    if args.impl == "reference":
        line = run_reference(args, world, rank, pg)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    line = run_ours(args, world, rank, local, pg)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        res = cpu_baseline_line(args, 2)
        line["cpu_baseline"] = {
            "value": round(res["value_us"], 3), "unit": UNIT, "cores": res["cores"], "kind": "reference",
            "sample": "reference transformCPU compiled from its sources, %d processes x 2 squarings at 33.2M bits "
                      "(set-up untimed); one core: %.0f us/squaring" % (res["cores"], res["single_us"])}
    if pg is not None:
        pg.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
