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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BITS = 33219281
SEED = 2
BASE = 3
SQ_PER_STEP = 512
PARITY_WINDOW = 8          # test-loop iterations compared word for word with the reference
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


def _dev(pg):
    """Tensors for collectives live on the GPU under NCCL, on the CPU under gloo."""
    return "cuda" if pg.get_backend() == "nccl" else "cpu"


def barrier(pg):
    if pg is not None:
        import torch
        t = torch.ones(1, device=_dev(pg))
        pg.all_reduce(t)
        if _dev(pg) == "cuda":
            torch.cuda.synchronize()


def allmax(pg, value):
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=_dev(pg))
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def allsum(pg, value):
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=_dev(pg))
    pg.all_reduce(t)
    return float(t.item())


def shard(items, rank, world):
    """The rank's share of independent work units (candidates): every world-th item."""
    return items[rank::world]


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


def issue_bound(names, per_ms, dom, instr, sq_us, sms, mhz):
    """Issue bound of the dominant launch and of the critical path (the R-domain
    chain, names[3:]): their warp instructions (ncu) at one instruction per clock
    on each of the 4 schedulers of every SM, at the sampled SM clock; None when
    a count is missing."""
    chain = names[3:]
    if not all(nm in instr for nm in chain + [names[dom]]):
        return None
    rate = sms * 4 * mhz * 1e6                           # warp instructions per second
    ms_of = dict(zip(names, per_ms))
    n_dom, n_chain = instr[names[dom]], sum(instr[nm] for nm in chain)
    return {"sms": sms, "sm_mhz": mhz,
            "dominant": {"kernel": names[dom], "warp_instructions": n_dom, "bound_us": round(n_dom / rate * 1e6, 2),
                         "us": round(per_ms[dom] * 1e3, 2), "frac": round(n_dom / rate / (per_ms[dom] * 1e-3), 3)},
            "critical_path": {"launches": chain, "warp_instructions": n_chain, "bound_us": round(n_chain / rate * 1e6, 2),
                              "us_alone": round(sum(ms_of[nm] for nm in chain) * 1e3, 2),
                              "frac_of_squaring": round(n_chain / rate / (sq_us * 1e-6), 3)},
            "source": "warp instructions per launch from profiles/ncu_traffic.json (ncu smsp__inst_executed.sum)"}


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
    names = ["colpass fwd Q of Reg0", "rowpass square (Q)", "colpass carry Q -> T_Q", "rowpass square (R)",
             "colpass carry R -> fwd R", "rowpass mul Ninv (R)", "colpass carry R+2 -> fwd Q", "rowpass mul N (Q)",
             "colpass carry-sub Q -> Reg0, fwd R"]
    units = [2, 2, 2, 2, 2, 3, 2, 3, 4]
    assert len(per) == len(names), "unexpected launch list of one squaring: %d launches" % len(per)
    peak, peak_kind = measured_peak()
    kernels = []
    for nm, u, ms in zip(names, units, per):
        gbs = u * A_bytes / (ms * 1e-3) / 1e9
        kernels.append({"name": nm, "ms": round(ms, 5), "alg_bytes": u * A_bytes, "GBps": round(gbs, 1)})
    dom = max(range(len(per)), key=lambda i: per[i])
    traffic, instr = None, {}
    tpath = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tj = json.load(f)
        traffic = tj.get(names[dom])
        instr = tj.get("_instructions", {})
    sq_ms = sum(per)
    roof = {
        "bound": "hbm", "kernel": names[dom],
        "achieved": kernels[dom]["GBps"], "peak": peak, "unit": "GB/s",
        "frac": round(kernels[dom]["GBps"] / peak, 4), "peak_source": peak_kind,
        "traffic": traffic,
        # whole squaring in the timed (graph-replayed, overlapped) schedule
        "per_squaring": {"alg_bytes": sum(units) * A_bytes, "us": round(value, 3),
                         "GBps": round(sum(units) * A_bytes / (value * 1e-6) / 1e9, 1),
                         "frac": round(sum(units) * A_bytes / (value * 1e-6) / 1e9 / peak, 4),
                         "GBps_27A_model": round(27 * A_bytes / (value * 1e-6) / 1e9, 1),
                         "serial_launch_sum_ms": round(sq_ms, 5)},
        "kernels": kernels,
    }
    if instr:
        import torch
        sms = torch.cuda.get_device_properties(local).multi_processor_count
        issue = issue_bound(names, per, dom, instr, value, sms, (clk or {}).get("sm_mhz") or 1965.0)
        if issue is not None:
            roof["issue"] = issue

    # ---- parity window (the same window the CPU-baseline leg runs on the
    # reference): Reg0 = 1, Reg1 = Reg0, PARITY_WINDOW iterations of the test
    # loop from the top bit of E, then Reg1 *= Reg0; the registers are checked
    # word for word after the run
    t.set1()
    t.copy(1, 0)
    E = N - 1
    for i in range(PARITY_WINDOW):
        t.square_mul(BASE if (E >> (top - i)) & 1 else 1)
    t.mul(1, 0)
    regs = np.concatenate([t.read_register(0), t.read_register(1)])
    t.close()

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
    return line, regs


def cpu_baseline_line(args, steps):
    """The reference's transformCPU on the host cores over the first `steps`
    iterations of the test loop (checker and CPU baseline: see oracle/cpu_baseline.py)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import cpu_baseline
    res = cpu_baseline.run(BITS, SEED, BASE, squarings=steps)
    return res


def parity_record(gpu_regs, res):
    """Word-for-word comparison of Reg0 || Reg1 after the parity window."""
    ref = res.get("regs") if res else None
    if ref is None:
        return {"checked": False, "equal": None, "why": "the reference's transformCPU is not built here"}
    ref = np.asarray(ref, dtype=np.uint32)
    n = min(len(ref), len(gpu_regs))
    diff = int(np.count_nonzero(ref[:n] != gpu_regs[:n])) + abs(len(ref) - len(gpu_regs))
    return {"checked": True, "equal": diff == 0, "words": int(len(gpu_regs)), "words_differing": diff,
            "against": "reference transformCPU (src/transformCPU.h), compiled from the reference sources",
            "window": "Reg0 = 1, Reg1 = Reg0, %d test-loop iterations from the top bit of E = N - 1, "
                      "then Reg1 *= Reg0; raw register words of Reg0 and Reg1" % PARITY_WINDOW}


def run_reference(args, world, rank, pg):
    if rank != 0:
        return None
    per_proc = max(1, min(16, args.steps // 5))            # about 15 s of CPU per process
    res = cpu_baseline_line(args, per_proc)
    v = res["value_us"]
    return {
        "metric": METRIC, "value": round(v, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(v * SQ_PER_STEP / 1e3, 3), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded random N)",
        "impl": "reference",
        "config": {"workload": WORKLOAD, "squarings_per_step": SQ_PER_STEP},
        "extrapolated": True,
        "timed_squarings": res["squarings"],
        "timed_seconds": round(res["seconds"], 3),
        "note": "value = the squarings actually timed (%d processes x %d, the first test-loop iterations) over the "
                "slowest process's time; ms_per_step extrapolates that rate to %d squarings per step"
                % (res["cores"], per_proc, SQ_PER_STEP),
        "cpu_baseline": {"value": round(v, 3), "unit": UNIT, "cores": res["cores"], "kind": "reference",
                         "sample": "reference transformCPU (src/transformCPU.h) compiled from the reference sources, "
                                   "%d processes x %d squarings at 33.2M bits, set-up untimed; one core: %.0f us/squaring"
                                   % (res["cores"], per_proc, res["single_us"])},
        "e2e": {"value": round(v, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ---------------------------------------------------------------- other workloads
SMALL_PRIMES = [p for p in range(3, 2000) if all(p % q for q in range(2, int(p ** 0.5) + 1))]

def run_batch_workload(args, world=1, rank=0, local=0, pg=None):
    """4096 Proth candidates k*2^n+1 (k odd in [3, 2^20), n in [500000, 3000000], seeded):
    candidates/hour of the batched path (autotuned per size class, graph-captured
    chunks) against the one-at-a-time CUDA path on the same B200."""
    import annie_b200 as A
    from annie_b200.synth import Xoshiro256ss, proth
    from concurrent.futures import ThreadPoolExecutor
    rng = Xoshiro256ss(2024)
    cands = [(rng.uniform(3, 1 << 20) | 1, rng.uniform(500000, 3000001)) for _ in range(4096)]

    # Euler base and size class of every candidate; those sharing a factor with R
    # are decided by the gcd at set-up (as in the reference) and need no squaring
    def info(kn):
        N = proth(*kn)
        a = _euler_base(N)
        p, failed = A.probe(N, a)                        # the gcd runs in C, outside the GIL
        return kn, a, p, failed
    with ThreadPoolExecutor(max_workers=min(32, os.cpu_count() or 1)) as ex:
        infos = list(ex.map(info, cands))
    classes = {}
    for kn, a, p, failed in infos:
        if not failed:
            classes.setdefault(p[:3], []).append((kn[0], kn[1], a))
    full = sum(len(m) for m in classes.values())
    # iterations a candidate needs: the bits of E = (N-1)/2 = k 2^(n-1), the final
    # Gerbicz-Li power (about B + log2 of the number of blocks) and Euler's extra one
    def need(k, n):
        eb = n - 1 + k.bit_length()
        B = _gl_block(eb)
        return eb + B + max(1, (eb // B).bit_length()) + 1
    CAP, S, REPS = args.batch_slots, 32, 4
    per_class = []
    t_batch = t_plain = 0.0
    for cls, members in sorted(classes.items()):
        k0, n0, a0 = members[0]
        N = proth(k0, n0)
        E = (N - 1) >> 1
        top = E.bit_length() - 1
        bits = [(E >> (top - i)) & 1 for i in range(S)]
        mult = [[a0 if bits[i] else 1] * CAP for i in range(S)]
        b = A.Batch(cls + (0,), capacity=CAP, max_steps=S, device=local)
        b.load(0, N, a0)
        b.slot(0).set1()
        lb = b.autotune(0, S)           # times every split on copies of slot 0 in the empty slots
        for s in range(1, CAP):
            b.clone(s, 0)
        b.steps(mult)
        b.synchronize()
        t0 = time.perf_counter()
        for _ in range(REPS):
            b.steps(mult)
        b.synchronize()
        batch_rate = CAP * S * REPS / (time.perf_counter() - t0)       # squarings / s
        b.close()
        # one at a time: the single-test path (graph-replayed runs of squarings,
        # the measured default split for the length)
        t = A.Transform(N, a0, device=local)
        t.set1()
        S1 = 256
        t.square_mul_bits(0, S1, a0)
        t.synchronize()
        t.timer_start()
        for _ in range(REPS):
            t.square_mul_bits(0, S1, a0)
        single_rate = S1 * REPS / (t.timer_stop() * 1e-3)
        t.close()
        squarings = sum(need(k, n) for k, n, _ in members)
        t_batch += squarings / batch_rate
        t_plain += squarings / single_rate
        per_class.append({"class": list(cls), "candidates": len(members), "row_levels": lb,
                          "batched_sq_per_s": round(batch_rate, 1), "single_us_per_sq": round(1e6 / single_rate, 2)})
    # (with several ranks, the plain path runs one test per GPU at a time);
    # rates in full tests per hour: the candidates that need the exponentiation
    micro = world * full / (t_batch / 3600.0)
    plain = world * full / (t_plain / 3600.0)

    # the runner on the whole candidate list: admission by size class and HBM
    # budget, autotuned split per class, graph-captured chunks, Gerbicz-Li
    # products; squarings completed in a fixed wall-clock window
    # (ranks: each runs its share of the list, no data-path collective)
    r = A.Runner(device=local, chunk=S, max_slots_per_class=CAP, hbm_budget_bytes=args.batch_hbm_gb << 30)
    for idx, (k, n) in shard(list(enumerate(cands)), rank, world):
        r.submit(proth(k, n), euler=True, tag=idx)
    c0 = time.perf_counter()
    active, queued = r.advance()
    r.synchronize()
    admit_s = time.perf_counter() - c0
    for _ in range(2):
        r.advance()
    r.synchronize()
    barrier(pg)
    s0 = r.stats()["squarings"]
    w0 = time.perf_counter()
    while time.perf_counter() - w0 < args.batch_window:
        r.advance()
    r.synchronize()
    window = allmax(pg, time.perf_counter() - w0)
    st = r.stats()
    done = int(allsum(pg, len(r.poll())))
    r.close()
    rate = allsum(pg, st["squarings"] - s0) / window
    # candidates decided at set-up take no squaring: the list's time is the
    # squarings of the others at the runner's rate
    total_need = sum(need(k, n) for m in classes.values() for k, n, _ in m)
    value = full * 3600.0 * rate / total_need
    return {"metric": "proth_full_tests_per_hour_batched", "value": round(value, 3), "unit": "full tests/hour",
            "n_gpus": 1, "steps": 1, "warmup": 2, "ms_per_step": round(window * 1e3, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded Proth candidates)",
            "config": {"workload": "4096 Proth k*2^n+1, k odd in [3,2^20), n in [500000,3000000] (xoshiro256** seed 2024), Euler",
                       "slots_per_class": CAP, "squarings_per_graph": S, "hbm_budget_gb": args.batch_hbm_gb,
                       "method": "continuous-batching runner over all 4096 candidates: squarings completed in a %.0f s "
                                 "window after admission; full tests per hour = the %d candidates without a factor in "
                                 "common with R over (the iterations they need / that rate); the other %d are decided "
                                 "at set-up by the gcd and are not counted" % (args.batch_window, full, len(cands) - full)},
            "runner": {"in_flight": active, "queued": queued, "batches": st["batches"], "admission_s": round(admit_s, 2),
                       "squarings_per_s": round(rate, 1), "decided_or_finished_in_window": done,
                       "candidates_per_hour_incl_gcd_decided": round(len(cands) * 3600.0 * rate / total_need, 3)},
            "plain_full_tests_per_hour": round(plain, 3), "speedup_vs_plain": round(value / plain, 3),
            "microbench_full_tests_per_hour": round(micro, 3),
            "classes": per_class}


def _serve_stream(rate, window, lo, hi, seed):
    """Seeded Poisson arrivals over `window` seconds: (time, N, euler, base), bit
    lengths log-uniform in [lo, hi], half Fermat base 3 on random odd N and half
    Proth k*2^n+1 (Euler); N without prime factors below 2000, so that every
    request needs the full test."""
    import math
    from annie_b200.synth import Xoshiro256ss, proth
    rng = Xoshiro256ss(seed)
    reqs, t = [], 0.0
    while True:
        t += -math.log(1.0 - rng.random()) / rate
        if t > window:
            return reqs
        bits = int(math.exp(math.log(lo) + rng.random() * (math.log(hi) - math.log(lo))))
        while True:
            if len(reqs) % 2 == 0:
                N, euler, base = rng.random_odd(bits), False, 3
            else:
                N, euler, base = proth(rng.uniform(3, 1 << 20) | 1, bits), True, 0
            if all(N % p for p in SMALL_PRIMES):
                break
        reqs.append((t, N, euler, base))


def _pct(v, q):
    v = sorted(v)
    return round(v[min(len(v) - 1, int(q * len(v)))], 3) if v else None


def serve_one_rate(rate, window, lo, hi, seed, gl_check_blocks=0, autotune=True, slots=64, latency_ln=0, epoch_us=20000):
    """One Poisson stream served for a fixed window two ways, on the same GPU:
    the continuous-batching runner, and the one-at-a-time path (each test run
    to completion in arrival order, the last one stopped at the window's end).
    Throughput is squarings of PRP tests per second of window; latencies are
    those of the requests completed in the window (the others are censored)."""
    import threading
    import annie_b200 as A
    reqs = _serve_stream(rate, window, lo, hi, seed)
    # served: requests are submitted as they arrive, the runner advances
    # continuously until the window ends
    r = A.Runner(chunk=32, max_slots_per_class=slots, gl_check_blocks=gl_check_blocks, autotune=autotune,
                 latency_ln=latency_ln, epoch_us=epoch_us)
    t0 = time.perf_counter()
    served, nxt, lat_s = {}, 0, []
    while True:
        now = time.perf_counter() - t0
        if now >= window:
            break
        while nxt < len(reqs) and reqs[nxt][0] <= now:
            _, N, euler, base = reqs[nxt]
            r.submit(N, euler=euler, base=base, tag=nxt)
            nxt += 1
        active, queued = r.advance()
        now = time.perf_counter() - t0
        for tag, res in r.poll():
            served[tag] = res
            lat_s.append(now - reqs[tag][0])
        if active == 0 and queued == 0 and nxt < len(reqs):
            time.sleep(max(0.0, min(0.01, reqs[nxt][0] - now)))
    r.synchronize()
    # squarings are counted when queued: the chunks queued before the window's
    # end finish here, and their time counts
    served_s = time.perf_counter() - t0
    sq_served = r.stats()["squarings"]
    classes, host_s = r.classes(), r.host_seconds()
    r.close()
    # plain: first come first served, one test at a time; a timer stops the
    # running test at the window's end (ab_prp_quit: it returns as aborted)
    L = A.lib()
    L.ab_prp_reset_quit()
    stop = threading.Timer(window, L.ab_prp_quit)
    t0 = time.perf_counter()
    stop.start()
    plain, lat_p, sq_plain, words_plain = {}, [], 0, 0
    for i, (ta, N, euler, base) in enumerate(reqs):
        now = time.perf_counter() - t0
        if now >= window:
            break
        if now < ta:
            time.sleep(min(ta - now, window - now))
            if time.perf_counter() - t0 >= window:
                break
        res = A.prp_check(N, euler=euler, base=base)
        sq_plain += res["squarings"]
        words_plain += res["squarings"] * (res["K"] + 1) << res["ln"]
        if res["status"] == 2:                     # stopped at the window's end
            break
        plain[i] = res
        lat_p.append(time.perf_counter() - t0 - ta)
    stop.cancel()
    L.ab_prp_reset_quit()
    # every result completed in the mix equals the same test run alone
    same = True
    for tag, res in served.items():
        alone = plain.get(tag)
        if alone is None:
            _, N, euler, base = reqs[tag]
            alone = A.prp_check(N, euler=euler, base=base)
        same &= (res["res64"], res["is_prp"], res["status"]) == (alone["res64"], alone["is_prp"], alone["status"])
    # work-normalised throughput: transform words squared per second (a
    # squaring of class (K, ln) transforms (K + 1) 2^ln words)
    words_served = sum(c["squarings"] * (c["class"][0] + 1) << c["class"][2] for c in classes)
    return {"rate_per_s": rate, "requests": len(reqs), "window_s": window,
            "policy": {"latency_ln": latency_ln, "epoch_us": epoch_us if latency_ln else None, "autotune": autotune,
                       "slots_per_class": slots},
            "served": {"squarings_per_s": round(sq_served / served_s, 1), "completed": len(served),
                       "censored": len(reqs) - len(served), "p50_s": _pct(lat_s, 0.5), "p99_s": _pct(lat_s, 0.99),
                       "host_s": host_s, "classes": classes},
            "plain": {"squarings_per_s": round(sq_plain / window, 1), "completed": len(plain),
                      "censored": len(reqs) - len(plain), "p50_s": _pct(lat_p, 0.5), "p99_s": _pct(lat_p, 0.99)},
            "throughput_vs_plain": round((sq_served / served_s) / max(1e-9, sq_plain / window), 3),
            "gwords_per_s": {"served": round(words_served / served_s / 1e9, 3), "plain": round(words_plain / window / 1e9, 3)},
            "results_equal_alone": bool(same)}


def run_serve_workload(args):
    """Poisson stream of PRP requests, bit lengths log-uniform (half Fermat base 3 on
    random odd N, half Proth k*2^n+1), one fixed window per rate: squarings per
    second and p50/p99 time-to-result of the continuous-batching runner against
    the one-at-a-time path on the same stream."""
    lo, hi = args.serve_bits
    out_rates = [serve_one_rate(rate, args.serve_window, lo, hi, int(rate * 1000) + 7, autotune=not args.serve_no_autotune,
                                slots=args.serve_slots, latency_ln=args.serve_latency_ln, epoch_us=args.serve_epoch_us)
                 for rate in args.serve_rates]
    head = max(out_rates, key=lambda x: x["throughput_vs_plain"])
    return {"metric": "served_squarings_per_s", "value": head["served"]["squarings_per_s"], "unit": "squarings/s", "n_gpus": 1,
            "steps": len(out_rates), "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u32", "data": "synthetic (seeded Poisson stream)",
            "config": {"workload": "Poisson PRP requests, bit lengths log-uniform in [%d, %d], half Fermat base 3 random odd N, "
                                   "half Proth (Euler), N without prime factors below 2000; a %.0f s window per rate and path"
                                   % (lo, hi, args.serve_window),
                       "rates_per_s": args.serve_rates},
            "rates": out_rates}


def _jacobi(a, n):
    """Jacobi symbol (a/n), n odd positive."""
    a %= n
    r = 1
    while a:
        while a % 2 == 0:
            a //= 2
            if n % 8 in (3, 5):
                r = -r
        a, n = n, a
        if a % 4 == 3 and n % 4 == 3:
            r = -r
        a %= n
    return r if n == 1 else 0


def _euler_base(N):
    """Smallest non-square a >= 2 with (a/N) = -1 (the PRP driver's rule)."""
    import math
    a = 2
    while _jacobi(a, N) != -1:
        a += 1
        s = math.isqrt(a)
        if s * s == a:
            a += 1
    return a


def _gl_block(size):
    L = 2 << ((size.bit_length() - 1) // 2)
    return (size - 1) // L + 1


def _chunk_sum(e, B):
    s, mask = 0, (1 << B) - 1
    while e:
        s += e & mask
        e >>= B
    return s


def _pack_bits(E, top, count):
    """Bits E_top, E_(top-1), ... (count of them) packed LSB-first."""
    lo = top - count + 1
    w = (E >> lo) & ((1 << count) - 1) if lo >= 0 else (E & ((1 << (top + 1)) - 1)) << (-lo)
    return int(format(w, "0%db" % count)[::-1], 2)


def run_proth2m_workload(args):
    """Proth k*2^2000000+1 (k seeded odd 20-bit), Euler test with the Jacobi base:
    device-timed run of 100,000 iterations of the test loop (Gerbicz-Li product every
    B iterations included), then one Gerbicz-Li check and an injected single-word
    error that the next check detects and rolls back."""
    import annie_b200 as A
    from annie_b200.synth import proth_2m
    k, N, a = proth_2m(args.proth_n, 11, usable=lambda N, a: not A.probe(N, a)[1])
    t = A.Transform(N, a)
    E = (N - 1) >> 1
    B = _gl_block(E.bit_length())
    state = {"i": E.bit_length() - 1}

    def run(count):
        """count iterations of the test loop from the current bit, the Gerbicz-Li
        product after each B-aligned iteration (as the driver)."""
        while count > 0:
            i = state["i"]
            stop = max(i - count + 1, (i // B) * B)
            n = i - stop + 1
            t.square_mul_bits(_pack_bits(E, i, n), n, a)
            count -= n
            state["i"] = stop - 1
            if stop % B == 0 and stop // B != 0:
                t.mul(1, 0)

    def to_boundary():
        run(state["i"] - (state["i"] // B) * B + 1)

    def check():
        """Periodic Gerbicz-Li check at the boundary just passed: d_now = d_prev^(2^B) a^C."""
        i = state["i"] + 1
        C = _chunk_sum(E >> i, B)
        stash = t.save_checkpoint()
        t.set1()
        hi = C.bit_length()
        if hi > B:
            t.square_mul_bits(_pack_bits(C, hi - 1, hi - B), hi - B, a)
        t.mul(0, 2)
        t.square_mul_bits(_pack_bits(C, B - 1, B), B, a)
        v1 = t.get(0)
        t.read_checkpoint(stash)
        return v1 == t.get(1), stash

    def block_with_check():
        """The next block with d_prev kept in Reg2, then its check."""
        run(state["i"] - (state["i"] // B) * B)          # up to the boundary iteration
        t.copy(2, 1)
        run(1)                                            # boundary iteration + product
        return check()

    t.set1()
    t.copy(1, 0)
    run(args.warmup * 512)
    t.synchronize()
    total = args.proth_squarings
    t.flush_l2(256 << 20)
    t.timer_start()
    run(total)
    ms = t.timer_stop()
    us = ms * 1e3 / total
    # one Gerbicz-Li check
    to_boundary()
    t.synchronize()
    c0 = time.perf_counter()
    ok, stash = block_with_check()
    gl_ms = (time.perf_counter() - c0) * 1e3
    # injected error: one 32-bit word of Reg0 moves by one, mid-block
    verified_i = state["i"]
    c0 = time.perf_counter()
    run(B // 2)
    t.inject_word(0, 12345, -1)
    bad, _ = block_with_check()
    t.read_checkpoint(stash)                              # roll back to the verified state
    state["i"] = verified_i
    redo, _ = block_with_check()
    rb_ms = (time.perf_counter() - c0) * 1e3
    blocks = total / B
    return {"metric": "us_per_squaring_proth_n2M", "value": round(us, 3), "unit": "us/squaring", "n_gpus": 1,
            "steps": int(round(blocks)), "warmup": args.warmup, "ms_per_step": round(ms / blocks, 4),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded Proth number)",
            "config": {"workload": "Proth k*2^%d+1, k=%d, Euler test base %d; %d test iterations timed "
                                   "(one step = one Gerbicz-Li block of B=%d iterations + its product)"
                                   % (args.proth_n, k, a, total, B),
                       "ln": t.ln, "K": t.K, "lbase": t.lbase, "gl_block": B,
                       "l2": "256 MiB write before the timed region; the working set (about 10 MB) stays in L2"},
            "gl_check": {"ms": round(gl_ms, 2), "passed": bool(ok)},
            "injected_error": {"detected": not bad, "rolled_back_and_verified": bool(redo), "ms": round(rb_ms, 2),
                               "note": "one 32-bit word of Reg0 changed by one mid-block; time from the change through the failed "
                                       "check, the reload of the verified state and the repeated, verified block"}}


def run_table_workload(args):
    """The reference's own benchmark table (annie::bench, src/annie.h:432-556):
    N = 3 2^e + 1 for its 13 exponents (33,216 to 159,200,000 bits), each a
    Gerbicz-Li-validated exponentiation to 6^50, then squarings for a fixed
    time; ms per bit and the estimated time of a full test."""
    import annie_b200 as A
    rows = A.bench_table(seconds=args.table_seconds)
    out = [{"N": "3*2^%d+1" % r["e"], "digits": r["digits"], "K": r["K"], "pck": r["pck"], "ln": r["ln"], "lbase": r["lbase"],
            "validated": {1: True, 0: False, -1: "N shares a factor with R (init_failed)"}[r["validated"]],
            "ms_per_bit": round(r["ms_per_bit"], 5),
            "estimated_test_hours": round(r["estimated_seconds"] / 3600, 3), "squarings_timed": r["squarings"]} for r in rows]
    head = [r for r in out if r["N"] == "3*2^33219278+1"]
    return {"metric": "ms_per_bit_3x2^33219278+1", "value": head[0]["ms_per_bit"] if head else None, "unit": "ms/bit",
            "n_gpus": 1, "steps": len(out), "warmup": 0, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "u32", "data": "synthetic (the reference's benchmark numbers 3*2^e+1)",
            "config": {"workload": "annie -h benchmark table: 3*2^e+1, base 3, e in %s" % A.BENCH_TABLE_E,
                       "seconds_per_size": args.table_seconds},
            "all_validated": all(r["validated"] is not False for r in out) and len(out) == len(A.BENCH_TABLE_E), "rows": out}


def side_proth2m(args):
    """C2 as a sub-object of the default line, with its own parity window."""
    r = run_proth2m_workload(args)
    out = {"us_per_iteration": r["value"], "iterations_timed": args.proth_squarings, "ms_per_gl_block": r["ms_per_step"],
           "gl_block": r["config"]["gl_block"], "params": {"K": r["config"]["K"], "ln": r["config"]["ln"], "lbase": r["config"]["lbase"]},
           "workload": r["config"]["workload"], "gl_check": r["gl_check"], "injected_error": r["injected_error"]}
    if not args.no_cpu_baseline:
        out["parity"] = proth2m_parity(args)
    return out


def proth2m_parity(args, count=64):
    """Registers after `count` Euler-test iterations from set1 and Reg1 *= Reg0,
    against the reference's transformCPU on the same N (checker leg)."""
    import annie_b200 as A
    from annie_b200.synth import proth_2m
    k, N, a = proth_2m(args.proth_n, 11, usable=lambda N, a: not A.probe(N, a)[1])
    E = (N - 1) >> 1
    top = E.bit_length() - 1
    mults = [a if (E >> (top - i)) & 1 else 1 for i in range(count)]
    t = A.Transform(N, a)
    t.set1()
    t.copy(1, 0)
    for m in mults:
        t.square_mul(m)
    t.mul(1, 0)
    regs = np.concatenate([t.read_register(0), t.read_register(1)])
    t.close()
    try:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import cpu_baseline
        ref = cpu_baseline.reference_registers(N, a, mults)
    except RuntimeError as e:
        return {"checked": False, "equal": None, "why": str(e)}
    rec = parity_record(regs, {"regs": ref})
    rec["window"] = "Reg0 = 1, Reg1 = Reg0, %d Euler-test iterations from the top bit of E = (N - 1)/2, then Reg1 *= Reg0" % count
    return rec


def side_c1():
    """C1 as a sub-object of the default line: the full Fermat test (base 3,
    Gerbicz-Li block 256) of the 262,144-bit seeded N, timed end to end through
    ab_prp_check, with its RES64 against the reference's (the golden fixture
    that tests/golden/make_golden.py took from the reference's transformCPU)."""
    import annie_b200 as A
    from annie_b200.synth import Xoshiro256ss
    rng = Xoshiro256ss(4)
    while True:
        N = rng.random_odd(262144)
        if all(N % p for p in SMALL_PRIMES):
            break
    with open(os.path.join(ROOT, "tests", "golden", "prp_vectors.json")) as f:
        gold = [v for v in json.load(f) if v["form"] == "random_odd" and v["bits"] == 262144 and v["seed"] == 4][0]
    A.prp_check(N, base=3)                                 # warm-up (graphs, twiddles)
    t0 = time.perf_counter()
    res = A.prp_check(N, base=3)
    sec = time.perf_counter() - t0
    return {"bits": 262144, "seconds": round(sec, 3), "squarings": res["squarings"],
            "us_per_squaring_e2e": round(sec * 1e6 / res["squarings"], 2), "params": [res["K"], res["pck"], res["ln"], res["lbase"]],
            "res64": "%016X" % res["res64"], "res64_equals_reference": "%016X" % res["res64"] == gold["res64"],
            "gl_validated": res["status"] == 0,
            "workload": "Fermat PRP base 3 on the seeded random odd 262,144-bit N (xoshiro256** seed 4, no factor below 2000), full test"}


def side_batch(args):
    """C4 as a sub-object of the default line (a shorter runner window)."""
    import copy
    a2 = copy.copy(args)
    a2.batch_window = args.side_batch_window
    r = run_batch_workload(a2)
    return {"full_tests_per_hour": r["value"], "plain_full_tests_per_hour": r["plain_full_tests_per_hour"],
            "speedup_vs_plain": r["speedup_vs_plain"], "microbench_full_tests_per_hour": r["microbench_full_tests_per_hour"],
            "runner_squarings_per_s": r["runner"]["squarings_per_s"], "window_s": a2.batch_window,
            "size_classes": len(r["classes"]), "workload": r["config"]["workload"], "method": r["config"]["method"]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    # 391 steps of 512 = 200,192 squarings: the 33.2M-bit loop is timed over about
    # 200k squarings (about a minute)
    ap.add_argument("--steps", type=int, default=391)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="square33M", choices=["square33M", "proth2M", "batch", "serve", "table"])
    ap.add_argument("--table-seconds", type=float, default=10.0)
    ap.add_argument("--batch-slots", type=int, default=64)
    ap.add_argument("--serve-rates", type=float, nargs="+", default=[0.5, 2.0])
    ap.add_argument("--serve-bits", type=int, nargs=2, default=[100000, 20000000])
    ap.add_argument("--serve-window", type=float, default=60.0)
    ap.add_argument("--side-serve-window", type=float, default=40.0)
    ap.add_argument("--serve-no-autotune", action="store_true", help="serve: size classes keep the default split")
    ap.add_argument("--serve-slots", type=int, default=64, help="serve: slots per size class")
    ap.add_argument("--serve-latency-ln", type=int, default=14,
                    help="serve: classes with ln <= this take turns with the larger ones (0 = all together)")
    ap.add_argument("--serve-epoch-us", type=int, default=20000)
    ap.add_argument("--side-serve-rate", type=float, default=1.0)
    ap.add_argument("--proth-squarings", type=int, default=100000)
    ap.add_argument("--proth-n", type=int, default=2000000)
    ap.add_argument("--batch-window", type=float, default=30.0)
    ap.add_argument("--batch-hbm-gb", type=int, default=16)
    ap.add_argument("--no-side-workloads", action="store_true",
                    help="default run: skip the Proth n=2M and 4096-candidate batch sub-objects")
    ap.add_argument("--side-batch-window", type=float, default=15.0)
    args = ap.parse_args()
    world, rank, local, pg = dist_setup()
    if args.workload == "batch":
        # candidates shard across ranks (each rank its own runner)
        line = run_batch_workload(args, world, rank, local, pg)
        line["n_gpus"] = world
        if pg is not None:
            pg.destroy_process_group()
        if rank == 0:
            print(json.dumps(line), flush=True)
        return
    if args.workload != "square33M":
        # single-test latency workloads: one GPU (rank 0); other ranks have no work
        if rank == 0:
            fn = {"proth2M": run_proth2m_workload, "serve": run_serve_workload, "table": run_table_workload}[args.workload]
            print(json.dumps(fn(args)), flush=True)
        if pg is not None:
            pg.destroy_process_group()
        return
    if args.impl == "reference":
        line = run_reference(args, world, rank, pg)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    line, regs = run_ours(args, world, rank, local, pg)
    if pg is not None:
        pg.destroy_process_group()
    if rank != 0:
        return
    res = None
    if not args.no_cpu_baseline:
        try:
            # rank 0: the reference over the parity window (at N > 1 one process,
            # only to check this rank's registers)
            procs = None if world == 1 else 1
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import cpu_baseline
            res = cpu_baseline.run(BITS, SEED, BASE, squarings=PARITY_WINDOW, procs=procs)
        except RuntimeError as e:
            res = None
            sys.stderr.write("no reference run: %s\n" % e)
    if res is not None and world == 1:
        line["cpu_baseline"] = {
            "value": round(res["value_us"], 3), "unit": UNIT, "cores": res["cores"], "kind": "reference",
            "sample": "reference transformCPU compiled from its sources, %d processes x %d squarings (the first test-loop "
                      "iterations) at 33.2M bits, set-up untimed; one core: %.0f us/squaring"
                      % (res["cores"], PARITY_WINDOW, res["single_us"])}
    line["parity"] = parity_record(regs, res)
    if world == 1 and not args.no_side_workloads:
        # the other configurations the driver should see measured: the full
        # 262,144-bit test (C1), the Proth n = 2,000,000 test (C2), the
        # 4096-candidate batch (C4) and the serving window (C5)
        line["c1"] = side_c1()
        line["proth2M"] = side_proth2m(args)
        line["batch"] = side_batch(args)
        lo, hi = args.serve_bits
        line["serve"] = serve_one_rate(args.side_serve_rate, args.side_serve_window, lo, hi, 1007,
                                       latency_ln=args.serve_latency_ln, epoch_us=args.serve_epoch_us)
    print(json.dumps(line), flush=True)
    if line["parity"]["checked"] and not line["parity"]["equal"]:
        sys.stderr.write("PARITY FAILURE: registers differ from the reference after the window\n")
        sys.exit(3)


if __name__ == "__main__":
    main()
