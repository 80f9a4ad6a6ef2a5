#!/usr/bin/env python
"""Benchmark of the B200 Flock prover: verified BLAKE3 compressions per second.

A step is one complete proof of 2^18 independent BLAKE3 compressions (the
reference's ranked workload: benchmark-tools/worker, README.md:17-31): inputs
from the benchmark generator's seed, witness -> commit -> zerocheck ->
lincheck -> ring switch -> Ligerito open -> FLOCK bytes.  Every proof is
byte-identical to the oracle, whose proofs the reference's verifier accepts
(tests/test_gpu_parity.py).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU runs are replicas (proofs are independent): each rank proves its
own seeds, timing is the max over ranks of the device time.
"""
import argparse
import json
import multiprocessing as mp
import os
import random
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "flock-challenge-multi_b200"))

LOG2 = 18
METRIC = "verified BLAKE3 compressions/sec on 1 B200 (2^18/proof); p50/p99 proof latency served"
PUBLISHED_CPU = 381080.0  # reference, c7i.4xlarge 16 vCPU (README.md:95-98)
SERVE_SLOTS = 4  # proofs in flight in the continuous-batching queue
BATCH_THREADS = 8  # host threads (one stream each) driving the batched proofs' transcript phases
def algorithmic_bytes(phase: str, log2: int) -> int:
    """Minimum HBM bytes of one proof phase: the data the phase must read and
    write once, whatever the implementation (m = 14 + log2 witness bits;
    packed vectors hold 2^(m-7) F128 values; the commitment has 64 lanes, rate
    1/2, 2^(m-13) message positions and 2^(m-12) leaves of 1 KiB)."""
    m = 14 + log2
    n = 1 << (m - 7)  # F128 values of one packed vector (z, a, b, b_combined)
    return {
        # read the 2^(m-7)-value message, write the 2^(m-6)-value codeword
        "rs_encode": 16 * n + 16 * 2 * n,
        # read the codeword (leaves x 1 KiB), write 32 B per leaf CV
        "merkle_commit": (1 << (m - 12)) * 1024 + 32 * (1 << (m - 12)),
        # write z, a, b (2^m bits each)
        "witness": 3 * (1 << m) // 8,
        # read a, b, c (c = z)
        "zerocheck_round1": 3 * (1 << m) // 8,
        # packed a, b read once, then per round over k values per vector
        # 2 x 16 k read + 16 k written, k from 2^(m-7) halving
        "zerocheck_rounds": 2 * (1 << m) // 8 + 48 * 2 * n,
        # the z-fold reads z
        "lincheck": (1 << m) // 8,
        # per claim (two): read z, write a 2^(m-7)-value vector
        "ring_switch_combine": 2 * ((1 << m) // 8 + 16 * n),
        # 6 rounds over f and b: 2 x 16 k per round, k from 2^(m-7) halving
        "ligerito_l0_folds": 2 * 16 * 2 * n,
        # the first recursive level's codeword (2^(m-11) values) written and read
        "ligerito_levels": 2 * 16 * (1 << (m - 11)),
    }[phase]


# phase -> (the phase's kernels, launches per proof, what the algorithmic bytes count)
PHASE_KERNEL = {
    "rs_encode": ("k_ntt_pass_w (4-bit table passes; the first reads the message)", 0,
                  "read the message (2^25 F128), write the codeword (2^26 F128)"),
    "merkle_commit": ("k_merkle_leaves/parents/top", 22, "read the 1 GiB codeword, write 32 B per leaf"),
    "zerocheck_round1": ("k_zc_round1_ab + k_zc_round1_c", 2, "read packed a, b, c (3 x 512 MiB)"),
    "zerocheck_rounds": ("k_zc_round", 26, "packed a, b once, then 3 x 16 B per value per halving round"),
    "ring_switch_combine": ("k_bcombined_ct", 2, "per claim: read z, write 2^25 F128"),
    "ligerito_l0_folds": ("k_lig_fold_msg", 12, "6 rounds over f, b (2 x 512 MiB, halving)"),
    "lincheck": ("k_lc_zvec", 12, "read z (512 MiB)"),
    "witness": ("k_witness_seed", 1, "write z, a, b (3 x 512 MiB)"),
    "ligerito_levels": ("levels", 60, "the first recursive level's codeword written and read"),
}

# GF(2^128) products per proof of the RS encode: 64 lanes x 2^19 pairs x 19
# butterfly layers at m = 32 (layer 0 is a copy)
NTT_PRODUCTS_2P18 = 64 * (1 << 19) * 19
def peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks + throttle reasons sampled during the timed region."""

    def __init__(self, device: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(device), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait(timeout=10)
        self.f.seek(0)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_backend() -> str:
    """nccl between GPU ranks; FLOCK_DIST_BACKEND=gloo runs the same plumbing on CPU."""
    return os.environ.get("FLOCK_DIST_BACKEND", "nccl")


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if dist_backend() == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(dist_backend(), timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def allreduce_max(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def rank_seed_base(rank: int) -> int:
    """Every replica proves its own inputs (distinct seeds per rank)."""
    return 0x5EED0000 + 1_000_003 * rank


def aggregate(local_ms: float, world: int, log2: int, steps: int):
    """Whole-job throughput of `world` replicas: all ranks' compressions over
    the slowest rank's device time.  Returns (value, max_ms)."""
    max_ms = allreduce_max(local_ms, world)
    return (1 << log2) * steps * world / (max_ms / 1e3), max_ms


def host_blocks(log2: int, seed: int):
    """Benchmark inputs on the host (the library's generate_compressions)."""
    import flockgpu
    return flockgpu.generate_compressions(log2, seed)


def cpu_baseline_sample() -> dict:
    """The oracle (CPU restatement of the reference prover) on a bounded sample."""
    sys.path.insert(0, str(REPO / "tests"))
    lib = REPO / "oracle/_build/libflockref.so"
    if not lib.exists():
        subprocess.run(["make", "-C", str(REPO / "oracle")], check=True, capture_output=True)
    import oracle_lib
    o = oracle_lib.Oracle()
    log2 = 12
    secs, _ = o.time_prove(log2, 1)
    return {"value": (1 << log2) / secs, "unit": "compressions/s", "cores": 1, "kind": "port",
            "sample": f"one 2^{log2}-compression proof by the single-threaded oracle ({secs:.1f} s); "
                      f"the reference's published figure is {PUBLISHED_CPU:.0f} c/s on 16 vCPU"}


def run_reference(args, world, rank):
    if rank != 0:
        return
    sys.path.insert(0, str(REPO / "tests"))
    lib = REPO / "oracle/_build/libflockref.so"
    if not lib.exists():
        subprocess.run(["make", "-C", str(REPO / "oracle")], check=True, capture_output=True)
    import oracle_lib
    log2 = 10
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    # one single-threaded oracle proof per host core, run concurrently: a step is
    # `cores` proofs of 2^10 compressions (a bounded sample of the 2^18 workload)
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        pool.map(_oracle_proof, [(log2, 1000 + i) for i in range(cores)] * max(args.warmup, 1))
        times = []
        for i in range(args.steps):
            t0 = time.perf_counter()
            pool.map(_oracle_proof, [(log2, 2000 + 97 * i + c) for c in range(cores)])
            times.append(time.perf_counter() - t0)
    tot = sum(times)
    value = args.steps * cores * (1 << log2) / tot
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "compressions/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": value / PUBLISHED_CPU, "dtype": "gf2^128/u32",
        "data": "synthetic (benchmark SplitMix64 generator)",
        "config": {"workload": f"{cores} concurrent proofs of 2^{log2} BLAKE3 compressions per step (bounded CPU "
                               f"sample of the 2^18 workload)", "log2": log2,
                   "parallelism": f"cpu, {cores} processes x 1 thread"},
        "cpu_baseline": {"value": value, "unit": "compressions/s", "cores": cores, "kind": "port",
                         "sample": f"{args.steps} steps of {cores} concurrent oracle proofs of 2^{log2} compressions "
                                   f"(the reference Rust prover cannot be built here: no cargo/rustc)"},
        "e2e": {"value": value, "unit": "compressions/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _oracle_proof(job):
    log2, seed = job
    sys.path.insert(0, str(REPO / "tests"))
    import oracle_lib
    return oracle_lib.Oracle().time_prove(log2, seed)[0]


def splitmix64(seed: int):
    """The benchmark's SplitMix64 stream (benchmark-tools/common/src/lib.rs)."""
    state = seed & (2**64 - 1)
    while True:
        state = (state + 0x9E3779B97F4A7C15) & (2**64 - 1)
        z = state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & (2**64 - 1)
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & (2**64 - 1)
        yield z ^ (z >> 31)


def job_mix(n: int, lo: int, hi: int, seed: int):
    """n jobs, log2 log-uniform over [lo, hi] (log2 = lo + floor(u (hi - lo + 1))), own seeds."""
    g = splitmix64(seed)
    return [(lo + (next(g) * (hi - lo + 1) >> 64), next(g)) for _ in range(n)]


def plain_seconds(ctx, jobs, per_job=False):
    """Wall time of the jobs proved one at a time through the plain entry point
    (setups made beforehand, untimed); with per_job, also each job's own
    time alone (ms), in job order."""
    import flockgpu
    provers = {l: flockgpu.Prover(ctx, l) for l in sorted({l for l, _ in jobs})}
    try:
        for l, p in provers.items():
            p.prove_seed(1)  # warm
        each = []
        t0 = time.perf_counter()
        for l, s in jobs:
            t1 = time.perf_counter()
            provers[l].prove_seed(s)
            each.append((time.perf_counter() - t1) * 1e3)
        total = time.perf_counter() - t0
        return (total, each) if per_job else total
    finally:
        for p in provers.values():
            p.close()


# size classes of the served report (log2 ranges, inclusive)
SIZE_CLASSES = ((10, 12), (13, 16), (17, 18), (19, 20))


def by_size_class(jobs, lat, alone, parts=None):
    """p50 / p99 latency per size class, beside the same jobs' latency alone;
    with parts, also where the slowest job of the class spent its time."""
    out = []
    for lo, hi in SIZE_CLASSES:
        idx = [i for i, (l, _) in enumerate(jobs) if lo <= l <= hi]
        if not idx:
            continue
        L, A = [lat[i] for i in idx], [alone[i] for i in idx]
        out.append({"log2": [lo, hi], "jobs": len(idx), "p50_ms": pct(L, 0.5), "p99_ms": pct(L, 0.99),
                    "alone_p50_ms": pct(A, 0.5), "alone_p99_ms": pct(A, 0.99),
                    "p99_over_alone_p99": pct(L, 0.99) / pct(A, 0.99)})
        if parts:
            w = max(idx, key=lambda i: lat[i])
            out[-1]["slowest"] = {"log2": jobs[w][0], "latency_ms": lat[w], "queue_ms": parts[w][0],
                                  "run_ms": parts[w][1], "alone_ms": alone[w]}
    return out


def served_run(ctx, jobs, rate=None):
    """Submit the jobs (all at once, or Poisson arrivals at `rate` jobs/s) and
    collect them; returns (wall seconds, latencies in ms, (queue ms, run ms) per job)."""
    rng = random.Random(7)
    t0 = time.perf_counter()
    tickets, when = [], 0.0
    for l, s in jobs:
        if rate:
            when += rng.expovariate(rate)
            dt = t0 + when - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
        tickets.append(ctx.submit(l, s))
    res = [ctx.poll(t) for t in tickets]
    return time.perf_counter() - t0, [r["latency_ms"] for r in res], [(r["queue_ms"], r["run_ms"]) for r in res]


def pct(v, q):
    v = sorted(v)
    k = (len(v) - 1) * q
    i = int(k)
    return v[i] + (v[min(i + 1, len(v) - 1)] - v[i]) * (k - i)


def serving_report(device: int, full: bool, slots: int = SERVE_SLOTS, threads: int = BATCH_THREADS):
    """Batched (64 uneven jobs, 2^12..2^18, all at once) and served (Poisson
    arrivals, p50/p99) against the plain one-proof-at-a-time form."""
    import flockgpu
    out = {}
    ctx = flockgpu.Context(device, hbm_budget_bytes=150 << 30)
    try:
        lo, hi = (10, 20) if full else (10, 18)
        batch_jobs = job_mix(64, 12, 18, 3)
        serve_jobs = job_mix(48 if not full else 96, lo, hi, 4)
        # the plain one-at-a-time times first, before the serving cache holds
        # its setups (the plain provers' memory is outside that budget)
        plain_batch = plain_seconds(ctx, batch_jobs)
        plain_serve, alone_serve = plain_seconds(ctx, serve_jobs, per_job=True)
        ctx.serve_start(slots)
        jobs = batch_jobs
        n = sum(1 << l for l, _ in jobs)
        ctx.prove_batch(jobs, threads=threads)  # warm: setups of every size cached
        t0 = time.perf_counter()
        res = ctx.prove_batch(jobs, threads=threads)
        wall = time.perf_counter() - t0
        lat = [r["latency_ms"] for r in res]
        cwall, clat, _ = served_run(ctx, jobs)  # the same jobs through the continuous-batching queue
        # and once more with every proof verified before it is returned
        ctx.serve_verify(True)
        vwall, vlat, _ = served_run(ctx, jobs)
        ctx.serve_verify(False)
        plain = plain_batch
        out["batched"] = {"jobs": len(jobs), "log2_range": [12, 18], "compressions": n,
                          "value": n / wall, "unit": "compressions/s", "plain_value": n / plain,
                          "speedup_vs_plain": plain / wall, "p50_ms": pct(lat, 0.5), "p99_ms": pct(lat, 0.99),
                          "threads": threads,
                          "form": "flock_prove_batch: fused witness + commit graphs over groups of 8 jobs, "
                                  "each overlapping the earlier groups' remaining phases on concurrent streams",
                          "continuous": {"value": n / cwall, "p50_ms": pct(clat, 0.5), "p99_ms": pct(clat, 0.99),
                                         "slots": slots},
                          "continuous_self_checked": {"value": n / vwall, "p50_ms": pct(vlat, 0.5),
                                                      "p99_ms": pct(vlat, 0.99), "slots": slots,
                                                      "form": "every proof verified (flock_verify) before it "
                                                              "is returned"}}
        jobs = serve_jobs
        n = sum(1 << l for l, _ in jobs)
        served_run(ctx, jobs)  # warm
        plain = plain_serve
        cap = len(jobs) / plain  # plain capacity in jobs/s for this size mix
        rates = [0.25, 0.5, 1.0, 2.0] if full else [1.0]
        out["served"] = []
        for f in rates:
            wall, lat, parts = served_run(ctx, jobs, rate=f * cap)
            out["served"].append({"arrival_rate_x_plain_capacity": f, "jobs": len(jobs), "log2_range": [lo, hi],
                                  "p50_ms": pct(lat, 0.5), "p99_ms": pct(lat, 0.99),
                                  "sustained_value": n / wall, "plain_value": n / plain,
                                  "unit": "compressions/s", "slots": slots,
                                  "hbm_budget_gb": 150,
                                  "by_size_class": by_size_class(jobs, lat, alone_serve, parts)})
    finally:
        ctx.close()
    return out


# Ceiling of the GF(2^128) product as built here (not an algorithmic bound: a
# cheaper product raises it): 144 IMAD.WIDE (9 Karatsuba 32x32 carry-less
# products of 16 each) at 32 per SM per clock, the FMA pipe's rate.  148 SMs
# at the measured maximum SM clock.
def sm_mhz() -> float:
    mhz = 1965.0
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        mhz = float(json.loads(p.read_text()).get("sm_max_mhz", mhz))
    return mhz


def int_product_peak() -> float:
    return 148 * sm_mhz() * 1e6 * 32 / 144


# Ceiling of the 4-bit window table product: 64 eight-byte lookups (512 B) per
# product on the shared-memory pipe, 128 B per SM per clock.
def table_product_peak() -> float:
    return 148 * sm_mhz() * 1e6 * 128 / 512


def product_ceiling(plan_desc: str) -> tuple:
    """(ceiling, definition) of the GF(2^128) product as the tuned plan's
    passes compute it: integer multiplies, table lookups, or both pipes at
    once (the mixed passes send half of the lanes each way)."""
    if "/tab+imad" in plan_desc:
        return 2 * min(int_product_peak(), table_product_peak()), "mixed: both pipes, half of the products each"
    if "/tab" in plan_desc:
        return table_product_peak(), "4-bit window tables: 148 SMs x max SM clock x 128 B / 512 B per product"
    return int_product_peak(), ("integer products: 148 SMs x max SM clock x 32 IMAD.WIDE per SM per clock / "
                                "144 IMAD.WIDE per product")


def round1_deg4_rows(ctx, hbm: float, sizes=(16, 18, 20, 22, 24, 26)) -> list:
    """Degree-4 zerocheck round 1 (round1_deg4_naive's message, the sizes of
    benches/round1_deg4.rs): device-resident seeded bit vectors, mean device
    time of one message (eq table + kernel).  Algorithmic bytes: the five bit
    vectors (5 * 2^m / 8) and the eq table (16 * 2^(m-6), written and read)."""
    out = []
    for m in sizes:
        ms, _, _ = ctx.bench_round1_deg4(m, 0xDEC0DE ^ m, iters=5)
        byts = 5 * (1 << m) // 8 + 2 * 16 * (1 << (m - 6))
        out.append({"kernel": "zerocheck_round1_deg4", "m": m, "ms": ms, "constraints_per_s": (1 << m) / (ms / 1e3),
                    "gbs": byts / (ms / 1e3) / 1e9, "hbm_frac": byts / (ms / 1e3) / 1e9 / hbm,
                    "l2_resident": byts < (126 << 20)})
    return out


def kernel_report(device: int) -> list:
    """Kernel microbenchmarks (additive NTT / RS encode, Merkle trees, degree-2
    and degree-3 sumcheck rounds) on device-resident seeded inputs, CUDA-event
    timed on the launching stream; each size is above the 126 MB L2 or is
    reported as L2-resident."""
    import flockgpu
    ctx = flockgpu.Context(device)
    hbm, kind = peaks()
    ipk = int_product_peak()
    rows = []
    try:
        for variant, name in ((0, "integer (bit classes + Karatsuba)"), (1, "4-bit window table"), (2, "half each"),
                              (3, "8-bit window table, one per CTA")):
            rate = ctx.bench_f128_product(variant)
            rows.append({"kernel": "f128_product_by_warp_constant", "variant": name, "products_per_s": rate,
                         "int_frac": rate / ipk})
        for log_msg, cols in [(16, 1), (16, 64), (16, 256), (20, 1), (20, 16), (20, 64), (24, 1), (24, 4)]:
            for rate in (1, 2):
                if log_msg + cols.bit_length() - 1 + rate > 27:
                    continue
                ms = ctx.bench_ntt(log_msg, cols, rate, iters=5)
                n_cw = (1 << (log_msg + rate)) * cols
                prods = cols * (n_cw // cols // 2) * log_msg  # layers rate..log_d-1, one product per pair
                byts = 16 * cols * (1 << log_msg) + 16 * n_cw  # algorithmic: read the message, write the codeword
                rows.append({"kernel": "ntt_rs_encode", "log_msg": log_msg, "columns": cols, "rate": f"1/{1 << rate}",
                             "ms": ms, "gf_products_per_s": prods / (ms / 1e3),
                             "int_frac": prods / (ms / 1e3) / ipk, "gbs": byts / (ms / 1e3) / 1e9,
                             "hbm_frac": byts / (ms / 1e3) / 1e9 / hbm, "l2_resident": 16 * n_cw < (126 << 20)})
        for log_l in (16, 19, 22):
            for size in (32, 64, 128, 256, 512, 1024):
                if (size << log_l) > (4 << 30):
                    continue
                ms = ctx.bench_merkle(1 << log_l, size, iters=5)
                comps = (1 << log_l) * ((size + 63) // 64) + (1 << log_l) - 1
                byts = (size << log_l) + 32 * ((2 << log_l) - 1)
                rows.append({"kernel": "merkle_tree", "leaves": 1 << log_l, "leaf_bytes": size, "ms": ms,
                             "blake3_compressions_per_s": comps / (ms / 1e3), "gbs": byts / (ms / 1e3) / 1e9,
                             "hbm_frac": byts / (ms / 1e3) / 1e9 / hbm, "l2_resident": byts < (126 << 20)})
        for log_n in (16, 20, 24):
            n = 1 << log_n
            ms = ctx.bench_sumcheck(n, iters=5)
            byts = 16 * (2 * n + n)  # read f, b; write the folded halves
            prods = 3 * (n // 2)      # fold: 1 per output value (n / 2); message: 2 per output pair
            rows.append({"kernel": "sumcheck_deg2_fold_round", "n": n, "ms": ms, "gbs": byts / (ms / 1e3) / 1e9,
                         "hbm_frac": byts / (ms / 1e3) / 1e9 / hbm, "gf_products_per_s": prods / (ms / 1e3),
                         "int_frac": prods / (ms / 1e3) / ipk, "l2_resident": 16 * 2 * n < (126 << 20)})
            ms = ctx.bench_sumcheck3(n, iters=5)
            byts = 16 * (2 * n + n + n // 4)  # read a, b, e; write the folded halves
            prods = 2 * n                     # fold: 1 per output value (n / 2); message: 4 per output pair
            rows.append({"kernel": "sumcheck_deg3_fold_round", "n": n, "ms": ms, "gbs": byts / (ms / 1e3) / 1e9,
                         "hbm_frac": byts / (ms / 1e3) / 1e9 / hbm, "gf_products_per_s": prods / (ms / 1e3),
                         "int_frac": prods / (ms / 1e3) / ipk, "l2_resident": 16 * 2 * n < (126 << 20)})
        rows += round1_deg4_rows(ctx, hbm)
    finally:
        ctx.close()
    for r in rows:
        r["hbm_peak_gbs"] = hbm
        r["peak_kind"] = kind
        r["int_product_peak_per_s"] = ipk
    return rows


def chain_report(prover, log2: int, steps: int = 5) -> dict:
    """The BLAKE3 hash-chain statement (Blake3Setup::prove_chain) on the same
    setup: the flock_chain CLI's honest chain of 2^log2 compressions, proved
    end to end through flock_prove_chain from pinned host records (H2D of the
    records, prove, D2H of the bundle), timed on the host clock; the device
    time is the sum of the proof's phase events.  The region fold and the
    shift sumcheck fall in the ring-switch phase."""
    import flockgpu
    recs = flockgpu.PinnedArray((1 << log2, 28), np.uint32)
    recs.array[:] = flockgpu.chain_blocks(0x5EED, 1 << log2)
    for _ in range(2):
        prover.prove_chain(recs.array)
    wall, dev = [], []
    for _ in range(steps):
        t0 = time.perf_counter()
        size = len(prover.prove_chain(recs.array))
        wall.append(time.perf_counter() - t0)
        ph = prover.phase_ms()
        dev.append(sum(ph.values()))
    n = 1 << log2
    e2e = pct(wall, 0.5)
    dms = pct(dev, 0.5)
    return {"chain": {"statement": f"hash chain of 2^{log2} BLAKE3 compressions (cv_(i+1) = out_lo(compress(cv_i)))",
                      "log2": log2, "proofs": steps, "e2e_ms_median": e2e * 1e3,
                      "e2e_compressions_per_s": n / e2e, "device_ms_median": dms,
                      "device_compressions_per_s": n / (dms / 1e3), "proof_bytes": size,
                      "h2d_bytes_per_proof": n * 112, "phases_ms": {k: round(v, 3) for k, v in ph.items()}}}


def sha256_report(ctx, sizes=(16, 18), steps: int = 5) -> dict:
    """The SHA-256 compression statement (Sha256HybridSetup::prove_fast,
    r1cs_hashes/sha2.rs) on its own setups: 2^16 compressions (the largest
    default size of the reference's benches/sha2_proof.rs) and 2^18 (the
    headline's count), inputs from that bench's generator.  Device time is
    the sum of the proof's phase events (seeded inputs generated on the GPU);
    e2e goes through flock_sha256_prove from pinned host compressions (H2D of
    the records, prove, D2H of the bundle), host clock, medians of `steps`."""
    import flockgpu
    rows = []
    for log2 in sizes:
        n = 1 << log2
        prover = flockgpu.Sha256Prover(ctx, n)
        comps = flockgpu.PinnedArray((n, 24), np.uint32)
        comps.array[:] = flockgpu.sha256_bench_inputs(n, flockgpu.sha256_bench_seed(n))
        for _ in range(2):
            prover.prove(comps.array)
        dev, wall = [], []
        for i in range(steps):
            prover.prove_seed(flockgpu.sha256_bench_seed(n, i + 1))
            ph = prover.phase_ms()
            dev.append(sum(ph.values()))
        for _ in range(steps):
            t0 = time.perf_counter()
            size = len(prover.prove(comps.array))
            wall.append(time.perf_counter() - t0)
        why = prover.verify(prover.prove(comps.array))
        prover.close()
        if why:
            raise SystemExit(f"sha256_report: proof rejected: {why}")
        d, e = pct(dev, 0.5), pct(wall, 0.5)
        rows.append({"log2": log2, "m": 15 + log2, "device_ms_median": d, "device_compressions_per_s": n / (d / 1e3),
                     "e2e_ms_median": e * 1e3, "e2e_compressions_per_s": n / e, "proof_bytes": size,
                     "h2d_bytes_per_proof": n * 96, "phases_ms": {k: round(v, 3) for k, v in ph.items()}})
    # Merkle paths (prove_merkle_path_ligerito) at the Merkle bench's largest
    # size, 2^15 hashes on one path (benches/sha2_merkle_proof.rs:264-268)
    n_log = 15
    comps, b, leaves, root = flockgpu.sha256_merkle_inputs(n_log)
    prover = flockgpu.Sha256Prover(ctx, 1 << n_log)
    for _ in range(2):
        prover.prove_merkle(comps, b)
    wall = []
    for _ in range(steps):
        t0 = time.perf_counter()
        size = len(prover.prove_merkle(comps, b))
        wall.append(time.perf_counter() - t0)
    ph = prover.phase_ms()
    why = ctx.sha256_merkle_verify(prover.prove_merkle(comps, b), 0, b, leaves, root)
    prover.close()
    if why:
        raise SystemExit(f"sha256_report: Merkle-path proof rejected: {why}")
    e = pct(wall, 0.5)
    merkle = {"log2": n_log, "paths": 1, "e2e_ms_median": e * 1e3, "e2e_hashes_per_s": (1 << n_log) / e,
              "proof_bytes": size, "phases_ms": {k: round(v, 3) for k, v in ph.items()}}
    return {"sha256": {"statement": "SHA-256 compressions, one per 2^15-bit block (hybrid R1CS, sha2.rs)",
                       "proofs": rows, "merkle_path": merkle}}


KECCAK_SIZES = (6144, 8192, 12288, 24576, 65536)


def keccak_report(ctx, sizes=KECCAK_SIZES, steps: int = 5, widths=(1, 3)) -> dict:
    """The Keccak-f[1600] statements (KeccakSetup::prove_fast of r1cs_hashes/
    keccak.rs, one permutation per 2^16-bit block, and of keccak3.rs, three
    per 2^17-bit block) at the permutation counts of the reference's
    benches/keccak3_proof.rs:301-305 (the single-vs-3-wide comparison) and at
    2^16, states from that bench's generator.  Device time is the sum of the
    proof's phase events (states generated on the GPU); e2e goes through
    flock_keccak_prove from pinned host states (H2D of the states, prove, D2H
    of the bundle), host clock, medians of `steps`."""
    import flockgpu
    rows = []
    for n, width in [(n, w) for w in widths for n in sizes]:
        prover = flockgpu.KeccakProver(ctx, n, width=width)
        states = flockgpu.PinnedArray((n, 25), np.uint64)
        states.array[:] = flockgpu.keccak_bench_inputs(n, flockgpu.keccak_bench_seed(n))
        for _ in range(2):
            prover.prove(states.array)
        dev, wall = [], []
        for i in range(steps):
            prover.prove_seed(flockgpu.keccak_bench_seed(n, i + 1))
            ph = prover.phase_ms()
            dev.append(sum(ph.values()))
        for _ in range(steps):
            t0 = time.perf_counter()
            size = len(prover.prove(states.array))
            wall.append(time.perf_counter() - t0)
        why = ctx.keccak_verify(prover.prove(states.array), width=width)
        prover.close()
        if why:
            raise SystemExit(f"keccak_report: proof rejected: {why}")
        d, e = pct(dev, 0.5), pct(wall, 0.5)
        n_log = max(3, (-(-n // width) - 1).bit_length())
        rows.append({"n": n, "encoder": "keccak.rs" if width == 1 else "keccak3.rs (3-wide)",
                     "m": (16 if width == 1 else 17) + n_log, "device_ms_median": d,
                     "device_permutations_per_s": n / (d / 1e3),
                     "e2e_ms_median": e * 1e3, "e2e_permutations_per_s": n / e, "proof_bytes": size,
                     "h2d_bytes_per_proof": n * 200, "phases_ms": {k: round(v, 3) for k, v in ph.items()}})
    return {"keccak": {"statement": "Keccak-f[1600] permutations: one per 2^16-bit block (keccak.rs) and three "
                                    "per 2^17-bit block (keccak3.rs)", "proofs": rows}}


def verify_report(prover, log2: int, reps: int = 3) -> dict:
    """The verifier behind flock_verify on this setup: one compression proof
    and one chain proof of 2^log2 compressions, host wall clock per call
    (median of `reps`); the lincheck's matrix combination runs on the GPU."""
    import flockgpu
    proof = prover.prove_seed(0x7E57)
    chain = prover.prove_chain(flockgpu.chain_blocks(0x7E57, 1 << log2))
    out = {}
    for name, b, dom in (("compression", proof, flockgpu.DOMAIN), ("chain", chain, flockgpu.CHAIN_DOMAIN)):
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            why = prover.verify(b, dom)
            ts.append(time.perf_counter() - t0)
            if why:
                raise SystemExit(f"verify_report: {name} proof rejected: {why}")
        out[f"{name}_ms"] = pct(ts, 0.5) * 1e3
    return {"verify": {"log2": log2, **out, "threads": 1}}


def run_ours(args, world, rank, local):
    import flockgpu
    log2 = args.log2
    ctx = flockgpu.Context(local)
    prover = flockgpu.Prover(ctx, log2)
    _, plan_desc = ctx.ntt_autotune(log2 + 1, 64, 1)  # the commitment's tuned plan (tuned by the setup)
    seed_base = rank_seed_base(rank)
    for i in range(args.warmup):
        prover.prove_seed(seed_base + 900 + i)
    barrier(world)
    sampler = ClockSampler(local)
    total_ms, phases, launches = prover.bench(seed_base, args.steps)
    clocks = sampler.stop()
    value, max_ms = aggregate(total_ms, world, log2, args.steps)
    # end to end through the public API with host inputs in pinned memory: H2D
    # of the compressions, prove, D2H of the proof bytes (all inside the timed
    # region)
    pinned = []
    for i in range(args.steps):
        pa = flockgpu.PinnedArray((1 << log2, 25), np.uint32)
        pa.array[:] = host_blocks(log2, seed_base + 500 + i)
        pinned.append(pa)
    blocks = [pa.array for pa in pinned]
    # untimed warm-up of this entry point: its first call allocates the
    # device staging buffer and loads the host-input witness kernel
    prover.prove_blocks(host_blocks(log2, seed_base + 499))
    barrier(world)
    t0 = time.perf_counter()
    sizes = [len(prover.prove_blocks(b)) for b in blocks]
    e2e_s = allreduce_max(time.perf_counter() - t0, world)
    if rank != 0:
        prover.close()
        return
    n = (1 << log2) * args.steps * world
    peak, peak_kind = peaks()
    dom = max(phases, key=phases.get)
    kname, klaunches, kdesc = PHASE_KERNEL[dom]
    if dom == "rs_encode":  # one launch per pass of the tuned plan
        klaunches = plan_desc.count(" + ") + 1
        if "/tab" not in plan_desc:
            kname = "k_ntt_pass (integer products; the first pass reads the message)"
    kbytes = algorithmic_bytes(dom, log2)
    # the phase's events bracket only its own launches on the prover stream:
    # algorithmic bytes of the phase over the phase's device time
    achieved = kbytes / (phases[dom] / 1e3) / 1e9
    traffic = None
    tfile = REPO / "profiles" / "traffic.json"
    if tfile.exists():
        t = json.loads(tfile.read_text()).get(dom)
        if t:
            traffic = t * (1 << log2) / (1 << 18)  # DRAM bytes grow with the codeword
    line = {
        "metric": METRIC, "value": value, "unit": "compressions/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": value / PUBLISHED_CPU, "dtype": "gf2^128/u32", "data": "synthetic (benchmark SplitMix64 generator)",
        "config": {"workload": f"single proof of 2^{log2} BLAKE3 compressions (m={14 + log2}), Ligerito fast "
                               f"profile, BLAKE3 Merkle + transcript", "log2": log2, "proofs_per_step": 1,
                   "parallelism": f"replicas x{world}", "l2": "working set ~5 GB per proof > 126 MB L2",
                   "proof_bytes": sizes[0]},
        "baseline_anchor": {"published_cpu_value": PUBLISHED_CPU, "unit": "compressions/s",
                            "hardware": "reference Rust prover, c7i.4xlarge, 16 vCPU",
                            "value_ratio": value / PUBLISHED_CPU, "e2e_ratio": n / e2e_s / PUBLISHED_CPU},
        "e2e": {"value": n / e2e_s, "unit": "compressions/s", "h2d_bytes_per_step": (1 << log2) * 100,
                "d2h_bytes_per_step": sizes[0]},
        "gpu_launches": int(launches),
        "phases_ms": {k: round(v, 3) for k, v in phases.items()},
        "roofline": {"bound": "hbm", "kernel": kname, "phase": dom, "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "algorithmic_bytes": kbytes, "traffic_over_algorithmic": (traffic / kbytes) if traffic else None,
                     "launches": klaunches,
                     "note": f"per phase (its {klaunches} launches): {kdesc}; peak {peak_kind}"},
        "clocks": clocks,
    }
    if dom == "rs_encode":
        prods = NTT_PRODUCTS_2P18 * (1 << log2) / (1 << 18)
        rate = prods / (phases[dom] / 1e3)
        ceil, cdef = product_ceiling(plan_desc)
        line["roofline"]["int_pipe"] = {
            "plan": plan_desc, "products": prods, "achieved_products_per_s": rate,
            "ceiling_as_built_products_per_s": ceil, "utilisation_as_built": rate / ceil,
            "floor_ms_at_ceiling": prods / ceil * 1e3,
            "ceiling_def": cdef + " (the product as built, not an algorithmic bound)"}
    if world == 1 and not args.no_chain:
        line.update(chain_report(prover, log2))
        line.update(verify_report(prover, log2))
    if world == 1 and not args.no_sha256:
        line.update(sha256_report(ctx))
    if world == 1 and not args.no_keccak:
        line.update(keccak_report(ctx))
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sample()
    if world == 1 and not args.no_serve:
        prover.close()
        line.update(serving_report(local, full=False))
    print(json.dumps(line), flush=True)
    prover.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--log2", type=int, default=LOG2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serve", action="store_true", help="skip the batched / served measurements")
    ap.add_argument("--no-chain", action="store_true", help="skip the hash-chain measurement")
    ap.add_argument("--no-sha256", action="store_true", help="skip the SHA-256 statement measurement")
    ap.add_argument("--sha256", default=None, metavar="LOG2[,LOG2...]",
                    help="only the SHA-256 statement report at these sizes")
    ap.add_argument("--no-keccak", action="store_true", help="skip the Keccak statement measurement")
    ap.add_argument("--keccak", default=None, metavar="N[,N...]",
                    help="only the Keccak statement report at these permutation counts")
    ap.add_argument("--deg4", default=None, metavar="M[,M...]",
                    help="only the degree-4 zerocheck round-1 microbenchmark at these m")
    ap.add_argument("--ntt-case", default=None, metavar="LOG_MSG,LANES,RATE,PLAN",
                    help="one RS encode with candidate pass plan PLAN (no autotuning launches): the case that "
                         "the NTT's ncu captures profile")
    ap.add_argument("--ntt-plans", default=None, metavar="LOG_MSG,LANES,RATE",
                    help="time every candidate pass plan of one RS-encode shape (device-resident seeded inputs), "
                         "then the autotuner's pick; one JSON line")
    ap.add_argument("--proof-once", type=int, default=None, metavar="LOG2",
                    help="setup + one warm-up proof, print the library's kernel launches so far, then one more "
                         "proof: the case a profiler's launch list covers (skip the printed count)")
    ap.add_argument("--kernels", action="store_true",
                    help="only the kernel microbenchmarks (NTT / Merkle / sumcheck sweeps), one JSON line each")
    ap.add_argument("--slots", type=int, default=SERVE_SLOTS, help="serving: proofs in flight")
    ap.add_argument("--batch-threads", type=int, default=BATCH_THREADS, help="batched form: host threads")
    ap.add_argument("--serve", action="store_true",
                    help="only the batched + served report: 64 uneven jobs, then Poisson arrivals at 4 rates")
    args = ap.parse_args()
    world, rank, local = dist_setup() if args.impl == "ours" else (int(os.environ.get("WORLD_SIZE", "1")),
                                                                    int(os.environ.get("RANK", "0")), 0)
    if args.ntt_case:
        import flockgpu
        log_msg, lanes, rate, plan = (int(x) for x in args.ntt_case.split(","))
        ctx = flockgpu.Context(0)
        msg = np.random.default_rng(1).integers(0, 2**64, 2 * (lanes << log_msg), dtype=np.uint64)
        out = ctx.ntt_rs_encode_plan(msg, log_msg, lanes, rate, plan)
        ctx.close()
        if out is None:
            raise SystemExit(f"no candidate plan {plan} for this shape")
        print(json.dumps({"ntt_case": args.ntt_case, "codeword_values": int(out.size // 2)}))
        return
    if args.ntt_plans:
        import flockgpu
        lm, lanes, rate = (int(x) for x in args.ntt_plans.split(","))
        ctx = flockgpu.Context(0)
        plans = sorted((ctx.bench_ntt_plan(lm, lanes, rate, i, iters=5), i, d)
                       for i, d in enumerate(flockgpu.ntt_plan_descs(lm, lanes, rate)))
        t0 = time.perf_counter()
        _, pick = ctx.ntt_autotune(lm, lanes, rate)
        tune_s = time.perf_counter() - t0
        ms = ctx.bench_ntt(lm, lanes, rate, iters=5)
        prods = lanes * (1 << (lm + rate - 1)) * lm
        print(json.dumps({"log_msg": lm, "lanes": lanes, "rate": rate,
                          "plans": [{"ms": p[0], "index": p[1], "desc": p[2]} for p in plans],
                          "autotune": {"pick": pick, "tune_s": tune_s, "encode_ms": ms,
                                       "products_per_s": prods / (ms / 1e3)}}), flush=True)
        ctx.close()
        return
    if args.proof_once is not None:
        import flockgpu
        ctx = flockgpu.Context(0)
        prover = flockgpu.Prover(ctx, args.proof_once)
        prover.prove_seed(1)
        print(json.dumps({"launches_before_proof": int(flockgpu.load().flock_launch_count())}), flush=True)
        prover.prove_seed(2)
        prover.close()
        ctx.close()
        return
    if args.sha256:
        import flockgpu
        ctx = flockgpu.Context(0)
        print(json.dumps(sha256_report(ctx, tuple(int(x) for x in args.sha256.split(",")))), flush=True)
        ctx.close()
        return
    if args.deg4:
        import flockgpu
        ctx = flockgpu.Context(0)
        for row in round1_deg4_rows(ctx, peaks()[0], tuple(int(x) for x in args.deg4.split(","))):
            print(json.dumps(row), flush=True)
        ctx.close()
        return
    if args.keccak:
        import flockgpu
        ctx = flockgpu.Context(0)
        print(json.dumps(keccak_report(ctx, tuple(int(x) for x in args.keccak.split(",")))), flush=True)
        ctx.close()
        return
    if args.kernels:
        if rank == 0:
            for row in kernel_report(0):
                print(json.dumps(row), flush=True)
        return
    if args.serve:
        if rank == 0:
            print(json.dumps({"metric": "served/batched proof throughput and latency",
                              **serving_report(0, True, args.slots, args.batch_threads)}),
                  flush=True)
        return
    if args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_ours(args, world, rank, local)
    if world > 1 and args.impl == "ours":
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
