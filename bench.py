#!/usr/bin/env python
"""Benchmark: RNS walk prime-steps/s on B200 (one JSON line on rank 0).

Workload (default, the uniform PCF batch): 4096 seeded PCFs, deg a <= 2,
deg b <= 4, coefficients in [-10, 10]; m = 2, K = 32.  Each PCF is walked to
depth 8000 with its depth-2000 convergent taken on the way; one step =
walk (residues + FP64 shadow at both depths) -> CRT of p, q at both depths
-> Dreams delta of the depth-2000 convergent against the PCF's own
depth-8000 convergent -> top-100 by delta, all on the device.
One prime-step = one (walk, prime, step); a step here is 4096 * 32 * 8000.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun each rank runs its own 4096 PCFs (weak scaling, no data-path
collective); the reported time is the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "dreams-rns-cuda_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "walk prime-steps/sec and p50/p99 request latency, bit-exact vs reference"
N_WALKS = 4096
DEPTH = 8000
CHECKPOINT = 2000
K = 32
TOPK = 100


def _compile(ab):
    import dreams_rns as dr
    return dr.compile_pcf(*ab).serialize()


def workload(seed: int):
    import dreams_rns as dr
    return dr.synth.uniform_pcfs(N_WALKS, seed=seed, depth=CHECKPOINT, limit_depth=DEPTH, K=K)


def compile_all(ws):
    with mp.get_context("spawn").Pool(min(os.cpu_count() or 4, 16)) as pool:
        return pool.map(_compile, [(w.a, w.b) for w in ws], chunksize=32)


# ---- reference (CPU) side -----------------------------------------------------

def _ref_walk(args):
    """One workload walk through the numpy restatement of the reference
    (oracle/walk_np), plus CRT and mpmath delta like the device step."""
    blob, a0 = args
    from oracle import walk_np
    r = walk_np.pcf_walk(blob, a0, DEPTH, K, 1, checkpoints=(CHECKPOINT,))
    c = r["checkpoints"][CHECKPOINT]
    pr = [int(p) for p in r["primes"]]
    vals = []
    for res in (r["p_residues"], r["q_residues"], c["p_residues"], c["q_residues"]):
        x, M = walk_np.crt([int(v) for v in res], pr)
        vals.append(walk_np.centered(x, M))
    import mpmath as mp_
    mp_.mp.dps = 200
    L = mp_.mpf(vals[0]) / mp_.mpf(vals[1]) if vals[1] else mp_.mpf(0)
    return walk_np.delta_exact(vals[2], vals[3], L, 200)


def cpu_reference(blobs, ws, budget_s: float = 12.0):
    """Time the numpy restatement on a bounded sample with every host core."""
    cores = os.cpu_count() or 1
    n = max(cores, 2)
    sample = [(blobs[i], ws[i].a0) for i in range(n)]
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
    with mp.get_context("spawn").Pool(cores) as pool:
        pool.map(_ref_walk, sample[:cores])           # warm the workers
        t0 = time.perf_counter()
        done = 0
        while True:
            pool.map(_ref_walk, sample)
            done += len(sample)
            if time.perf_counter() - t0 > budget_s:
                break
        dt = time.perf_counter() - t0
    ps = done * K * DEPTH
    return {"value": ps / dt, "unit": "prime-steps/s", "cores": cores, "kind": "port",
            "sample": f"{done} of the workload's walks (depth 8000, checkpoint 2000, K=32) "
                      f"through oracle/walk_np (numpy restatement of runner.py) + CRT + mpmath "
                      f"delta, multiprocessing over {cores} cores, {dt:.1f} s"}


# ---- clocks -------------------------------------------------------------------

class ClockSampler:
    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def start(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.samples.append([v.strip() for v in out.split(",")])
            except Exception:  # noqa: BLE001 - sampling is best effort
                pass
            self._stop.wait(0.2)

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if len(s) > 3 + i and s[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


# ---- roofline accounting ------------------------------------------------------

def algorithmic_int_ops(info, K_, depth):
    """Integer lane-instructions one walk needs with the difference-table
    companion algorithm: per prime-step, D modular additions per stream
    (add + min) and for each of the m last-column entries m wide multiply-adds,
    2 per extra product beyond two (fold), and a Montgomery reduction (2 wide
    multiplies + add + min)."""
    m = 2
    D = max(info["degree"], 1)
    per = 2 * m * D + m * (m + 2 * max(0, m - 2) + 4)
    return per * K_ * depth


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    config = {"workload": "uniform PCF batch: 4096 seeded PCFs, deg a<=2, deg b<=4, coeffs in "
                          "[-10,10], m=2, depth 8000 with the depth-2000 convergent on the way, "
                          "K=32, delta(2000) vs own depth-8000 convergent, top-100",
              "walks_per_gpu": N_WALKS, "K": K, "depth": DEPTH, "checkpoint": CHECKPOINT,
              "parallelism": f"walk-sharded x{world}"}

    if args.impl == "reference":
        if rank != 0:
            return
        ws = workload(seed=2)
        blobs = compile_all(ws)
        cb = cpu_reference(blobs, ws)
        line = {"metric": METRIC, "value": cb["value"], "unit": "prime-steps/s", "impl": "reference",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": N_WALKS * K * DEPTH / cb["value"] * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
                "config": config, "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": "prime-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    ws = workload(seed=2 + 1000 * rank)
    blobs = compile_all(ws)          # process pool before the first GPU call

    import numpy as np
    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist_
        dist = dist_
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(local)

    import dreams_rns as dr
    from dreams_rns import _native as N
    from dreams_rns.engine import WalkBatch, pcf_request, run_walks

    N.init(local)
    reqs = [pcf_request(b, w.a0, DEPTH, K, checkpoint=CHECKPOINT) for b, w in zip(blobs, ws)]
    batch = WalkBatch(reqs)
    batch.set_pipeline(delta="self", topk=TOPK)
    stream = torch.cuda.Stream()       # a real stream: the legacy default stream's handle is 0
    torch.cuda.set_stream(stream)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")   # > 126 MB L2

    for _ in range(max(args.warmup, 3)):
        batch.run(stream.cuda_stream)
    torch.cuda.synchronize()

    sampler = ClockSampler(local)
    sampler.start()
    times = []
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        batch.run(stream.cuda_stream)
        e1.record(stream)
        times.append((e0, e1))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    total_ms = sum(a.elapsed_time(b) for a, b in times)
    t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    st = batch.stats()
    prime_steps = st["prime_steps"]
    value = prime_steps * world * args.steps / (total_ms * 1e-3)

    # correctness spot check of this run's top walk against the result dicts
    pipe = batch.read_pipeline()

    # ---- roofline: the walk kernels alone (no shadow, no pipeline)
    walk_only = WalkBatch([pcf_request(b, w.a0, DEPTH, K, checkpoint=CHECKPOINT, shadow=False)
                           for b, w in zip(blobs, ws)])
    for _ in range(3):
        walk_only.run(stream.cuda_stream)
    wt = []
    for _ in range(5):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        walk_only.run(stream.cuda_stream)
        e1.record(stream)
        wt.append((e0, e1))
    torch.cuda.synchronize()
    walk_ms = statistics.median(a.elapsed_time(b) for a, b in wt)
    infos = {}
    ops = 0
    for b in blobs:
        if b not in infos:
            infos[b] = N.program_info(b)
        ops += algorithmic_int_ops(infos[b], K, DEPTH)
    import ctypes
    peak = ctypes.c_double()
    N.check(N.lib().dr_bench_int_peak(2, ctypes.byref(peak)), "int peak")
    achieved = ops / (walk_ms * 1e-3)
    roofline = {"bound": "int", "achieved": achieved / 1e12, "peak": peak.value / 1e12,
                "unit": "Tops/s", "frac": achieved / peak.value, "traffic": None,
                "kernel": "k_walk (companion classes), walk-only batch, median of 5",
                "kernel_ms": walk_ms,
                "peak_source": "measured live: dr_bench_int_peak mix of mad.wide.u32 and add/min"}
    walk_only.close()

    # ---- end to end through the public API with host buffers: the walk
    # (descriptors and programs up, residues and shadows down), then CRT and
    # delta (residues up, limbs down, limbs up, deltas down)
    e2e_times = []
    h2d = d2h = 0
    n = len(reqs)
    for it in range(3):
        t0 = time.perf_counter()
        res = run_walks(reqs)
        p = np.stack([r["p_residues"] for r in res] + [r["checkpoint"]["p_residues"] for r in res]).astype(np.uint32)
        q = np.stack([r["q_residues"] for r in res] + [r["checkpoint"]["q_residues"] for r in res]).astype(np.uint32)
        pv = dr.crt_batch(p, K)
        qv = dr.crt_batch(q, K)
        targets = [((a if b > 0 else -a), abs(b)) for a, b in zip(pv[:n], qv[:n])]
        deltas = dr.delta_batch(pv[n:], qv[n:], targets)
        e2e_times.append(time.perf_counter() - t0)
    limbs = (31 * K + 31) // 32 + 2
    blob_bytes = sum(len(b) for b in set(blobs))
    h2d = (n * 72 + blob_bytes + n * 4 * 8          # descriptors, programs, axis parameters
           + p.nbytes + q.nbytes                    # residues into CRT
           + 2 * n * (limbs + 1) * 4 * 2 + n * (limbs + 1) * 4 * 2)   # limbs into delta
    d2h = (2 * 2 * n * K * 4 + 6 * n * 8 + n * 4    # residues, shadows, status
           + 2 * 2 * n * (limbs * 4 + 8)            # CRT limbs, signs, lengths
           + n * 8)                                  # deltas
    e2e_s = statistics.median(e2e_times)
    e2e_val = prime_steps * world / e2e_s
    n_launch = int(st["launches"]) + 1 + 1 + 1     # walk/shadow groups + CRT + delta + top-k

    line = {"metric": METRIC, "value": value, "unit": "prime-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded PCF generator; the reference's datasets are not shipped)",
            "config": dict(config, l2="flushed: 512 MB write between timed steps",
                           timing="CUDA events on the launching stream, max over ranks"),
            "clocks": clocks,
            "e2e": {"value": e2e_val, "unit": "prime-steps/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "seconds_per_step": e2e_s,
                    "path": "run_walks + crt_batch + delta_batch (host buffers)"},
            "gpu_launches": n_launch,
            "roofline": roofline,
            "top1_delta": float(pipe["topk_val"][0]) if len(pipe["topk_val"]) else None}
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_reference(blobs, ws)
    batch.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
