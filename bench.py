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
# the reference package, installed unmodified from its source by
#   pip install --no-index --no-build-isolation --no-deps --target baseline/_ref <reference>/python
REF_DIR = os.path.join(ROOT, "baseline", "_ref")

METRIC = "walk prime-steps/sec and p50/p99 request latency, bit-exact vs reference"
N_WALKS = 4096
DEPTH = 8000
CHECKPOINT = 2000
K = 32
TOPK = 100


def _use_repo_package():
    """Make ``import dreams_rns`` load this repository's package (the B200 arm)."""
    for p in (PKG, ROOT):
        if p not in sys.path:
            sys.path.insert(0, p)


def _standalone(name: str, filename: str):
    """Load one pure-Python module of the package by its path, without the
    package itself (whose ``__init__`` loads the native library)."""
    import importlib.util
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(PKG, "dreams_rns", filename))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod          # dataclasses resolve their module by name
    spec.loader.exec_module(mod)
    return mod


def _host_cores() -> int:
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except (AttributeError, OSError):
        return max(1, os.cpu_count() or 1)


def _compile(ab):
    import dreams_rns as dr
    return dr.compile_pcf(*ab).serialize()


def workload(seed: int):
    return _standalone("_bench_synth", "synth.py").uniform_pcfs(
        N_WALKS, seed=seed, depth=CHECKPOINT, limit_depth=DEPTH, K=K)


def compile_all(ws):
    with mp.get_context("spawn").Pool(min(_host_cores(), 16)) as pool:
        return pool.map(_compile, [(w.a, w.b) for w in ws], chunksize=32)


# ---- CPU legs: the reference's own walk, or the numpy port of it ---------------

def cpu_kind() -> str:
    """"reference" when the reference package is installed in baseline/_ref,
    else "port" (oracle/walk_np, the numpy restatement of its runner.py)."""
    return "reference" if os.path.isfile(os.path.join(REF_DIR, "dreams_rns", "runner.py")) else "port"


_CPU_KIND = None


def _cpu_init(kind: str):
    """Pool-worker set-up: ``import dreams_rns`` resolves to the installed
    reference (kind "reference"), never to this repository's package."""
    global _CPU_KIND
    _CPU_KIND = kind
    os.environ["OMP_NUM_THREADS"] = "1"
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    pkg = os.path.realpath(PKG)
    sys.path[:] = [p for p in sys.path if os.path.realpath(p or os.curdir) != pkg]
    if kind == "reference":
        sys.path.insert(0, REF_DIR)
        import dreams_rns  # noqa: F401  (the reference package)
    else:
        if ROOT not in sys.path:
            sys.path.insert(0, ROOT)
        from oracle import walk_np  # noqa: F401
    import mpmath  # noqa: F401


def _cpu_compile(ab):
    """Program bytes: the reference's own compile_pcf, or (port) this
    repository's pure-Python compiler loaded without the package."""
    if _CPU_KIND == "reference":
        import dreams_rns
        return dreams_rns.compile_pcf(*ab).serialize()
    return _standalone("_bench_compiler", "compiler.py").compile_pcf(*ab).serialize()


def _cpu_walk(task):
    """One workload walk on the CPU: residues at depth 8000 and 2000, CRT and
    the exact delta of the depth-2000 convergent against the depth-8000 one.
    The reference's run_pcf_walk has no checkpoint, so it walks twice."""
    blob, a0 = task
    if _CPU_KIND == "reference":
        import dreams_rns as ref
        prog = ref.CmfProgram.deserialize(blob)
        cp = ref.run_pcf_walk(prog, a0, CHECKPOINT, K)
        fin = ref.run_pcf_walk(prog, a0, DEPTH, K)
        crt, cen, dex = ref.crt_reconstruct, ref.centered, ref.compute_dreams_delta_exact
    else:
        from oracle import walk_np
        fin = walk_np.pcf_walk(blob, a0, DEPTH, K, 1, checkpoints=(CHECKPOINT,))
        cp = fin["checkpoints"][CHECKPOINT]
        crt, cen, dex = walk_np.crt, walk_np.centered, walk_np.delta_exact
    res = [fin["p_residues"], fin["q_residues"], cp["p_residues"], cp["q_residues"]]
    pr = [int(p) for p in fin["primes"]]
    vals = [cen(*crt([int(v) for v in r], pr)) for r in res]
    import mpmath
    mpmath.mp.dps = 200
    L = mpmath.mpf(vals[0]) / mpmath.mpf(vals[1]) if vals[1] else mpmath.mpf(0)
    d = dex(vals[2], vals[3], L, 200)
    return [[int(v) for v in r] for r in res], float(d)


def cpu_leg(pairs, blobs=None, passes=None, budget_s=12.0, warmup=0):
    """Run ``pairs`` = [(a, b, a0)] (one walk per host core) through the CPU
    path in timed passes on a spawn pool over every host core: ``passes``
    passes, or as many as ``budget_s`` allows (at least one).  Programs are
    compiled before the timed passes (the reference's compiler for kind
    "reference"; the given ``blobs`` for the port)."""
    kind = cpu_kind()
    cores = _host_cores()
    with mp.get_context("spawn").Pool(cores, initializer=_cpu_init, initargs=(kind,)) as pool:
        if blobs is None or kind == "reference":
            blobs = pool.map(_cpu_compile, [(a, b) for a, b, _ in pairs], chunksize=1)
        tasks = [(bl, a0) for bl, (_, _, a0) in zip(blobs, pairs)]
        for _ in range(warmup):
            pool.map(_cpu_walk, tasks, chunksize=1)
        times, first = [], None
        t_all = time.perf_counter()
        while True:
            t0 = time.perf_counter()
            out = pool.map(_cpu_walk, tasks, chunksize=1)
            times.append(time.perf_counter() - t0)
            if first is None:
                first = out
            if passes is not None:
                if len(times) >= passes:
                    break
            elif time.perf_counter() - t_all >= budget_s:
                break
    return {"kind": kind, "cores": cores, "walks": len(tasks), "pass_s": times, "outputs": first,
            "blobs": blobs}


def _cpu_what(kind: str) -> str:
    if kind == "reference":
        return ("the reference's own run_pcf_walk (twice: to depth 2000 and to 8000, it has no "
                "checkpoint) + crt_reconstruct + centered + compute_dreams_delta_exact, installed "
                "unmodified from its source into baseline/_ref")
    return ("oracle/walk_np (numpy restatement of the reference's runner.py; the reference package "
            "is not installed here) + CRT + mpmath delta")


def cpu_baseline_entry(leg) -> dict:
    total = sum(leg["pass_s"])
    done = leg["walks"] * len(leg["pass_s"])
    return {"value": done * K * DEPTH / total, "unit": "prime-steps/s", "cores": leg["cores"],
            "kind": leg["kind"],
            "sample": f"{done} walk runs over {len(leg['pass_s'])} passes of the workload's first "
                      f"{leg['walks']} PCFs (one per core; depth 8000 with the depth-2000 convergent, "
                      f"K=32) through {_cpu_what(leg['kind'])}; multiprocessing over {leg['cores']} "
                      f"cores, {total:.1f} s"}


def parity_vs_cpu(dev, delta, blobs, leg) -> dict:
    """The timed batch's results for the CPU leg's walks against the CPU
    outputs: p, q residues at both depths bit-exact, delta within 1e-9,
    program bytes identical."""
    bad = 0
    for i, (res, d) in enumerate(leg["outputs"]):
        r = dev[i]
        c = r["checkpoint"]
        same = (list(r["p_residues"]) == res[0] and list(r["q_residues"]) == res[1] and
                list(c["p_residues"]) == res[2] and list(c["q_residues"]) == res[3])
        g = float(delta[i])
        if math.isinf(d) or math.isinf(g) or math.isnan(d) or math.isnan(g):
            same &= (g == d) or (math.isnan(g) and math.isnan(d))
        else:
            same &= abs(g - d) <= 1e-9
        bad += not same
    prog_same = sum(bytes(a) == bytes(b) for a, b in zip(leg["blobs"], blobs))
    return {"walks": len(leg["outputs"]), "against": leg["kind"], "mismatches": bad,
            "programs_identical": prog_same,
            "checked": "p, q residues at depth 8000 and 2000 bit-exact, delta(2000 vs own 8000) "
                       "within 1e-9, program bytes"}


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

# HBM copy bandwidth of a B200 from an earlier STREAM-style copy measurement,
# used when the measured-peaks file is absent
HBM_FALLBACK_GBS = 6650.0


def hbm_peak():
    """(GB/s, source): the measured copy bandwidth of MEASURED_PEAKS.json, else
    the fallback figure."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (copy bandwidth), of measured"
    except (OSError, KeyError, ValueError, TypeError):
        return HBM_FALLBACK_GBS, "fallback: 6.65 TB/s, an earlier B200 copy-bandwidth measurement, of fallback"


def companion_op_split(D: int, m: int):
    """Integer lane-instructions one prime-step of the difference-table
    companion step needs, by the pipe that can execute them on B200 (ncu's
    pipe counters on the dr_bench_int_peak kernels put mad.wide.u32 on the ALU
    pipe and the low multiply mad.lo.u32 on the FMA pipe):
      wide  m+1 per last-column entry: its m products and the Montgomery
            reduction's q*p (ALU only)
      low   1 per entry: the reduction's quotient q = t*(-p^-1) (FMA only)
      mins  per entry the reduction's conditional subtraction and one per
            extra product's fold, plus one per difference-table addition (ALU)
      adds  the subtraction beside each of those mins, plus the addition
            itself per difference-table update (either pipe)."""
    D = max(int(D), 1)
    wide = m * (m + 1)
    low = m
    mins = m * (1 + max(0, m - 2)) + m * D
    adds = m * (1 + max(0, m - 2)) + 2 * m * D
    return wide, low, mins, adds


def pipe_bound(splits, peaks):
    """Shortest time the integer pipes allow for work given as
    [(prime_steps, (wide, low, mins, adds))]: ALU-only work at the ALU rate,
    FMA-only work at the FMA rate, everything over both pipes together, and
    everything at the issue rate -- whichever is slowest.  peaks: measured
    lane-ops/s of mad.wide.u32 alone (ALU pipe), mad.lo.u32 alone (FMA pipe)
    and add+min (both pipes, issue-bound)."""
    alu = sum(n * (w + mi) for n, (w, lo, mi, ad) in splits)
    fma = sum(n * lo for n, (w, lo, mi, ad) in splits)
    tot = sum(n * (w + lo + mi + ad) for n, (w, lo, mi, ad) in splits)
    t = {"alu": alu / peaks["alu"], "fma": fma / peaks["fma"],
         "alu+fma": tot / (peaks["alu"] + peaks["fma"]), "issue": tot / peaks["issue"]}
    return max(t.values()), t, tot


def int_peaks(N):
    import ctypes
    out = {}
    for name, kind in (("alu", 0), ("fma", 3), ("issue", 1)):
        v = ctypes.c_double()
        N.check(N.lib().dr_bench_int_peak(kind, ctypes.byref(v)), "int peak")
        out[name] = v.value
    return out


def walk_roofline(splits, ms, peaks, kernel):
    t_bound, parts, tot = pipe_bound(splits, peaks)
    t = ms * 1e-3
    return {"bound": "int", "achieved": tot / t / 1e12, "peak": tot / t_bound / 1e12, "unit": "Tops/s",
            "frac": t_bound / t, "traffic": None, "kernel": kernel, "kernel_ms": ms,
            "binding_pipe": max(parts, key=parts.get),
            "pipe_frac": {k: v / t for k, v in parts.items()},
            "peaks_tops": {k: v / 1e12 for k, v in peaks.items()},
            "model": "algorithmic lane-ops of the difference-table companion step split by pipe "
                     "(bench.companion_op_split); peak = the rate the binding pipe allows for this "
                     "mix, from live microbenchmarks (dr_bench_int_peak kinds 0, 3, 1)"}


# ---- further workloads (single-GPU runs) ------------------------------------

def _compile_cmf(mat):
    import dreams_rns as dr
    return dr.compile_cmf_from_dict(mat, m=3, dim=3, axis_names=["x", "y", "z"]).serialize()


def _time_batch(batch, stream, torch, reps=3):
    batch.run(stream.cuda_stream)
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        batch.run(stream.cuda_stream)
        e1.record(stream)
        ts.append((e0, e1))
    torch.cuda.synchronize()
    return statistics.median(a.elapsed_time(b) for a, b in ts)


def bench_rational(stream, torch):
    """Uneven batch: 8192 rational PCFs (INV every step), depth log-uniform in
    [200, 50000], K in {16,32,64,128}, bytecode 10..200 ops, one graph-captured
    persistent launch set with device top-256 by delta against pi."""
    import mpmath as mp_
    import dreams_rns as dr
    from dreams_rns.engine import WalkBatch, pcf_request
    cand = dr.synth.rational_pcfs(10000, seed=3)
    blobs = compile_all(cand)
    n_ops = lambda b: int.from_bytes(b[8:12], "little")  # noqa: E731  (blob header: m, dim, n_ops, n_consts)
    keep = [(b, w) for b, w in zip(blobs, cand) if 10 <= n_ops(b) <= 200][:8192]
    reqs = [pcf_request(b, w.a0, w.depth, w.K) for b, w in keep]
    tuned = dr.autotune(reqs)
    batch = WalkBatch(reqs)
    mp_.mp.dps = 200
    batch.set_pipeline(delta="fixed", target=dr.runner.target_ratio(mp_.pi), topk=256)
    ms = _time_batch(batch, stream, torch)
    st = batch.stats()
    pl = batch.read_pipeline()
    groups = _launch_groups(batch)
    batch.close()
    return {"walks": len(reqs), "prime_steps": st["prime_steps"], "ms": ms,
            "prime_steps_per_s": st["prime_steps"] / (ms * 1e-3), "launches": st["launches"],
            "autotuned": tuned,
            "launch_groups": groups,
            "span_ms_eager": max((g["end_ms"] for g in groups), default=None),
            "walks_end_ms": max((g["end_ms"] for g in groups if g["kind"] == "walk"), default=None),
            "shadows_end_ms": max((g["end_ms"] for g in groups if g["kind"] != "walk"), default=None),
            "top1_delta": float(pl["topk_val"][0]) if len(pl["topk_val"]) else None}


def _launch_groups(batch):
    """Balance across a batch's launch groups (one persistent launch per
    class, m and difference depth, each on its own stream): every group's
    span in one eager run of the batch (dr_debug_batch_timeline, ms after the
    first launch; an interpreted shadow's span runs from its evaluation to
    the end of its chain) beside its time alone (dr_batch_profile)."""
    import ctypes
    import numpy as np
    from dreams_rns import _native as N
    prof = batch.profile()
    cnt = ctypes.c_int32()
    spans = np.zeros(4 * 64, dtype=np.float32)
    N.check(N.lib().dr_debug_batch_timeline(batch.handle, 64, ctypes.byref(cnt), N.ptr(spans)),
            "dr_debug_batch_timeline")
    kinds = {0: "walk", 1: "shadow (interpreted or split)", 2: "shadow (integer differences)"}
    out = []
    for i, p in enumerate(prof[:cnt.value]):
        s = [float(x) for x in spans[4 * i:4 * i + 4]]
        out.append({"kind": kinds.get(p["kind"], str(p["kind"])), "m": p["m"], "degree": p["degree"],
                    "items": p["items"],
                    "alone_ms": round(p["ms"] + (p["ms2"] if p["kind"] == 1 else 0.0), 3),
                    "start_ms": round(s[0], 3), "end_ms": round(max(s[1], s[3]), 3)})
    return out


def bench_crt_stage(torch, n=1 << 20, reps=5):
    """The CRT stage alone, on residues already in HBM: ``n`` values of K = 32
    residues through dr_crt_batch_device on one stream, each call timed with
    CUDA events around it (median of ``reps`` after two untimed calls).  The
    residues (128 MiB) and limbs (132 MiB) together exceed L2.  Algorithmic
    bytes per value: 4K read, 4 * ceil(31K / 32) limb bytes plus sign and
    significant-limb count written."""
    import ctypes
    from dreams_rns import _native as N
    stride = (31 * K + 31) // 32 + 2
    dev = torch.device("cuda")
    g = torch.Generator(device=dev)
    g.manual_seed(5)
    # every prime of the table lies in (2^30, 2^31), so values below 2^30 are residues
    res = torch.randint(0, 1 << 30, (n, K), dtype=torch.int32, device=dev, generator=g)
    limbs = torch.empty((n, stride), dtype=torch.int32, device=dev)
    sign = torch.empty(n, dtype=torch.int32, device=dev)
    nl = torch.empty(n, dtype=torch.int32, device=dev)
    st = torch.cuda.Stream()
    times = []
    with torch.cuda.stream(st):
        for i in range(2 + reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            N.check(N.lib().dr_crt_batch_device(res.data_ptr(), K, n, None, limbs.data_ptr(), stride,
                                                sign.data_ptr(), nl.data_ptr(),
                                                ctypes.c_void_p(st.cuda_stream)), "dr_crt_batch_device")
            e1.record(st)
            e1.synchronize()
            if i >= 2:
                times.append(e0.elapsed_time(e1))
    ms = statistics.median(times)
    per_value = 4 * K + 4 * ((31 * K + 31) // 32) + 8
    gbs = per_value * n / (ms * 1e-3) / 1e9
    peak, peak_source = hbm_peak()
    del res, limbs, sign, nl
    # integer work per value of the lane kernel: K(K-1)/2 Garner steps of a
    # modular subtraction (3) and a Montgomery product (5), the Horner limb
    # updates (one wide multiply-add per limb, about K^2/2 * 31/32 of them)
    # and three borrow passes of the centring over L limbs (3 each)
    L = (31 * K + 31) // 32 + 2
    ops = K * (K - 1) // 2 * 8 + (K * (K - 1) // 2) * 31 // 32 + 9 * L
    issue = int_peaks(N)["issue"]
    return {"values": n, "K": K, "ms": ms, "bytes_per_value": per_value, "achieved_gbs": gbs,
            "hbm_peak_gbs": peak, "hbm_frac": gbs / peak if peak else None,
            "peak_source": peak_source,
            "int_roofline": {"bound": "int", "ops_per_value": ops, "achieved": ops * n / (ms * 1e-3) / 1e12,
                             "peak": issue / 1e12, "unit": "Tops/s",
                             "frac": ops * n / (ms * 1e-3) / issue,
                             "peak_source": "dr_bench_int_peak kind 1 (issue-bound add+min), measured live"},
            "kernel": "k_crt_lanes (Garner column recurrence per lane, 32 values per warp; Horner to limbs)"}


def bench_topk_stage(torch, n=1 << 24, k=256, reps=5):
    """Top-k by delta on HBM-resident deltas: n doubles through
    dr_topk_device (a strided-sample threshold, one filtering pass over the
    values, a sort of the few candidates), each call timed with CUDA events
    (median of ``reps`` after two untimed calls).  Algorithmic bytes: the n
    deltas read once, the k (index, value) pairs written."""
    import ctypes
    from dreams_rns import _native as N
    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    d = torch.randn(n, dtype=torch.float64, device="cuda", generator=g) * 0.01 - 1.0
    idx = torch.zeros(k, dtype=torch.int32, device="cuda")
    val = torch.zeros(k, dtype=torch.float64, device="cuda")
    st = torch.cuda.Stream()
    flag = ctypes.c_int32()
    times = []
    for i in range(2 + reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        N.check(N.lib().dr_topk_device(d.data_ptr(), n, k, idx.data_ptr(), val.data_ptr(),
                                       ctypes.c_void_p(st.cuda_stream), ctypes.byref(flag)), "dr_topk_device")
        e1.record(st)
        e1.synchronize()
        if i >= 2:
            times.append(e0.elapsed_time(e1))
    ms = statistics.median(times)
    # the result against torch's own sort of the same values (checker, untimed)
    ref = torch.sort(d, descending=True, stable=True).indices[:k].to(torch.int32)
    ok = bool(torch.equal(ref, idx))
    peak, peak_source = hbm_peak()
    nbytes = 8 * n + 12 * k
    gbs = nbytes / (ms * 1e-3) / 1e9
    del d, idx, val
    return {"values": n, "k": k, "ms": ms, "bytes": nbytes, "achieved_gbs": gbs, "hbm_peak_gbs": peak,
            "hbm_frac": gbs / peak if peak else None, "peak_source": peak_source,
            "threshold_filter": bool(flag.value),
            "matches_torch_sort": ok,
            "kernel": "k_topk_filter (one pass over the deltas) + sample and candidate tile sorts"}


def bench_cmf3(stream, torch, n_walks=16384):
    """3x3 CMF sweep: 16384 (shift, direction) pairs over 64 cubic CMFs, depth
    5000, K=64, top-100 by delta against zeta(3); plus the plain path (one walk
    per launch, per-step interpreter) on a few walks for comparison."""
    import mpmath as mp_
    import dreams_rns as dr
    from dreams_rns import _native as N
    from dreams_rns.engine import WalkBatch, cmf_request
    ws = dr.synth.cmf3_sweep(n_walks, n_cmfs=64, seed=4)
    keys = {}
    for w in ws:
        keys.setdefault(w.program_key, w.matrix)
    with mp.get_context("spawn").Pool(min(os.cpu_count() or 4, 16)) as pool:
        kb = dict(zip(keys, pool.map(_compile_cmf, list(keys.values()))))
    reqs = [cmf_request(kb[w.program_key], w.depth, w.K, w.shifts, w.trajectory) for w in ws]
    tuned = dr.autotune(reqs)
    batch = WalkBatch(reqs)
    mp_.mp.dps = 200
    batch.set_pipeline(delta="fixed", target=dr.runner.target_ratio(mp_.zeta(3)), topk=100)
    ms = _time_batch(batch, stream, torch)
    st = batch.stats()
    batch.close()
    rate = st["prime_steps"] / (ms * 1e-3)
    # the plain path: one walk per launch (a batch of one walk on the plain
    # engine: the same per-class step code, one warp per 32-prime block over
    # the whole depth, its FP64 shadow, CRT and delta), the sweep's first
    # n_plain walks back to back on one stream, inputs resident
    n_plain = 256
    tgt = dr.runner.target_ratio(mp_.zeta(3))
    plain = []
    for w in ws[:n_plain]:
        b = WalkBatch([cmf_request(kb[w.program_key], w.depth, w.K, w.shifts, w.trajectory)],
                      engine=N.DR_ENGINE_PLAIN)
        b.set_pipeline(delta="fixed", target=tgt)
        plain.append(b)
    for _ in range(2):              # direct run, then graph capture
        for b in plain:
            b.run(stream.cuda_stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for b in plain:
        b.run(stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    plain_ms = e0.elapsed_time(e1)
    plain_steps = sum(w.depth * w.K for w in ws[:n_plain])
    for b in plain:
        b.close()
    plain_rate = plain_steps / (plain_ms * 1e-3)
    # integer-pipe roofline of the walk kernels on this sweep (no shadow)
    import ctypes
    # at the launch shape the timed sweep runs with (the tuner's choice)
    walk_only = WalkBatch([cmf_request(kb[w.program_key], w.depth, w.K, w.shifts, w.trajectory, shadow=False)
                           for w in ws], chunk_steps=tuned["chunk_steps"], warps_per_block=tuned["warps_per_block"])
    walk_ms = _time_batch(walk_only, stream, torch, reps=5)
    walk_only.close()
    infos = {k: N.program_info(b) for k, b in kb.items()}
    splits = [(w.K * w.depth, companion_op_split(infos[w.program_key]["degree"], 3)) for w in ws]
    roof = walk_roofline(splits, walk_ms, int_peaks(N), "k_walk<COMPANION, 3, D>, walk-only sweep")
    roof["classes"] = sorted({(i["class"], i["degree"]) for i in infos.values()})
    return {"walks": len(reqs), "prime_steps": st["prime_steps"], "ms": ms, "prime_steps_per_s": rate,
            "walk_roofline": roof,
            "autotuned": tuned,
            "plain_one_walk_per_launch_prime_steps_per_s": plain_rate,
            "plain_path": {"walks": n_plain, "ms": plain_ms, "ms_per_walk": plain_ms / n_plain,
                           "what": "batch of one walk per launch on DR_ENGINE_PLAIN (same per-class "
                                   "step code, K/32 warps over the whole depth, FP64 shadow, CRT, "
                                   "delta), back to back on one stream, CUDA events"},
            "batched_over_plain": rate / plain_rate}


def bench_serving(seconds=3.0, rate=1000.0, inflight=6, plain=False):
    """Serving stream: Poisson arrivals drawn from the single-PCF, uniform-PCF
    and rational-PCF generators, plus 1% deep walks (deg-1 a, b, depth 10^6,
    K=512); p50/p99 request latency and prime-steps/s.  ``plain`` serves the
    same stream with one plain walk launch per request instead."""
    import random
    import numpy as np
    import dreams_rns as dr
    from dreams_rns.engine import pcf_request
    from dreams_rns.serving import WalkServer
    rng = random.Random(11)
    nrng = np.random.default_rng(12)
    uni = dr.synth.uniform_pcfs(96, seed=21, depth=2000, limit_depth=2000)
    rat = dr.synth.rational_pcfs(96, seed=22)
    deep = [dr.synth.deep_pcf(nrng) for _ in range(6)]
    ub = compile_all(uni)
    rb = compile_all(rat)
    db = compile_all(deep)
    single = dr.compile_pcf("2", "n**2").serialize()
    pool = ([("single", pcf_request(single, 2, 2000, 32))] +
            [("uniform", pcf_request(b, w.a0, 2000, 32)) for b, w in zip(ub, uni)] +
            [("rational", pcf_request(b, w.a0, w.depth, w.K)) for b, w in zip(rb, rat)])
    deep_reqs = [pcf_request(b, w.a0, w.depth, w.K) for b, w in zip(db, deep)]
    arrivals = []
    t = 0.0
    while t < seconds:
        t += rng.expovariate(rate)
        if rng.random() < 0.01:
            arrivals.append((t, "deep", rng.choice(deep_reqs)))
        else:
            kind, req = rng.choice(pool)
            arrivals.append((t, kind, req))
    lat = {}
    kinds = {}
    if plain:
        # the same stream served by the plain path: one request at a time in
        # arrival order, each one walk per launch (run_walks on the plain
        # engine: build, walk with its shadow, read back)
        from dreams_rns import _native as N
        from dreams_rns.engine import run_walks
        t0 = time.perf_counter()
        steps = 0
        for at, kind, req in arrivals:
            left = at - (time.perf_counter() - t0)
            if left > 0:
                time.sleep(left)
            run_walks([req], engine=N.DR_ENGINE_PLAIN)
            lat.setdefault(kind, []).append(time.perf_counter() - t0 - at)
            steps += req.K * req.depth
        wall = time.perf_counter() - t0
        allv = sorted(v for vs in lat.values() for v in vs)
        pct = lambda v, q: v[min(len(v) - 1, int(q * len(v)))] * 1e3  # noqa: E731
        return {"requests": len(arrivals), "arrival_rate_per_s": rate, "seconds": seconds,
                "p50_ms": pct(allv, 0.50), "p99_ms": pct(allv, 0.99),
                "p50_ms_by_kind": {k: pct(sorted(v), 0.5) for k, v in lat.items()},
                "p99_ms_by_kind": {k: pct(sorted(v), 0.99) for k, v in lat.items()},
                "prime_steps": steps, "prime_steps_per_s": steps / wall, "wall_s": wall,
                "what": "one request at a time in arrival order, each a one-walk launch on "
                        "DR_ENGINE_PLAIN (run_walks: build, walk + shadow, read)"}
    with WalkServer(max_inflight=inflight) as srv:
        t0 = time.perf_counter()
        ids = []
        for at, kind, req in arrivals:
            while True:     # wait for the arrival time: sleep, then spin the last half millisecond
                left = at - (time.perf_counter() - t0)
                if left <= 0:
                    break
                if left > 1e-3:
                    time.sleep(left - 5e-4)
            rid = srv.submit(req)
            ids.append(rid)
            kinds[rid] = kind
        res = srv.wait(ids, timeout=600)
        wall = time.perf_counter() - t0
        st = srv.stats()
    for rid, r in res.items():
        lat.setdefault(kinds[rid], []).append(r["latency_s"])
    allv = sorted(v for vs in lat.values() for v in vs)
    pct = lambda v, q: v[min(len(v) - 1, int(q * len(v)))] * 1e3  # noqa: E731
    return {"requests": len(ids), "arrival_rate_per_s": rate, "seconds": seconds,
            "p50_ms": pct(allv, 0.50), "p99_ms": pct(allv, 0.99),
            "p50_ms_by_kind": {k: pct(sorted(v), 0.5) for k, v in lat.items()},
            "p99_ms_by_kind": {k: pct(sorted(v), 0.99) for k, v in lat.items()},
            "prime_steps": st["prime_steps"], "prime_steps_per_s": st["prime_steps"] / wall,
            "wall_s": wall}


def main():
    global N_WALKS
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the rational, CMF-sweep and serving measurements")
    ap.add_argument("--no-autotune", action="store_true",
                    help="use the built-in launch-shape policy (profiler captures)")
    ap.add_argument("--walks", type=int, default=N_WALKS,
                    help="PCFs per GPU (default 4096, the benchmark workload; smaller values "
                         "give the same workload shape for profiler captures)")
    ap.add_argument("--stage", choices=["crt", "topk"],
                    help="measure one pipeline stage alone on HBM-resident inputs (CRT of 2^20 "
                         "K=32 residue vectors, or top-256 of 2^24 deltas) and print its JSON")
    args = ap.parse_args()
    N_WALKS = args.walks
    if args.stage:
        _use_repo_package()
        import torch
        from dreams_rns import _native as N
        N.init(int(os.environ.get("LOCAL_RANK", "0")))
        fn = bench_crt_stage if args.stage == "crt" else bench_topk_stage
        print(json.dumps({"stage": args.stage, **fn(torch)}), flush=True)
        return

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    config = {"workload": f"uniform PCF batch: {N_WALKS} seeded PCFs, deg a<=2, deg b<=4, coeffs in "
                          "[-10,10], m=2, depth 8000 with the depth-2000 convergent on the way, "
                          "K=32, delta(2000) vs own depth-8000 convergent, top-100",
              "walks_per_gpu": N_WALKS, "K": K, "depth": DEPTH, "checkpoint": CHECKPOINT,
              "parallelism": f"walk-sharded x{world}"}

    if args.impl == "reference":
        if rank != 0:
            return
        # The reference's own code on the host cores; this process never
        # imports the repository's package (its synthetic generator is loaded
        # by path).  One step = one timed pass over a bounded sample: the
        # workload's first PCFs, one per host core.
        ws = workload(seed=2)
        cores = _host_cores()
        pairs = [(w.a, w.b, w.a0) for w in ws[:cores]]
        blobs = None
        if cpu_kind() == "port":
            comp = _standalone("_bench_compiler", "compiler.py")
            blobs = [comp.compile_pcf(a, b).serialize() for a, b, _ in pairs]
        leg = cpu_leg(pairs, blobs=blobs, passes=max(args.steps, 1), warmup=args.warmup)
        cb = cpu_baseline_entry(leg)
        step_s = leg["pass_s"]
        value = cb["value"]
        line = {"metric": METRIC, "value": value, "unit": "prime-steps/s", "impl": "reference",
                "n_gpus": args.gpus, "steps": len(step_s), "warmup": args.warmup,
                "ms_per_step": statistics.mean(step_s) * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
                "config": dict(config, step=f"one pass over a bounded sample: the workload's first "
                                            f"{leg['walks']} PCFs, one per host core",
                               prime_steps_per_step=leg["walks"] * K * DEPTH,
                               prime_steps_note="the workload's prime-steps (depth 8000 x K per walk); "
                                                "the reference walks 2000 + 8000 steps to produce them"),
                "cpu_baseline": cb,
                "e2e": {"value": value, "unit": "prime-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    _use_repo_package()
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
    tuned = None if args.no_autotune else dr.autotune(reqs)   # launch shape by measurement (untimed set-up)
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
    # at the launch shape the timed batch runs with (the tuner's choice)
    walk_only = WalkBatch([pcf_request(b, w.a0, DEPTH, K, checkpoint=CHECKPOINT, shadow=False)
                           for b, w in zip(blobs, ws)],
                          chunk_steps=(tuned or {}).get("chunk_steps", 0),
                          warps_per_block=(tuned or {}).get("warps_per_block", 0))
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
    for b in blobs:
        if b not in infos:
            infos[b] = N.program_info(b)
    splits = [(K * DEPTH, companion_op_split(infos[b]["degree"], 2)) for b in blobs]
    import ctypes
    peaks = int_peaks(N)
    roofline = walk_roofline(splits, walk_ms, peaks,
                             "k_walk<COMPANION, 2, D> (D = 1..4), walk-only batch at the timed batch's launch shape, median of 5")
    walk_only.close()

    # ---- the step's critical path: the FP64 shadow chains, serial recurrences
    # bound by the latency of one step.  Each shadow launch group of the
    # benchmark batch runs alone (CUDA events); the floor is the same fast step
    # on one warp with its step matrices computed in registers.
    prof = batch.profile()
    chains = [(p["ms2"] if p["kind"] == 1 else p["ms"], p) for p in prof if p["kind"] in (1, 2)]
    # integer-difference launches the tuner packs two chain warps per
    # scheduler (chain_pack_depth) are slower by design, to give the walks
    # their SMs; the latency figure is over the one-warp-per-scheduler ones
    pack = int((tuned or {}).get("chain_pack_depth", 0))
    def _packed(p):
        return p["kind"] == 2 and pack and p["degree"] <= pack
    solo = [c for c in chains if not _packed(c[1])] or chains
    chain_ms, chain_p = max(solo, key=lambda x: x[0])
    floor = ctypes.c_double()
    N.check(N.lib().dr_bench_chain_step(DEPTH, ctypes.byref(floor)), "chain floor")
    chain_ns = chain_ms * 1e6 / DEPTH
    shadow_chain = {"bound": "latency", "achieved_ns_per_step": chain_ns, "floor_ns_per_step": floor.value,
                    "frac": floor.value / chain_ns, "chain_ms": chain_ms, "steps": DEPTH,
                    "kernel": (f"k_shadow_split<1,2,{chain_p['degree']}>" if chain_p["degree"] else "k_shadow_chain<2,1>")
                    if chain_p["kind"] == 1 else f"k_shadow_intfd<1,2,{chain_p['degree']},0>",
                    "floor_source": "dr_bench_chain_step: the same fast step on one warp, "
                                    "step matrices computed in registers",
                    "packed_launches": [{"kernel": f"k_shadow_intfd<1,2,{p['degree']},0>", "ms": c,
                                         "warps_per_scheduler": 2} for c, p in chains if _packed(p)]}

    # ---- end to end through the public API with host buffers: one sweep()
    # call per step packs the requests, uploads descriptors and programs,
    # walks, runs CRT -> delta -> top-k on the device and copies residues,
    # shadows, statuses, deltas and the top-k back to host memory
    e2e_times = []
    n = len(reqs)
    out = dr.sweep(reqs, delta="self", topk=TOPK)     # untimed: first-call buffer growth
    n_e2e = 5
    dr.stage_times(reset=True)
    for it in range(n_e2e):
        t0 = time.perf_counter()
        out = dr.sweep(reqs, delta="self", topk=TOPK)
        e2e_times.append(time.perf_counter() - t0)
    stages = dr.stage_times(reset=True)
    e2e_stages = {k[:-3]: stages[k] / n_e2e for k in stages if k.endswith("_ms")}
    import numpy as np_
    names = ("plan_lookup", "descriptors", "code_copy", "walks", "shape", "tile_count", "tile_fill",
             "tile_order", "shadow_lists", "geometry", "table_copy", "buffers_events", "sync")
    phases = np_.zeros(len(names))
    N.check(N.lib().dr_debug_build_phases(N.ptr(phases), len(names)), "build phases")
    e2e_stages["build_phases_cumulative"] = dict(zip(names, [round(float(v), 3) for v in phases]))
    from dreams_rns import _native as N_
    blob_bytes = sum(len(b) for b in set(blobs))
    h2d = n * N_.WALK_DTYPE.itemsize + blob_bytes + 8 * n * 4      # descriptors, programs, axes
    n_res = int(out["p_residues"].size)
    d2h = 2 * 4 * n_res + 6 * n * 8 + 4 * n + 8 * n + TOPK * 12      # residues, shadows, status, deltas, top-k
    assert np.array_equal(np.asarray(out["topk_idx"]), np.asarray(pipe["topk_idx"])), "sweep top-k differs"
    e2e_s = statistics.median(e2e_times)
    e2e_val = prime_steps * world / e2e_s
    # A sweep over many lists (the workload each): dreams_rns.sweep_many
    # packs, builds and uploads the next lists on host threads while the
    # device walks the current one.  Every list is still copied in and its
    # results read back inside the timed region; the time per list is the
    # whole loop's over the number of lists, pipeline fill and drain included.
    for _ in dr.sweep_many([reqs] * 2, delta="self", topk=TOPK):
        pass                                            # untimed: thread and buffer set-up
    n_pipe = 12
    t0 = time.perf_counter()
    last = None
    for last in dr.sweep_many([reqs] * n_pipe, delta="self", topk=TOPK):
        pass
    pipe_s = (time.perf_counter() - t0) / n_pipe
    assert np.array_equal(np.asarray(last["topk_idx"]), np.asarray(pipe["topk_idx"])), "sweep_many top-k differs"
    pipe_val = prime_steps * world / pipe_s
    n_launch = int(st["launches"]) + 1 + 1 + 1     # walk/shadow groups + CRT + delta + top-k

    line = {"metric": METRIC, "value": value, "unit": "prime-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded PCF generator; the reference's datasets are not shipped)",
            "config": dict(config, l2="flushed: 512 MB write between timed steps",
                           launch_shape=tuned,
                           timing="CUDA events on the launching stream, max over ranks"),
            "clocks": clocks,
            "e2e": {"value": pipe_val, "unit": "prime-steps/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "seconds_per_step": pipe_s,
                    "path": f"dreams_rns.sweep_many over {n_pipe} lists of the workload's requests "
                            "(delta='self', topk=100): each list's host descriptors in and its "
                            "residues/shadows/deltas/top-k out, the next lists' host work "
                            "overlapping the device; time per list over the whole loop",
                    "single_call": {"value": e2e_val, "seconds_per_step": e2e_s,
                                    "stage_ms_per_call": e2e_stages,
                                    "path": "one dreams_rns.sweep(requests, delta='self', topk=100) "
                                            "call per step, median of 5"}},
            "gpu_launches": n_launch,
            "roofline": roofline,
            "shadow_chain": shadow_chain,
            "top1_delta": float(pipe["topk_val"][0]) if len(pipe["topk_val"]) else None}
    if dist:
        from dreams_rns.distributed import global_topk
        base = rank * N_WALKS
        local = [(float(v), base + int(i)) for i, v in zip(pipe["topk_idx"], pipe["topk_val"])]
        g = global_topk(local, TOPK)
        line["global_top1_delta"] = g[0][0] if g else None
    if world == 1 and not args.no_extras:
        line["rational_pcf_batch"] = bench_rational(stream, torch)
        line["cmf3_sweep"] = bench_cmf3(stream, torch)
        line["serving"] = bench_serving()
        line["p50_ms"] = line["serving"]["p50_ms"]
        line["p99_ms"] = line["serving"]["p99_ms"]
        # the same arrivals (1 s of the 1k/s stream) through the plain path,
        # and the continuous-batching server on that same second
        pl = bench_serving(seconds=1.0, plain=True)
        cb = bench_serving(seconds=1.0)
        line["serving_vs_plain"] = {"plain": pl, "batched": {k: cb[k] for k in (
            "requests", "p50_ms", "p99_ms", "prime_steps_per_s", "wall_s")},
            "prime_steps_per_s_ratio": cb["prime_steps_per_s"] / pl["prime_steps_per_s"],
            "p99_ratio": pl["p99_ms"] / cb["p99_ms"]}
        # the same stream at the top of the 1k-50k requests/s range (2 s each);
        # at 50k/s the 1% deep walks alone (~2.5e11 prime-steps/s) exceed what
        # the GPU walks, so that run is past saturation and its latency grows
        line["serving_rates"] = {}
        for rate in (10000.0, 50000.0):
            r = bench_serving(seconds=2.0, rate=rate)
            line["serving_rates"][str(int(rate))] = {k: r[k] for k in (
                "requests", "p50_ms", "p99_ms", "p50_ms_by_kind", "p99_ms_by_kind", "prime_steps_per_s")}
    if world == 1 and not args.no_extras:
        try:
            line["crt_stage"] = bench_crt_stage(torch)
        except Exception as exc:  # noqa: BLE001 - report it, keep the bench line
            line["crt_stage"] = {"error": f"{type(exc).__name__}: {exc}"}
        try:
            line["topk_stage"] = bench_topk_stage(torch)
        except Exception as exc:  # noqa: BLE001 - report it, keep the bench line
            line["topk_stage"] = {"error": f"{type(exc).__name__}: {exc}"}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the CPU path on the workload's first PCFs, one per host core; its
        # outputs also check the timed batch's results for those walks
        cores = _host_cores()
        leg = cpu_leg([(w.a, w.b, w.a0) for w in ws[:cores]], blobs=blobs[:cores])
        line["cpu_baseline"] = cpu_baseline_entry(leg)
        line["parity_checked"] = parity_vs_cpu(batch.read()[:cores], pipe["delta"], blobs, leg)
    batch.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
