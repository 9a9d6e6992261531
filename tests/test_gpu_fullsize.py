"""GPU parity at the benchmark workloads' own sizes.

Each test runs a seeded sample of one benchmark workload at its full depth
and prime count through the engine -- inside the full benchmark batch where
that batch is cheap to build -- with the device CRT -> delta pipeline, and
checks it against the C oracle (a restatement of the reference's
runner.py:338-413 / cmf_walk.py:363-431, pinned to the reference's golden
vectors by test_oracle_golden.py):

* p, q residues (and the checkpoint's): bit-exact;
* CRT values from the device pipeline: bit-exact against the oracle's CRT of
  the oracle's residues (reference runner.py:57-81);
* delta: within 1e-9 of the mpmath delta (reference runner.py:103-125);
* FP64 shadow: within 1e-12 relative (log_scale 1e-13), as elsewhere.

Sizes: the uniform PCF batch at depth 8000 with its depth-2000 convergent,
difference depths 1..4 (the headline workload); rational PCFs at depth
>= 40000 with K = 128, one of them meeting INV(0) mod a prime; the 3x3 CMF
sweep at depth 5000, K = 64; one depth-10^6, K = 512 serving walk.
"""

import math
import multiprocessing as mp
import os

import mpmath
import numpy as np
import pytest

import dreams_rns as dr
from dreams_rns import _native as N
from dreams_rns.engine import WalkBatch, cmf_request, pcf_request
from oracle import walk_c
from oracle.walk_np import centered, crt, delta_exact

pytestmark = pytest.mark.gpu

SHADOW_RTOL = 1e-12
DELTA_ATOL = 1e-9


def _close(a, b, rtol=SHADOW_RTOL):
    if a == b or (math.isnan(a) and math.isnan(b)):
        return True
    return abs(a - b) <= rtol * max(abs(a), abs(b), 1e-300)


def _shadow_ok(got, want):
    return (_close(got["p_float"], want["p_float"]) and _close(got["q_float"], want["q_float"])
            and _close(got["log_scale"], want["log_scale"], 1e-13))


def _crt_value(res, K):
    pr = [int(p) for p in N.prime_table(K)]
    x, M = crt([int(v) for v in res], pr)
    return centered(x, M)


def _delta_ok(got, want):
    if math.isinf(want) or math.isinf(got) or math.isnan(want) or math.isnan(got):
        return got == want or (math.isnan(got) and math.isnan(want))
    return abs(got - want) <= DELTA_ATOL


def _compile_pcf(ab):
    import dreams_rns as dr_
    return dr_.compile_pcf(*ab).serialize()


def _compile_many(pairs):
    with mp.get_context("spawn").Pool(min(os.cpu_count() or 4, 16)) as pool:
        return pool.map(_compile_pcf, pairs, chunksize=32)


def test_uniform_pcf_batch_full_size():
    """The headline batch: 4096 PCFs to depth 8000 with the depth-2000
    convergent, delta of each checkpoint against its own final convergent,
    top-100; 32 walks (8 per difference depth 1..4) against the oracle."""
    ws = dr.synth.uniform_pcfs(4096, seed=2, depth=2000, limit_depth=8000, K=32)
    blobs = _compile_many([(w.a, w.b) for w in ws])
    reqs = [pcf_request(b, w.a0, 8000, 32, checkpoint=2000) for b, w in zip(blobs, ws)]
    batch = WalkBatch(reqs)
    batch.set_pipeline(delta="self", topk=100)
    batch.run()
    res = batch.read()
    pipe = batch.read_pipeline(values=True)
    batch.close()
    by_d = {}
    for i, b in enumerate(blobs):
        by_d.setdefault(N.program_info(b)["degree"], []).append(i)
    assert sorted(by_d) == [1, 2, 3, 4]
    picks = [i for d in (1, 2, 3, 4) for i in by_d[d][:8]]
    mpmath.mp.dps = 200
    for i in picks:
        w = ws[i]
        fin = walk_c.pcf_walk(blobs[i], w.a0, 8000, 32)
        cp = walk_c.pcf_walk(blobs[i], w.a0, 2000, 32)
        r = res[i]
        assert list(r["p_residues"]) == list(fin["p_residues"]), i
        assert list(r["q_residues"]) == list(fin["q_residues"]), i
        assert list(r["checkpoint"]["p_residues"]) == list(cp["p_residues"]), i
        assert list(r["checkpoint"]["q_residues"]) == list(cp["q_residues"]), i
        assert _shadow_ok(r, fin), (i, r["p_float"], fin["p_float"])
        assert _shadow_ok(r["checkpoint"], cp), i
        vals = [_crt_value(x, 32) for x in (fin["p_residues"], fin["q_residues"],
                                            cp["p_residues"], cp["q_residues"])]
        assert [pipe["p"][i], pipe["q"][i], pipe["cp_p"][i], pipe["cp_q"][i]] == vals, i
        L = mpmath.mpf(vals[0]) / mpmath.mpf(vals[1])
        want = delta_exact(vals[2], vals[3], L, 200)
        assert _delta_ok(float(pipe["delta"][i]), float(want)), (i, pipe["delta"][i], want)
    # top-100 of all 4096: the device deltas in the device order (highest
    # first, NaN last, ties by lower index)
    d = np.asarray(pipe["delta"], dtype=np.float64)
    key = np.where(np.isnan(d), -np.inf, d)
    order = sorted(range(len(d)), key=lambda j: (np.isnan(d[j]), -key[j], j))[:100]
    assert list(pipe["topk_idx"]) == order


def _rational_sample():
    """16 rational PCFs of the uneven batch's generator with depth >= 40000
    and bytecode of 10..200 ops, walked with K = 128, plus one whose
    denominator n + (p0 - 100) is 0 mod the first prime p0 at n = 100."""
    cand = dr.synth.rational_pcfs(3000, seed=3)
    out = []
    for w in cand:
        if w.depth < 40000:
            continue
        blob = dr.compile_pcf(w.a, w.b).serialize()
        n_ops = int.from_bytes(blob[8:12], "little")
        if 10 <= n_ops <= 200:
            out.append((blob, w.a0, w.depth))
        if len(out) == 15:
            break
    p0 = int(N.prime_table(1)[0])
    inv0 = dr.compile_pcf("3*n + 1", f"(n**2 + 1)/(n + {p0 - 100})").serialize()
    out.append((inv0, 1, 41000))
    return out


def test_rational_pcfs_deep_full_size():
    sample = _rational_sample()
    assert len(sample) == 16
    reqs = [pcf_request(b, a0, depth, 128) for b, a0, depth in sample]
    batch = WalkBatch(reqs)
    mpmath.mp.dps = 200
    tnum, tden = dr.runner.target_ratio(mpmath.pi)
    batch.set_pipeline(delta="fixed", target=(tnum, tden), topk=16)
    batch.run()
    res = batch.read()
    pipe = batch.read_pipeline(values=True)
    batch.close()
    for i, (blob, a0, depth) in enumerate(sample):
        o = walk_c.pcf_walk(blob, a0, depth, 128)
        r = res[i]
        assert list(r["p_residues"]) == list(o["p_residues"]), i
        assert list(r["q_residues"]) == list(o["q_residues"]), i
        assert _shadow_ok(r, o), (i, r["p_float"], o["p_float"])
        p, q = _crt_value(o["p_residues"], 128), _crt_value(o["q_residues"], 128)
        assert (pipe["p"][i], pipe["q"][i]) == (p, q), i
        want = delta_exact(p, q, mpmath.mpf(tnum) / tden, 200)
        assert _delta_ok(float(pipe["delta"][i]), float(want)), (i, pipe["delta"][i], want)
    assert res[-1]["status"] & N.DR_STATUS_INV0
    assert not any(r["status"] & N.DR_STATUS_INV0 for r in res[:-1])


def test_cmf3_sweep_full_size():
    """The 3x3 CMF sweep batch (16384 walks, depth 5000, K = 64, top-100 by
    delta against zeta(3)); its first 64 walks against the oracle."""
    ws = dr.synth.cmf3_sweep(16384, n_cmfs=64, seed=4)
    progs = {}
    for w in ws:
        if w.program_key not in progs:
            progs[w.program_key] = dr.compile_cmf_from_dict(w.matrix, m=3, dim=3,
                                                            axis_names=["x", "y", "z"]).serialize()
    reqs = [cmf_request(progs[w.program_key], w.depth, w.K, w.shifts, w.trajectory) for w in ws]
    batch = WalkBatch(reqs)
    mpmath.mp.dps = 200
    tnum, tden = dr.runner.target_ratio(mpmath.zeta(3))
    batch.set_pipeline(delta="fixed", target=(tnum, tden), topk=100)
    batch.run()
    res = batch.read()
    pipe = batch.read_pipeline(values=True)
    batch.close()
    for i, w in enumerate(ws[:64]):
        o = walk_c.cmf_walk(progs[w.program_key], 5000, 64, w.shifts, w.trajectory)
        r = res[i]
        assert list(r["p_residues"]) == list(o["p_residues"]), i
        assert list(r["q_residues"]) == list(o["q_residues"]), i
        assert _shadow_ok(r, o), (i, r["p_float"], o["p_float"])
        p, q = _crt_value(o["p_residues"], 64), _crt_value(o["q_residues"], 64)
        assert (pipe["p"][i], pipe["q"][i]) == (p, q), i
        want = delta_exact(p, q, mpmath.mpf(tnum) / tden, 200)
        assert _delta_ok(float(pipe["delta"][i]), float(want)), (i, pipe["delta"][i], want)


def test_deep_serving_walk_full_size():
    """A config-5 deep walk (deg-1 a and b, depth 10^6, K = 512) through the
    continuous-batching server, resumed from device state segment by
    segment, against the oracle."""
    from dreams_rns.serving import WalkServer
    w = dr.synth.deep_pcf(np.random.default_rng(12))
    blob = dr.compile_pcf(w.a, w.b).serialize()
    req = pcf_request(blob, w.a0, w.depth, w.K)
    assert (req.depth, req.K) == (1_000_000, 512)
    with WalkServer(max_inflight=2) as srv:
        rid = srv.submit(req)
        got = srv.wait([rid], timeout=600)[rid]
    o = walk_c.pcf_walk(blob, w.a0, w.depth, w.K)
    assert list(got["p_residues"]) == list(o["p_residues"])
    assert list(got["q_residues"]) == list(o["q_residues"])
    assert _shadow_ok(got, o), (got["p_float"], o["p_float"], got["log_scale"], o["log_scale"])
