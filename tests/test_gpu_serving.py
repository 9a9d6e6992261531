"""Serving: results are identical alone and in the mix; admission, resume
from device state, cancellation."""

import random
import time

import numpy as np
import pytest

import dreams_rns as dr
from dreams_rns import _native as N
from dreams_rns.engine import cmf_request, pcf_request, run_walks
from dreams_rns.serving import WalkServer

pytestmark = pytest.mark.gpu


def _mix(seed, n=40):
    rng = random.Random(seed)
    reqs = []
    ws = dr.synth.uniform_pcfs(n // 2, seed=seed, depth=10, limit_depth=10)
    for w in ws:
        reqs.append(pcf_request(dr.compile_pcf(w.a, w.b), w.a0, rng.randrange(0, 3000),
                                rng.choice([16, 32, 64])))
    for w in dr.synth.rational_pcfs(n // 4, seed=seed + 1, depth_range=(100, 2000)):
        reqs.append(pcf_request(dr.compile_pcf(w.a, w.b), w.a0, w.depth, w.K))
    c = dr.synth.cmf3_sweep(n // 4, n_cmfs=2, seed=seed + 2, depth=700, K=40)
    for w in c:
        prog = dr.compile_cmf_from_dict(w.matrix, m=3, dim=3, axis_names=["x", "y", "z"])
        reqs.append(cmf_request(prog, w.depth, w.K, w.shifts, w.trajectory))
    # a long walk that needs several segments (walk and shadow)
    reqs.append(pcf_request(dr.compile_pcf("2*n+1", "-n**2 + 3"), 1, 150_000, 96))
    return reqs


def _same(a, b):
    assert list(a["p_residues"]) == list(b["p_residues"])
    assert list(a["q_residues"]) == list(b["q_residues"])
    for k in ("p_float", "q_float", "log_scale"):
        assert a[k] == b[k] or (np.isnan(a[k]) and np.isnan(b[k])), k


def test_alone_and_in_the_mix():
    reqs = _mix(5)
    batch = run_walks(reqs)
    with WalkServer(max_inflight=3, chunk_steps=2048) as srv:
        # each request alone
        alone = {}
        for i in (0, 7, len(reqs) - 1):
            rid = srv.submit(reqs[i])
            alone[i] = srv.wait([rid])[rid]
        # all of them, arriving in waves while earlier ones run
        ids = []
        for i, r in enumerate(reqs):
            ids.append(srv.submit(r))
            if i % 9 == 0:
                time.sleep(0.002)
        got = srv.wait(ids, timeout=120)
        st = srv.stats()
    for i, rid in enumerate(ids):
        _same(got[rid], batch[i])
    for i, r in alone.items():
        _same(r, batch[i])
    assert st["completed"] == len(reqs) + len(alone)
    assert st["queue_depth"] == 0 and st["admitted_bytes"] == 0


def test_admission_cap_queues_requests():
    reqs = _mix(8, n=16)[:-1]
    batch = run_walks(reqs)
    # cap small enough that only a couple of walks fit at once
    with WalkServer(mem_cap_bytes=12_000, max_inflight=2) as srv:
        ids = [srv.submit(r) for r in reqs]
        got = srv.wait(ids, timeout=120)
    for i, rid in enumerate(ids):
        _same(got[rid], batch[i])


def test_oversize_and_cancel():
    big = pcf_request(dr.compile_pcf("1", "n"), 1, 1000, 2048)
    with WalkServer(mem_cap_bytes=20_000) as srv:
        with pytest.raises(MemoryError):
            srv.submit(big)
        long = pcf_request(dr.compile_pcf("n", "n**2"), 0, 400_000, 64)
        rid = srv.submit(long)
        srv.cancel(rid)
        r2 = srv.submit(pcf_request(dr.compile_pcf("2", "n**2"), 2, 2000, 32))
        res = srv.wait([r2])[r2]
    g = run_walks([pcf_request(dr.compile_pcf("2", "n**2"), 2, 2000, 32)])[0]
    _same(res, g)


def test_short_requests_overtake_a_long_one():
    """A long request (many shadow segments) runs in its own waves; a short
    request submitted behind it completes first, with the same results as a
    batch, and the scheduler's wave record is consistent."""
    long = pcf_request(dr.compile_pcf("2*n+1", "-n**2 + 3"), 1, 150_000, 96)
    short = pcf_request(dr.compile_pcf("2", "n**2"), 2, 2000, 32)
    with WalkServer(max_inflight=3) as srv:
        rl = srv.submit(long)
        rs = srv.submit(short)
        got_s = srv.wait([rs])[rs]
        assert srv.poll(rl) is None          # the long request is still in flight
        got_l = srv.wait([rl], timeout=120)[rl]
        log = srv.wave_log()
    ref = run_walks([long, short])
    _same(got_l, ref[0])
    _same(got_s, ref[1])
    assert got_s["latency_s"] < got_l["latency_s"]
    assert len(log) >= 150_000 // 8192
    t_sel, t_launched, t_harvest, gpu_ms, n_req, has_long, slot = (log[:, i] for i in range(7))
    assert np.all(t_sel <= t_launched) and np.all(t_launched <= t_harvest)
    assert np.all(gpu_ms > 0) and np.all(n_req >= 1)
    assert set(np.unique(has_long)) <= {0.0, 1.0} and has_long.max() == 1.0
    assert np.all((slot >= 0) & (slot < 3))


def _collect(srv, ids, timeout=120.0):
    """Poll every request to its end: results, and the ids that raised
    MemoryError (requests whose allocation failed)."""
    got, failed = {}, []
    left = list(ids)
    t0 = time.monotonic()
    while left:
        nxt = []
        for rid in left:
            try:
                r = srv.poll(rid)
            except MemoryError:
                failed.append(rid)
                continue
            if r is None:
                nxt.append(rid)
            else:
                got[rid] = r
        left = nxt
        assert time.monotonic() - t0 < timeout, f"{len(left)} requests still running"
        time.sleep(0.0005)
    return got, failed


def test_injected_allocation_failures():
    """Host-side fault injection: admissions and a wave launch whose device
    allocation fails end their requests with MemoryError; every other
    request completes with the batch's results, the server keeps serving
    and its accounting returns to zero."""
    reqs = _mix(9, n=16)
    batch = run_walks(reqs)
    with WalkServer(max_inflight=2) as srv:
        assert srv.inject_failures(admissions=2) == 0
        ids = [srv.submit(r) for r in reqs]
        got, failed = _collect(srv, ids)
        assert len(failed) == 2
        for i, rid in enumerate(ids):
            if rid in got:
                _same(got[rid], batch[i])
        st = srv.stats()
        assert st["admitted_bytes"] == 0 and st["queue_depth"] == 0
        # a wave whose buffers cannot grow: only its own requests fail
        srv.inject_failures(waves=1)
        ids2 = [srv.submit(r) for r in reqs[:8]]
        got2, failed2 = _collect(srv, ids2)
        assert len(failed2) >= 1
        for i, rid in enumerate(ids2):
            if rid in got2:
                _same(got2[rid], batch[i])
        # and the server still serves
        rid = srv.submit(reqs[0])
        _same(srv.wait([rid])[rid], batch[0])
        st = srv.stats()
        assert st["admitted_bytes"] == 0 and st["queue_depth"] == 0
        assert srv.inject_failures() == 2 + len(failed2)
