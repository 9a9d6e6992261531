"""GPU parity: the CUDA engine against the reference fixtures and the C oracle.

Residues, CRT values: bit-exact.  Float shadow: identical when the engine
uses integer differences (all reference intermediates exact), otherwise
within 1e-12 relative (the reference's own pow() is not correctly rounded,
so only the shadow may differ, by ulps).  Delta: within 1e-9 of mpmath.
"""

import math
import random
from fractions import Fraction

import numpy as np
import pytest

import dreams_rns as dr
from dreams_rns import _native as N
from dreams_rns.engine import WalkBatch, WalkRequest, cmf_request, pcf_request, run_walks
from oracle import walk_c
from progfuzz import random_axis, random_program

pytestmark = pytest.mark.gpu

SHADOW_RTOL = 1e-12


def _close(a, b, rtol=SHADOW_RTOL):
    if a == b:
        return True
    if math.isnan(a) and math.isnan(b):
        return True
    return abs(a - b) <= rtol * max(abs(a), abs(b), 1e-300)


def _shadow_ok(r, w):
    pf, qf, ls = (float.fromhex(w[k]) for k in ("p_float", "q_float", "log_scale"))
    return _close(r["p_float"], pf) and _close(r["q_float"], qf) and _close(r["log_scale"], ls, 1e-13)


@pytest.mark.parametrize("engine", [N.DR_ENGINE_AUTO, N.DR_ENGINE_INTERP])
def test_pcf_fixtures(golden, engine):
    reqs = [pcf_request(bytes.fromhex(w["blob"]), w["a0"], w["depth"], w["K"], w["shift"])
            for w in golden["pcf_walks"]]
    for chunk in (0, 97):
        res = run_walks(reqs, chunk_steps=chunk, engine=engine)
        for w, r in zip(golden["pcf_walks"], res):
            assert list(r["p_residues"]) == w["p_residues"], (w["name"], engine, chunk)
            assert list(r["q_residues"]) == w["q_residues"], (w["name"], engine, chunk)
            assert _shadow_ok(r, w), (w["name"], r["p_float"], w["p_float"])


def test_inv0_status(golden):
    by = {w["name"]: w for w in golden["pcf_walks"]}
    reqs = [pcf_request(bytes.fromhex(by[n]["blob"]), by[n]["a0"], by[n]["depth"], by[n]["K"])
            for n in ("inv0_one_prime", "int_root_inv0", "config1")]
    res = run_walks(reqs)
    assert res[0]["status"] & N.DR_STATUS_INV0
    assert res[1]["status"] & N.DR_STATUS_INV0
    assert not res[2]["status"] & N.DR_STATUS_INV0


def test_cmf_fixtures(golden):
    reqs = []
    for w in golden["cmf_walks"]:
        tr = w["trajectory"]
        reqs.append(cmf_request(bytes.fromhex(w["blob"]), w["depth"], w["K"],
                                [tuple(x) for x in w["shifts"]],
                                None if tr is None else [tuple(x) for x in tr]))
    for engine in (N.DR_ENGINE_AUTO, N.DR_ENGINE_INTERP):
        res = run_walks(reqs, engine=engine)
        for w, r in zip(golden["cmf_walks"], res):
            assert list(r["p_residues"]) == w["p_residues"], w["name"]
            assert list(r["q_residues"]) == w["q_residues"], w["name"]
            assert _shadow_ok(r, w), w["name"]


def test_dropin_run_pcf_walk_config1(golden):
    w = golden["pcf_walks"][0]
    prog = dr.compile_pcf("2", "n**2")
    r = dr.run_pcf_walk(prog, dr.pcf_initial_values("2"), 2000, 32)
    assert r["p_residues"].dtype == np.int64 and r["p_residues"].shape == (32,)
    assert list(r["p_residues"]) == w["p_residues"]
    assert list(r["q_residues"]) == w["q_residues"]
    assert list(r["primes"]) == golden["primes_512"][:32]
    assert r["p_float"] == float.fromhex(w["p_float"])
    assert r["q_float"] == float.fromhex(w["q_float"])
    with pytest.raises(AssertionError):
        dr.run_pcf_walk(dr.compile_cmf_from_dict({(0, 0): "x0"}, 1, 1), 0, 10, 8)


def test_crt_fixtures(golden):
    for c in golden["crt"]:
        x, M = dr.crt_reconstruct(c["residues"], c["primes"])
        assert hex(x) == c["x"] and hex(M) == c["M"]
        assert hex(dr.centered(x, M)) == c["centered"]


def test_crt_batch_matches_oracle():
    from oracle.walk_np import centered, crt
    rng = np.random.default_rng(5)
    for K in (1, 2, 16, 31, 32, 33, 64, 100, 512):
        pr = [int(p) for p in dr.generate_rns_primes(K)]
        res = np.stack([rng.integers(0, p, size=40) for p in pr], axis=1).astype(np.uint32)
        res[0, :] = 0
        res[1, :] = 1
        res[2, :] = [p - 1 for p in pr]
        got = dr.crt_batch(res, K)
        for i in range(res.shape[0]):
            x, M = crt([int(v) for v in res[i]], pr)
            assert got[i] == centered(x, M), (K, i)


def test_delta_fixtures(golden):
    for d in golden["delta_exact"]:
        got = dr.compute_dreams_delta_exact(int(d["p"], 16), int(d["q"], 16), d["target"], d["dps"])
        want = float(d["delta"])
        if math.isinf(want) or math.isinf(got):
            assert got == want, d["name"]
        else:
            assert abs(got - want) < 1e-9, (d["name"], got, want)


def test_verify_pcf(golden):
    for v in golden["verify_pcf"]:
        r = dr.verify_pcf(v["a"], v["b"], v["limit"], v["depth"], v["K"])
        want = v["result"]
        assert r["p_bits"] == want["p_bits"]
        assert abs(r["delta_exact"] - float(want["delta_exact"])) < 1e-9
        assert abs(r["delta_float"] - float(want["delta_float"])) < 1e-9
        assert r["target"] == float(want["target"])


def test_random_programs_vs_oracle():
    rng = random.Random(11)
    reqs, refs = [], []
    for trial in range(300):
        blob, m, dim = random_program(rng)
        try:
            N.program_info(blob)
        except Exception:
            continue
        K = rng.choice([1, 5, 32, 40, 64])
        depth = rng.randrange(0, 300)
        axis = random_axis(rng, dim, rng.random() < 0.4)
        pcf = m == 2 and rng.random() < 0.5
        a0 = rng.randrange(-9, 10)
        cp = rng.randrange(1, depth) if depth > 2 and rng.random() < 0.4 else 0
        req = WalkRequest(blob=blob, K=K, depth=depth, a0=a0, pcf_init=pcf, q_row=1 if pcf else m - 1,
                          axis=[tuple(axis[4 * a:4 * a + 4]) for a in range(dim)], checkpoint=cp,
                          shadow=False)
        init = np.eye(m, dtype=np.int64)
        if pcf:
            init[0, 1] = a0
        refs.append((blob, K, depth, np.array(axis, np.int64), init, req.q_row, cp))
        reqs.append(req)
    for chunk in (0, 16):
        res = run_walks(reqs, chunk_steps=chunk)
        for (blob, K, depth, axis, init, qrow, cp), r in zip(refs, res):
            o = walk_c.walk(blob, depth, K, axis, init, 0, qrow, shadow=False)
            assert list(r["p_residues"]) == list(o["p_residues"])
            assert list(r["q_residues"]) == list(o["q_residues"])
            if cp:
                o2 = walk_c.walk(blob, cp, K, axis, init, 0, qrow, shadow=False)
                assert list(r["checkpoint"]["p_residues"]) == list(o2["p_residues"])


def test_shadow_vs_oracle():
    rng = random.Random(3)
    reqs = []
    for trial in range(60):
        a = dr.synth.poly_str([rng.randrange(-9, 10) for _ in range(rng.randrange(1, 4))])
        b = dr.synth.poly_str([rng.randrange(-9, 10) for _ in range(rng.randrange(1, 6))])
        if rng.random() < 0.3:
            b = f"({b})/({dr.synth.poly_str([rng.randrange(1, 9), rng.randrange(-3, 4)])})"
        prog = dr.compile_pcf(a, b)
        reqs.append((prog, pcf_request(prog, dr.pcf_initial_values(a), rng.randrange(1, 3000), 32,
                                       rng.randrange(-3, 4))))
    res = run_walks([r for _, r in reqs])
    for (prog, req), r in zip(reqs, res):
        o = walk_c.pcf_walk(req.blob, req.a0, req.depth, 32, req.axis[0][0])
        assert list(r["p_residues"]) == list(o["p_residues"])
        assert _close(r["p_float"], o["p_float"]) and _close(r["q_float"], o["q_float"])
        assert _close(r["log_scale"], o["log_scale"], 1e-13)


def test_shadow_rounds_match_single_pass():
    """A small step-matrix buffer splits the interpreted shadow into rounds
    with resident state; results (checkpoints included) must not change."""
    rng = random.Random(5)
    reqs = []
    for trial in range(40):
        a = dr.synth.poly_str([rng.randrange(-9, 10) for _ in range(3)])
        b = dr.synth.poly_str([rng.randrange(-9, 10) for _ in range(5)])
        if trial % 2:
            b = f"({b})/({dr.synth.poly_str([rng.randrange(1, 9), rng.randrange(-3, 4)])})"
        depth = rng.randrange(1, 6000)
        cp = rng.randrange(1, depth) if depth > 2 and trial % 3 == 0 else 0
        reqs.append(pcf_request(dr.compile_pcf(a, b), dr.pcf_initial_values(a), depth, 32, checkpoint=cp))
    one = run_walks(reqs)
    rounds = run_walks(reqs, shadow_buffer_mb=1)
    for req, x, y in zip(reqs, one, rounds):
        for k in ("p_float", "q_float", "log_scale"):
            assert x[k] == y[k] or (math.isnan(x[k]) and math.isnan(y[k])), k
        if req.checkpoint:
            for k in ("p_float", "q_float", "log_scale"):
                assert x["checkpoint"][k] == y["checkpoint"][k], k
        o = walk_c.pcf_walk(req.blob, req.a0, req.depth, 32)
        assert _close(x["p_float"], o["p_float"]) and _close(x["q_float"], o["q_float"])


def test_rescale_division_is_correctly_rounded():
    """The shadow's rescale division (reciprocal + Markstein correction, IEEE
    fallback outside its domain) must equal IEEE x / b bit for bit."""
    import ctypes
    rng = np.random.default_rng(17)
    n = 1 << 20
    b = 10.0 ** rng.uniform(10.0, 300.0, n)
    x = b * rng.uniform(-1.0, 1.0, n)
    # edges: zeros of both signs, tiny and subnormal numerators, huge and
    # power-of-two divisors, all-ones mantissas, |x| == b
    k = 4096
    x[:k] = np.concatenate([[0.0, -0.0, 5e-324, -5e-324, 2.2250738585072014e-308, 1e-300, 1e-290,
                             2.0 ** -969, 2.0 ** -970, np.nextafter(2.0 ** -968, 0)],
                            rng.uniform(-1, 1, k - 10) * 10.0 ** rng.uniform(-320, 0, k - 10)])
    b[:k] = 10.0 ** rng.uniform(10, 308, k)
    b[k:2 * k] = 2.0 ** rng.integers(34, 1023, k).astype(np.float64)
    b[2 * k:3 * k] = np.nextafter(2.0 ** rng.integers(34, 1024, k).astype(np.float64), 0)
    b[3 * k:3 * k + 16] = [1.7976931348623157e308, 2.0 ** 1022, np.nextafter(2.0 ** 1022, 0),
                           np.nextafter(2.0 ** 1022, np.inf)] * 4
    x[3 * k:4 * k] = b[3 * k:4 * k] * rng.choice([-1.0, 1.0], k)
    out = np.zeros(n)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    N.check(N.lib().dr_debug_rescale(p(x), p(b), n, p(out)), "dr_debug_rescale")
    want = x / b
    same = (out.view(np.uint64) == want.view(np.uint64))
    assert same.all(), (x[~same][:4], b[~same][:4], out[~same][:4], want[~same][:4])


def test_prepared_batch_replay():
    ws = dr.synth.uniform_pcfs(64, seed=9, depth=500, limit_depth=1200)
    reqs = [pcf_request(dr.compile_pcf(w.a, w.b), w.a0, w.depth, 32, checkpoint=w.checkpoint)
            for w in ws]
    b = WalkBatch(reqs)
    b.run()
    r1 = b.read()
    b.run()
    b.run()
    r2 = b.read()
    for x, y, req in zip(r1, r2, reqs):
        assert list(x["p_residues"]) == list(y["p_residues"])
        assert list(x["checkpoint"]["q_residues"]) == list(y["checkpoint"]["q_residues"])
        o = walk_c.pcf_walk(req.blob, req.a0, req.checkpoint, 32)
        assert list(x["checkpoint"]["p_residues"]) == list(o["p_residues"])
    assert b.stats()["prime_steps"] == 64 * 1200 * 32
    b.close()


def test_topk():
    rng = np.random.default_rng(1)
    for n, k in ((10, 3), (5000, 100), (20000, 256), (3, 10)):
        v = rng.standard_normal(n)
        v[rng.integers(0, n, size=min(n, 5))] = np.inf
        v[: min(n, 2)] = v[-1]  # ties
        idx = np.zeros(min(n, k), dtype=np.int32)
        val = np.zeros(min(n, k))
        N.init()
        N.check(N.lib().dr_topk(N.ptr(v), n, k, N.ptr(idx), N.ptr(val)))
        order = sorted(range(n), key=lambda i: (-v[i], i))[:k]
        assert list(idx) == order


def test_pipeline_self_and_fixed():
    import mpmath as mp
    from oracle import walk_np
    ws = dr.synth.uniform_pcfs(48, seed=17, depth=300, limit_depth=900)
    reqs = [pcf_request(dr.compile_pcf(w.a, w.b), w.a0, w.depth, 32, checkpoint=w.checkpoint)
            for w in ws]
    b = WalkBatch(reqs)
    b.set_pipeline(delta="self", topk=10)
    b.run()
    res = b.read()
    pl = b.read_pipeline(values=True)
    pr = [int(p) for p in dr.generate_rns_primes(32)]
    want = []
    for i, r in enumerate(res):
        vals = []
        for arr in (r["p_residues"], r["q_residues"], r["checkpoint"]["p_residues"],
                    r["checkpoint"]["q_residues"]):
            x, M = walk_np.crt([int(v) for v in arr], pr)
            vals.append(walk_np.centered(x, M))
        assert [pl["p"][i], pl["q"][i], pl["cp_p"][i], pl["cp_q"][i]] == vals
        mp.mp.dps = 200
        L = mp.mpf(vals[0]) / mp.mpf(vals[1])
        d = walk_np.delta_exact(vals[2], vals[3], L, 200)
        want.append(d)
        if math.isinf(d):
            assert pl["delta"][i] == d
        else:
            assert abs(pl["delta"][i] - d) < 1e-9, (i, pl["delta"][i], d)
    order = sorted(range(len(want)), key=lambda i: (-pl["delta"][i], i))[:10]
    assert list(pl["topk_idx"]) == order
    # fixed target: pi as an exact binary ratio at dps 200
    mp.mp.dps = 200
    num, den = dr.runner.target_ratio(mp.pi)
    b.set_pipeline(delta="fixed", target=(num, den), topk=5)
    b.run()
    pl2 = b.read_pipeline(values=True)
    for i in range(len(res)):
        d = walk_np.delta_exact(pl2["p"][i], pl2["q"][i], mp.pi, 200)
        assert (pl2["delta"][i] == d) if math.isinf(d) else abs(pl2["delta"][i] - d) < 1e-9
    b.close()


def test_sweep_matches_walks_crt_and_delta():
    """sweep(): one call with array results equals run_walks + per-walk CRT and
    delta through the oracle, for mixed K, checkpoints and rational programs."""
    import mpmath as mp
    from oracle import walk_np
    rng = random.Random(23)
    reqs = []
    for i in range(40):
        a = dr.synth.poly_str([rng.randrange(-9, 10) for _ in range(3)])
        b = dr.synth.poly_str([rng.randrange(-9, 10) for _ in range(4)])
        if i % 4 == 1:
            b = f"({b})/({dr.synth.poly_str([rng.randrange(1, 9), rng.randrange(-3, 4)])})"
        prog = dr.compile_pcf(a, b)
        depth = rng.randrange(300, 1500)
        reqs.append(pcf_request(prog, dr.pcf_initial_values(a), depth, rng.choice([16, 32, 64]),
                                checkpoint=depth // 3))
    out = dr.sweep(reqs, delta="self", topk=7, values=True)
    res = run_walks(reqs)
    for i, (req, r) in enumerate(zip(reqs, res)):
        o = int(out["res_offset"][i])
        c = int(out["cp_res_offset"][i])
        assert list(out["p_residues"][o:o + req.K]) == list(r["p_residues"])
        assert list(out["q_residues"][c:c + req.K]) == list(r["checkpoint"]["q_residues"])
        assert out["shadow"][i][0] == r["p_float"] and out["shadow"][i][2] == r["log_scale"]
        pr = [int(p) for p in dr.generate_rns_primes(req.K)]
        vals = []
        for arr in (r["p_residues"], r["q_residues"], r["checkpoint"]["p_residues"],
                    r["checkpoint"]["q_residues"]):
            x, M = walk_np.crt([int(v) for v in arr], pr)
            vals.append(walk_np.centered(x, M))
        assert [out["p"][i], out["q"][i], out["cp_p"][i], out["cp_q"][i]] == vals
        mp.mp.dps = 200
        d = walk_np.delta_exact(vals[2], vals[3], mp.mpf(vals[0]) / mp.mpf(vals[1]), 200)
        assert (out["delta"][i] == d) if math.isinf(d) else abs(out["delta"][i] - d) < 1e-9
    order = sorted(range(len(reqs)), key=lambda i: (-out["delta"][i], i))[:7]
    assert list(out["topk_idx"]) == order


def test_autotune_keeps_results():
    """The autotuner only changes launch shapes: a batch built after tuning
    (which then uses the remembered shape) gives the same residues."""
    ws = dr.synth.uniform_pcfs(256, seed=31, depth=700, limit_depth=2100)
    reqs = [pcf_request(dr.compile_pcf(w.a, w.b), w.a0, 2100, 32, checkpoint=700) for w in ws]
    before = run_walks(reqs)
    choice = dr.autotune(reqs)
    assert choice["chunk_steps"] >= 256 and choice["warps_per_block"] in (1, 2, 4)
    assert choice["ms"] > 0
    after = run_walks(reqs)
    for x, y in zip(before, after):
        assert list(x["p_residues"]) == list(y["p_residues"])
        assert list(x["checkpoint"]["q_residues"]) == list(y["checkpoint"]["q_residues"])
        assert x["p_float"] == y["p_float"]


def test_large_batch_build_matches_small_batches():
    """Batches of 1024 walks or more are built by several host threads whose
    groups and chunk slots are merged in walk order; the same walks built as
    small batches (one thread) must give identical residues and shadows."""
    rng = random.Random(41)
    progs = [dr.compile_pcf(w.a, w.b) for w in dr.synth.uniform_pcfs(40, seed=41, depth=10, limit_depth=10)]
    rat = [dr.compile_pcf(w.a, w.b) for w in dr.synth.rational_pcfs(12, seed=42, depth_range=(100, 400))]
    reqs = []
    for i in range(2400):
        prog = rat[i % len(rat)] if i % 5 == 0 else progs[i % len(progs)]
        depth = rng.randrange(1, 3000)
        cp = rng.randrange(1, depth) if depth > 2 and i % 3 == 0 else 0
        reqs.append(pcf_request(prog, rng.randrange(-3, 4), depth, rng.choice([16, 32, 64, 96]), checkpoint=cp))
    whole = run_walks(reqs)
    parts = []
    for i in range(0, len(reqs), 600):
        parts += run_walks(reqs[i:i + 600])
    for req, x, y in zip(reqs, whole, parts):
        assert list(x["p_residues"]) == list(y["p_residues"])
        assert list(x["q_residues"]) == list(y["q_residues"])
        for k in ("p_float", "q_float", "log_scale"):
            assert x[k] == y[k] or (math.isnan(x[k]) and math.isnan(y[k])), k
        if req.checkpoint:
            assert list(x["checkpoint"]["p_residues"]) == list(y["checkpoint"]["p_residues"])


def test_vec_walk_golden(golden):
    """run_cmf_walk_vec against the reference's own output (fixture)."""
    from fractions import Fraction
    for w in golden["vec_walks"]:
        prog = CmfProgramFromHex(w["blob"])
        r = dr.run_cmf_walk_vec(prog, w["depth"], w["K"], [tuple(x) for x in w["shifts"]],
                                [Fraction(a, b) for a, b in w["initial_state"]], w["acc_idx"],
                                w["const_idx"], [tuple(x) for x in w["trajectory"]])
        assert list(r["p_residues"]) == w["p_residues"], w["name"]
        assert list(r["q_residues"]) == w["q_residues"], w["name"]
        pf, qf, ls = (float.fromhex(w[k]) for k in ("p_float", "q_float", "log_scale"))
        assert _close(r["p_float"], pf) and _close(r["q_float"], qf) and _close(r["log_scale"], ls, 1e-13)


def CmfProgramFromHex(h):
    return dr.CmfProgram.deserialize(bytes.fromhex(h))


def test_vec_walks_vs_oracle():
    """State-vector walks of random m x m programs (m = 2..4, rational shifts
    and trajectories, rational v(0), any acc/const entries) against the numpy
    restatement of the reference, batched with ordinary walks."""
    from fractions import Fraction
    from oracle import walk_np
    rng = random.Random(41)
    cases, reqs = [], []
    for trial in range(24):
        blob, m, dim = random_program(rng, m_choices=(2, 3, 4))
        shifts = [(rng.randrange(-5, 6), rng.choice([1, 2, 3])) for _ in range(dim)]
        traj = [(rng.randrange(-3, 4), rng.choice([1, 2])) for _ in range(dim)]
        v0 = [Fraction(rng.randrange(-9, 10), rng.randrange(1, 5)) for _ in range(m)]
        acc, const = rng.randrange(m), rng.randrange(m)
        depth = rng.randrange(0, 400)
        K = rng.choice([8, 32, 40])
        cases.append((blob, depth, K, shifts, v0, acc, const, traj))
        reqs.append(dr.vec_request(blob, depth, K, shifts, v0, acc, const, traj))
        if trial % 4 == 0:   # ordinary walks in the same batch
            reqs.append(cmf_request(blob, depth, K, shifts, traj))
            cases.append(None)
    res = run_walks(reqs)
    for c, r in zip(cases, res):
        if c is None:
            continue
        blob, depth, K, shifts, v0, acc, const, traj = c
        o = walk_np.cmf_walk_vec(blob, depth, K, shifts, v0, acc, const, traj)
        assert list(r["p_residues"]) == list(o["p_residues"]), (depth, K)
        assert list(r["q_residues"]) == list(o["q_residues"]), (depth, K)
        if not (math.isnan(o["p_float"]) or math.isnan(r["p_float"])):
            assert _close(r["p_float"], o["p_float"], 1e-9) and _close(r["q_float"], o["q_float"], 1e-9)


def test_shadow_chunks_outside_the_markstein_domain_rerun_exactly():
    """State-vector walks whose v(0) has a tiny or subnormal entry: with a
    diagonal step matrix that entry stays far below the other, so every
    rescale divides numbers outside the domain where the fast chunks'
    Markstein quotient is exact; those chunks must run again with the IEEE
    division and match the reference's numpy results bit for bit."""
    from fractions import Fraction
    from oracle import walk_np
    prog = dr.compile_cmf_from_dict({(0, 0): "x", (1, 1): "x + 1"}, m=2, dim=1, axis_names=["x"])
    blob = prog.serialize()
    cases, reqs = [], []
    for i in range(40):
        v0 = [Fraction(1, 10 ** (310 if i % 2 else 300)), Fraction(1 + i % 3)]
        depth = 100 + i
        cases.append((depth, v0))
        reqs.append(dr.vec_request(blob, depth, 8, [1 + i % 4], v0, 0, 1))
    res = run_walks(reqs)
    for (depth, v0), req, r in zip(cases, reqs, res):
        o = walk_np.cmf_walk_vec(blob, depth, 8, [req.axis[0][0]], v0, 0, 1)
        assert list(r["p_residues"]) == list(o["p_residues"])
        assert r["p_float"] == o["p_float"] and r["q_float"] == o["q_float"], (depth, r["p_float"], o["p_float"])
        assert _close(r["log_scale"], o["log_scale"], 1e-13)


def test_device_crt_overflow_flag_matches_host_rule():
    """The pipeline's CRT-overflow status bits equal the host rule
    (runner.crt_overflowed, the reference's 1% test against the shadow) for
    walks whose K ranges from far too small to ample."""
    from dreams_rns.runner import crt_overflowed
    rng = random.Random(43)
    reqs = []
    for i in range(48):
        a = dr.synth.poly_str([rng.randrange(-9, 10) for _ in range(3)])
        b = dr.synth.poly_str([rng.randrange(-9, 10) for _ in range(4)])
        depth = rng.randrange(60, 900)
        reqs.append(pcf_request(dr.compile_pcf(a, b), dr.pcf_initial_values(a), depth,
                                rng.choice([1, 2, 4, 8, 16, 64, 128]), checkpoint=depth // 2))
    out = dr.sweep(reqs, values=True)
    flagged = 0
    for i, r in enumerate(reqs):
        sh, cps = out["shadow"][i], out["checkpoint_shadow"][i]
        want = crt_overflowed(out["p"][i], out["q"][i], sh[0] / sh[1])
        want_cp = crt_overflowed(out["cp_p"][i], out["cp_q"][i], cps[0] / cps[1])
        st = int(out["status"][i])
        assert bool(st & N.DR_STATUS_CRT_OVERFLOW) == want, (i, r.K, r.depth)
        assert bool(st & N.DR_STATUS_CP_CRT_OVERFLOW) == want_cp, (i, r.K, r.depth)
        flagged += want
    assert 0 < flagged < len(reqs)


def test_constant_bank_on_device():
    """Device bank scores of the top-k hits equal the reference rule
    (compute_delta_against_constant, fixture values for fixed pairs; mpmath
    for the hits) within 1e-9, and the single-pair GPU path matches the
    reference's fixture."""
    import json
    import os
    import mpmath as mp
    from dreams_rns import constants as C
    from oracle import walk_np
    consts = C.load_constants(200)
    by = {c["name"]: c for c in consts}
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "constants.json")))
    for p, q, name, want in g["delta_against"]:
        got = C.compute_delta_against_constant(int(p), int(q), by[name]["value"], 200)
        assert (got == want) if math.isinf(want) else abs(got - want) < 1e-9, (p, q, name, got, want)
    ws = dr.synth.uniform_pcfs(64, seed=47, depth=300, limit_depth=900)
    reqs = [pcf_request(dr.compile_pcf(w.a, w.b), w.a0, 900, 64, checkpoint=300) for w in ws]
    out = dr.sweep(reqs, delta="self", topk=6, values=True, bank=consts)
    bd = out["bank_delta"]
    assert bd.shape == (6, len(consts))
    mp.mp.dps = 200
    for h, w in enumerate(out["topk_idx"]):
        p, q = out["p"][w], out["q"][w]
        for j in (0, 1, 29, 30, 35, len(consts) - 1):
            want = walk_np.delta_exact(p, q, consts[j]["value"], 200)
            got = bd[h][j]
            assert (got == want) if math.isinf(want) else abs(got - want) < 1e-9, (h, j, got, want)
        assert out["bank_best"][h] == consts[int(np.argmax(bd[h]))]["name"]


def test_cmf_sweep_front_end_matches_host_rule():
    """run_cmf_sweep (device walks, CRT, overflow check, bank) reproduces the
    reference's per-walk hit rule computed on the host from the numpy oracle."""
    import mpmath as mp
    from dreams_rns import constants as C
    from dreams_rns.cmf_sweep import run_cmf_sweep
    from dreams_rns.cmf_walk import compile_cmf_spec, shift_to_axis_offsets
    from oracle import walk_np
    consts = C.load_constants(200)
    specs = [{"name": "2F1_a", "p": 2, "q": 1, "a_params": ["1/2", "1"], "b_params": ["3/2"]},
             {"name": "3F2_b", "p": 3, "q": 2, "a_params": ["1", "1", "1"], "b_params": ["2", "2"]}]
    trajs = {2: [[1, 1, 1], [1, 0, 1], [2, 1, 1]], 3: [[1, 1, 1, 1, 1], [1, 0, 0, 1, 1]]}
    shifts = [{"nums": [0, 0, 0, 0, 0]}, {"nums": [1, 0, 2, 0, 1]}, {"nums": [0, 3, 0, 1, 0]}]
    hits = []
    for spec in specs:
        _, h, stats = run_cmf_sweep([spec], trajs[spec["p"]], shifts, depth=120, K=64,
                                    constants=consts, proximity=5e-2)
        hits += h
    mp.mp.dps = 200
    want = []
    for spec in specs:
        dim = spec["p"] + spec["q"]
        for ti, traj in enumerate(trajs[spec["p"]]):
            blob = compile_cmf_spec(spec, trajectory=traj).serialize()
            for si, sh in enumerate(shifts):
                so = (shift_to_axis_offsets(sh, spec["p"]) + [1] * dim)[:dim]
                r = walk_np.cmf_walk(blob, 120, 64, so)
                pr = [int(p) for p in r["primes"]]
                x, M = walk_np.crt([int(v) for v in r["p_residues"]], pr)
                y, _ = walk_np.crt([int(v) for v in r["q_residues"]], pr)
                p_big, q_big = walk_np.centered(x, M), walk_np.centered(y, M)
                est = r["p_float"] / r["q_float"] if abs(r["q_float"]) > 1e-300 else float("nan")
                if not math.isfinite(est):
                    continue
                try:
                    cr = float(p_big) / float(q_big)
                    ok = math.isfinite(cr) and ((abs(cr - est) / abs(est) < 0.01) if abs(est) > 1e-10
                                                else abs(cr - est) < 0.01)
                except (OverflowError, ZeroDivisionError):
                    ok = False
                prox = C.match_against_constants(est, consts, 5e-2)
                log_q = r["log_scale"] + (math.log(abs(r["q_float"])) if abs(r["q_float"]) > 1e-300 else 0.0)
                cand = ([next(c for c in consts if c["name"] == m["name"]) for m in prox] if prox
                        else [c for c in consts if abs(est - c["value_float"]) < 1.0])
                best, bc = float("-inf"), None
                for c in cand:
                    if ok:
                        d = walk_np.delta_exact(p_big, q_big, c["value"], 200)
                    else:
                        err = abs(est - c["value_float"])
                        d = -(1.0 + math.log(err) / log_q) if err > 0 and log_q > 0 else float("-inf")
                    if d > best:
                        best, bc = d, c["name"]
                if best > 0 or prox:
                    want.append((spec["name"], ti, si, bc, best, [m["name"] for m in prox]))
    got = [(h["cmf_name"], h["traj_idx"], h["shift_idx"], h["best_const"], h["best_delta"],
            h["proximity_matches"]) for h in hits]
    assert len(got) == len(want) and len(want) > 0
    for g, w in zip(got, want):
        assert g[:4] == w[:4] and g[5] == w[5], (g, w)
        assert (g[4] == w[4]) if math.isinf(w[4]) else abs(g[4] - w[4]) < 1e-9, (g, w)
