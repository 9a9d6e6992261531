"""Native library checks that need no GPU: exports, prime table, planner,
and the host re-statement of the device schedule against the C oracle."""

import ctypes
import os
import random
import re

import numpy as np
import pytest

from conftest import ROOT, native_lib_path
from oracle import walk_c
from progfuzz import random_axis, random_program


@pytest.fixture(scope="module")
def L():
    path = native_lib_path()
    if not os.path.exists(path):
        pytest.skip("libdreams_b200.so not built")
    lib = ctypes.CDLL(path)
    lib.dr_debug_sim_walk.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_int32, ctypes.c_uint64,
                                      ctypes.c_uint64, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64,
                                      ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int32, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    lib.dr_program_info.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_void_p]
    lib.dr_last_error.restype = ctypes.c_char_p
    return lib


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*|int32_t)\s*(dr_\w+)\s*\(", text, re.M)))


def test_exports_every_declared_symbol(L):
    names = _declared("dreams_b200.h") + _declared("dreams_b200_debug.h")
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_prime_table(L, golden):
    out = np.zeros(512, dtype=np.uint32)
    assert L.dr_prime_table(512, out.ctypes.data_as(ctypes.c_void_p)) == 0
    assert list(out) == golden["primes_512"]


def _info(L, blob):
    c, d, r = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
    rc = L.dr_program_info(blob, len(blob), ctypes.byref(c), ctypes.byref(d), ctypes.byref(r))
    return rc, c.value, d.value


def test_program_errors(L, golden):
    blob = bytes.fromhex(golden["pcf_walks"][0]["blob"])
    assert _info(L, blob)[0] == 0
    assert _info(L, blob[:20])[0] == -3                     # truncated
    bad = bytearray(blob)
    bad[16] = 77                                             # opcode 77
    assert _info(L, bytes(bad))[0] == -4
    bad = bytearray(blob)
    bad[16 + 4:16 + 8] = (5).to_bytes(4, "little")           # LOAD_X axis 5 of 1
    assert _info(L, bytes(bad))[0] == -5


def test_classes_of_reference_programs(L, golden):
    seen = {}
    for w in golden["pcf_walks"] + golden["cmf_walks"]:
        rc, cls, deg = _info(L, bytes.fromhex(w["blob"]))
        assert rc == 0
        seen.setdefault(cls, []).append(w["name"])
    assert "config1" in seen[1]                              # b = n^2: companion polynomial
    assert "rational" in seen[2] and "inv0_one_prime" in seen[2]
    assert "config4_full" in seen[1]


def test_instances_cover_planner(L):
    L.dr_debug_template_degree.argtypes = [ctypes.c_int32] * 3
    text = open(os.path.join(ROOT, "dreams-rns-cuda_b200", "csrc", "instances.h")).read()
    lists = {}
    for name, cls in (("COMPANION", 1), ("RATIONAL", 2), ("DENSE", 3)):
        body = text.split(f"DR_{name}_INSTANCES(X)")[1].split("\n\n")[0]
        lists[cls] = set((int(a), int(b)) for a, b in re.findall(r"X\((\d+), (\d+)\)", body))
    for cls in (1, 2, 3):
        for m in range(1, 9):
            for deg in range(0, 18):
                D = L.dr_debug_template_degree(cls, m, deg)
                if D >= 0:
                    assert (m, D) in lists[cls], (cls, m, deg, D)


def _sim(L, blob, K, depth, axis, pcf, a0, qrow, chunk, cp=0, force=0):
    p = np.zeros(K, np.uint32)
    q = np.zeros(K, np.uint32)
    cpp = np.zeros(K, np.uint32)
    cpq = np.zeros(K, np.uint32)
    axis = np.ascontiguousarray(axis, np.int64)
    rc = L.dr_debug_sim_walk(blob, len(blob), K, depth, cp, axis.ctypes.data, pcf, a0, qrow,
                             chunk, force, p.ctypes.data, q.ctypes.data, cpp.ctypes.data,
                             cpq.ctypes.data)
    assert rc == 0, L.dr_last_error()
    return p, q, cpp, cpq


def test_schedule_matches_reference_fixtures(L, golden):
    from oracle.walk_np import parse_blob
    for w in golden["pcf_walks"]:
        blob = bytes.fromhex(w["blob"])
        dirs = parse_blob(blob)[4]
        axis = np.array([[w["shift"], 1, d, 1] for d in dirs]).reshape(-1)
        for chunk in (0, 7):
            p, q, _, _ = _sim(L, blob, w["K"], w["depth"], axis, 1, w["a0"], 1, chunk)
            assert list(p) == w["p_residues"] and list(q) == w["q_residues"], w["name"]
    for w in golden["cmf_walks"]:
        blob = bytes.fromhex(w["blob"])
        m, dim, _, _, dirs = parse_blob(blob)
        sh = w["shifts"]
        tr = w["trajectory"] or [[d, 1] for d in dirs]
        axis = np.array([[sh[a][0], sh[a][1], tr[a][0], tr[a][1]] for a in range(dim)]).reshape(-1)
        p, q, _, _ = _sim(L, blob, w["K"], w["depth"], axis, 0, 0, m - 1, 13)
        assert list(p) == w["p_residues"] and list(q) == w["q_residues"], w["name"]


def test_schedule_random_programs(L):
    rng = random.Random(7)
    for trial in range(250):
        blob, m, dim = random_program(rng)
        if _info(L, blob)[0] != 0:
            continue
        K = rng.choice([1, 3, 8])
        depth = rng.randrange(0, 50)
        axis = np.array(random_axis(rng, dim, rng.random() < 0.4), np.int64)
        pcf = int(m == 2 and rng.random() < 0.5)
        a0 = rng.randrange(-9, 10)
        init = np.eye(m, dtype=np.int64)
        if pcf:
            init[0, 1] = a0
        qrow = 1 if pcf else m - 1
        ref = walk_c.walk(blob, depth, K, axis, init, 0, qrow, shadow=False)
        cp = rng.randrange(1, depth) if depth > 2 and rng.random() < 0.5 else 0
        p, q, cpp, cpq = _sim(L, blob, K, depth, axis, pcf, a0, qrow, rng.choice([0, 1, 5, 17]), cp)
        assert list(p) == list(ref["p_residues"]) and list(q) == list(ref["q_residues"]), trial
        if cp:
            r2 = walk_c.walk(blob, cp, K, axis, init, 0, qrow, shadow=False)
            assert list(cpp) == list(r2["p_residues"]) and list(cpq) == list(r2["q_residues"])


def test_walk_without_init_is_an_error():
    import subprocess, sys
    code = ("import sys; sys.path.insert(0, %r); import ctypes; from dreams_rns import _native as N; "
            "L = N.lib(); rc = L.dr_walk_batch(None, 0, None, None, 0, None, 0, None, None, None, 0, None, None); "
            "print(rc)") % os.path.join(ROOT, "dreams-rns-cuda_b200")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert out.stdout.strip() == "-8", out.stderr


def test_request_packing_extension_matches_python():
    """The packing extension (csrc/pack.c) gives the same arrays as its
    pure-Python statement, including the negative-depth clamp and the errors."""
    import copy
    from fractions import Fraction

    import dreams_rns as dr
    from dreams_rns import engine
    if engine._pack_ext is None:
        pytest.skip("dreams_rns._pack not built")
    rng = random.Random(7)
    pcfs = [dr.compile_pcf(a, b) for a, b in [("2", "n**2"), ("3*n+1", "-2*n**2"), ("n", "(n+1)/(n+2)")]]
    cmf = dr.compile_cmf_from_dict({(0, 0): "1", (0, 1): "x", (1, 0): "y", (1, 1): "x+y"}, m=2, dim=2,
                                   axis_names=["x", "y"])
    reqs = []
    for i in range(300):
        kind = i % 4
        if kind == 0:
            depth = rng.randrange(-5, 900)
            cp = rng.randrange(1, depth) if depth > 2 and i % 3 == 0 else 0
            reqs.append(engine.pcf_request(pcfs[i % 3], rng.randrange(-9, 10), depth, rng.choice([1, 16, 32, 96]),
                                           checkpoint=cp, shadow=i % 5 != 0))
        elif kind == 1:
            reqs.append(engine.cmf_request(cmf, rng.randrange(1, 600), rng.choice([8, 32]),
                                           [Fraction(rng.randrange(-5, 6), rng.randrange(1, 4)), 2],
                                           [1, Fraction(rng.randrange(1, 4), rng.randrange(1, 3))]))
        elif kind == 2:
            reqs.append(engine.vec_request(cmf, rng.randrange(1, 400), 8, [1, 1], [1, Fraction(1, 3)], 0, 1))
        else:
            reqs.append(engine.pcf_request(pcfs[0], 2, rng.randrange(0, 50), 64))
    for batch in (reqs, reqs[:1], []):
        a_reqs, b_reqs = copy.deepcopy(batch), copy.deepcopy(batch)
        a, b = engine._pack_ext.pack(a_reqs), engine._pack_py(b_reqs)
        assert (a[0], a[7], a[8]) == (b[0], b[7], b[8])
        n = len(batch)
        sizes = [8 * (a[0] + 1), None, engine.N.WALK_DTYPE.itemsize * n, 8 * n, 8 * n, 8 * max(a[7], 1)]
        for k, (x, y) in enumerate(zip(a[1:7], b[1:7])):
            lim = sizes[k]
            assert bytes(x)[:lim] == bytes(y)[:lim], k
        assert [r.depth for r in a_reqs] == [r.depth for r in b_reqs]   # negative depths clamped alike
    # requests of another type than the first one's (a subclass with a
    # property over a slot), blobs equal by content but not identity: the
    # generic attribute path and content de-duplication
    class Req(engine.WalkRequest):
        __slots__ = ()

        @property
        def K(self):
            return 8

        @K.setter
        def K(self, v):
            pass

    mixed = copy.deepcopy(reqs[:40])
    for i in range(0, 40, 3):
        r = mixed[i]
        mixed[i] = Req(blob=bytes(bytearray(r.blob)), K=r.K, depth=r.depth, axis=r.axis, a0=r.a0,
                       pcf_init=r.pcf_init, q_row=r.q_row, checkpoint=r.checkpoint, shadow=r.shadow,
                       p_row=r.p_row, vec=r.vec)
    a_reqs, b_reqs = copy.deepcopy(mixed), copy.deepcopy(mixed)
    a, b = engine._pack_ext.pack(a_reqs), engine._pack_py(b_reqs)
    assert (a[0], a[7], a[8]) == (b[0], b[7], b[8])
    for k, (x, y) in enumerate(zip(a[1:7], b[1:7])):
        assert bytes(x) == bytes(y), k
    unset = engine.pcf_request(pcfs[0], 2, 10, 1)
    del unset.K                          # an empty slot raises as attribute access does
    for f in (engine._pack_ext.pack, engine._pack_py):
        with pytest.raises(AttributeError):
            f([copy.deepcopy(reqs[0]), copy.copy(unset)])
    bad_k = [engine.pcf_request(pcfs[0], 2, 10, 1)]
    bad_k[0].K = 0
    bad_a0 = [engine.pcf_request(pcfs[0], 2, 10, 1)]
    bad_a0[0].a0 = 2 ** 70
    bad_axis = [engine.pcf_request(pcfs[0], 2, 10, 1)]
    bad_axis[0].axis = [(2 ** 70, 1, 1, 1)]
    for bad, exc in ((bad_k, ValueError), (bad_a0, OverflowError), (bad_axis, OverflowError)):
        with pytest.raises(exc):
            engine._pack_ext.pack(copy.deepcopy(bad))
        with pytest.raises(exc):
            engine._pack_py(copy.deepcopy(bad))


def test_host_pool_covers_every_index_once(L):
    """The batch build's host thread pool: jobs with 1..16 contiguous parts
    over [0, n) visit every index exactly once, job after job."""
    L.dr_debug_host_pool.argtypes = [ctypes.c_int32, ctypes.c_uint64, ctypes.c_int32, ctypes.c_void_p,
                                     ctypes.c_void_p]
    for n in (0, 1, 7, 1000, 100_003):
        s, v = ctypes.c_uint64(), ctypes.c_uint64()
        assert L.dr_debug_host_pool(16, n, 64, ctypes.byref(s), ctypes.byref(v)) == 0
        assert v.value == 64 * n
        assert s.value == 64 * (n * (n - 1) // 2)


def test_read_pipeline_limb_stride_from_descriptors(monkeypatch):
    """WalkBatch.read_pipeline passes no limb buffer unless values are asked
    for, and then a limb stride of ceil(31 Kmax / 32) + 2 with Kmax taken from
    the packed descriptors (a stand-in library records the call; no GPU)."""
    import dreams_rns as dr
    from dreams_rns import engine
    prog = dr.compile_pcf("2", "n**2")
    reqs = [engine.pcf_request(prog, 2, 50, K, checkpoint=20) for K in (16, 96, 32)]
    seen = {}

    class Lib:
        def dr_batch_read_pipeline(self, h, delta, ti, tv, limbs, signs, stride):
            seen["limbs"], seen["stride"] = limbs is not None, stride
            return 0

    monkeypatch.setattr(engine.N, "lib", lambda: Lib())
    b = object.__new__(engine.WalkBatch)
    b.reqs, b.pk, b.handle = reqs, engine._Packed(reqs), 1
    b.pipeline = {"topk": 2, "delta": True}
    try:
        out = b.read_pipeline()
        assert seen == {"limbs": False, "stride": 0}
        assert sorted(out) == ["delta", "topk_idx", "topk_val"]
        out = b.read_pipeline(values=True)
        assert seen == {"limbs": True, "stride": (31 * 96 + 31) // 32 + 2}
        assert len(out["p"]) == len(out["cp_q"]) == 3
    finally:
        b.handle = 0


def test_stage_timers_need_no_gpu(L):
    """dr_stage_times reads and resets the per-stage sums without a device;
    a batch call that fails before building adds nothing to them."""
    ms = (ctypes.c_double * 5)()
    calls = (ctypes.c_uint64 * 5)()
    L.dr_stage_times.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32]
    assert L.dr_stage_times(ms, calls, 5, 1) == 0
    assert L.dr_stage_times(ms, calls, 5, 0) == 0
    assert list(calls) == [0] * 5 and list(ms) == [0.0] * 5
    assert L.dr_stage_times(None, None, 5, 0) != 0          # null output
    assert L.dr_stage_times(ms, None, -1, 0) != 0           # negative count
    assert L.dr_stage_times(ms, None, 2, 0) == 0            # a prefix is fine


def test_debug_build_exports_the_same_symbols():
    """The DR_DEBUG library (build.py --debug) offers the same C ABI and
    reports its checks; the normal one reports none."""
    dbg = os.path.join(os.path.dirname(native_lib_path()), "libdreams_b200_debug.so")
    if not os.path.exists(dbg):
        pytest.skip("debug library not built")
    names = _declared("dreams_b200.h") + _declared("dreams_b200_debug.h")
    D = ctypes.CDLL(dbg)
    assert [n for n in names if not hasattr(D, n)] == []
    flag = ctypes.c_int32(-1)
    assert D.dr_debug_build_info(ctypes.byref(flag)) == 0 and flag.value == 1
    R = ctypes.CDLL(native_lib_path())
    assert R.dr_debug_build_info(ctypes.byref(flag)) == 0 and flag.value == 0
