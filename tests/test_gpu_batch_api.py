"""The reference's batched GPU entry points (python/dreams_rns/gpu_walk.py:279-489)
on the B200 engine: same result keys, every walk against the C oracle.

Differences from the reference that are by design: every walk gets its own
FP64 shadow (the reference reports the first walk's shadow for the whole
batch, gpu_walk.py:345-363) and INV runs on the device.
"""

import numpy as np
import pytest

import dreams_rns as dr
from oracle import walk_c

pytestmark = pytest.mark.gpu

PCF_KEYS = {"p_residues", "q_residues", "p_float", "q_float", "log_scale", "primes", "shift_val"}
CMF_KEYS = {"p_residues", "q_residues", "p_float", "q_float", "log_scale", "primes", "shift_vals"}


def _close(a, b, rtol=1e-12):
    return a == b or abs(a - b) <= rtol * max(abs(a), abs(b), 1e-300)


def test_run_pcf_walk_batch_gpu_matches_oracle():
    prog = dr.compile_pcf("3*n + 1", "-2*n**2 + n")
    shifts = [1, 2, 5, -3, 17, 0]
    out = dr.run_pcf_walk_batch_gpu(prog, 1, 1500, 48, shift_vals=shifts, batch_size=4)
    assert len(out) == len(shifts)
    for sv, r in zip(shifts, out):
        assert set(r) == PCF_KEYS
        assert r["shift_val"] == sv
        assert r["p_residues"].dtype == np.int64 and r["p_residues"].shape == (48,)
        o = walk_c.pcf_walk(prog.serialize(), 1, 1500, 48, shift=sv)
        assert list(r["p_residues"]) == list(o["p_residues"]), sv
        assert list(r["q_residues"]) == list(o["q_residues"]), sv
        assert list(r["primes"]) == list(o["primes"])
        assert _close(r["p_float"], o["p_float"]) and _close(r["q_float"], o["q_float"]), sv
        assert _close(r["log_scale"], o["log_scale"], 1e-13), sv
    single = dr.run_pcf_walk_gpu(prog, 1, 1500, 48, shift_val=5)
    assert list(single["p_residues"]) == list(out[2]["p_residues"])
    with pytest.raises(AssertionError):
        dr.run_pcf_walk_batch_gpu(dr.compile_cmf_from_dict({(0, 0): "x0"}, 1, 1), 0, 10, 8)


def test_run_cmf_walk_batch_gpu_matches_oracle():
    mat = {(0, 2): "x*y + z", (1, 0): "1", (1, 2): "x - 2*z**2", (2, 1): "1", (2, 2): "x + y + z"}
    prog = dr.compile_cmf_from_dict(mat, m=3, dim=3, axis_names=["x", "y", "z"])
    shifts = [[1, 1, 1], [2, -1, 0], [0, 3, -2], [-3, -3, 1]]
    out = dr.run_cmf_walk_batch_gpu(prog, 900, 40, shift_val_list=shifts, batch_size=2)
    assert len(out) == len(shifts)
    for sv, r in zip(shifts, out):
        assert set(r) == CMF_KEYS
        assert r["shift_vals"] == sv
        o = walk_c.cmf_walk(prog.serialize(), 900, 40, sv)
        assert list(r["p_residues"]) == list(o["p_residues"]), sv
        assert list(r["q_residues"]) == list(o["q_residues"]), sv
        assert _close(r["p_float"], o["p_float"]) and _close(r["q_float"], o["q_float"]), sv
    one = dr.run_cmf_walk_gpu(prog, 900, 40, shifts[1])
    assert list(one["q_residues"]) == list(out[1]["q_residues"])


def test_stage_times_cover_a_sweep():
    """The per-stage timers see every stage of one sweep() call."""
    from dreams_rns.engine import pcf_request
    prog = dr.compile_pcf("2", "n**2")
    reqs = [pcf_request(prog, 2, 2000, 32, shift_val=s, checkpoint=500) for s in (1, 2, 3, 4)]
    dr.stage_times(reset=True)
    out = dr.sweep(reqs, delta="self", topk=2)
    st = dr.stage_times(reset=True)
    assert len(out["topk_idx"]) == 2
    for k in ("pack", "build", "upload", "run", "read", "device"):
        assert st[f"{k}_calls"] >= 1 and st[f"{k}_ms"] > 0, (k, st)
    assert dr.stage_times()["build_calls"] == 0


def test_sweep_many_equals_sweep_per_list():
    """sweep_many over several lists (the next lists built while the device
    walks the current one) gives each list what sweep() gives it, in order;
    closing the generator early releases the batches it had prepared."""
    from dreams_rns.engine import pcf_request
    progs = [dr.compile_pcf("2", "n**2"), dr.compile_pcf("3*n + 1", "-2*n**2 + n"),
             dr.compile_pcf("n + 5", "n**3 - 7")]
    lists = []
    for j in range(5):
        lists.append([pcf_request(progs[(j + i) % 3], 1 + i, 1200 + 300 * j, 32, shift_val=1 + i,
                                  checkpoint=400) for i in range(6 + 2 * j)])
    want = [dr.sweep(r, delta="self", topk=3) for r in lists]
    got = list(dr.sweep_many(lists, delta="self", topk=3, lookahead=2))
    assert len(got) == len(lists)
    for w, g in zip(want, got):
        for key in ("p_residues", "q_residues", "topk_idx"):
            assert np.array_equal(np.asarray(w[key]), np.asarray(g[key])), key
        assert np.array_equal(w["shadow"], g["shadow"])
        assert np.array_equal(w["delta"], g["delta"], equal_nan=True)
    gen = dr.sweep_many(lists, delta="self", topk=3, lookahead=3)
    first = next(gen)
    assert np.array_equal(np.asarray(first["topk_idx"]), np.asarray(want[0]["topk_idx"]))
    gen.close()
    assert np.array_equal(np.asarray(dr.sweep(lists[1], delta="self", topk=3)["p_residues"]),
                          np.asarray(want[1]["p_residues"]))


def test_chain_packing_changes_no_result():
    """Two integer-difference chain warps per scheduler (dr_tune.chain_pack_depth)
    is a launch-shape choice: residues, shadows and statuses are the same."""
    from dreams_rns.engine import WalkBatch, pcf_request
    progs = [dr.compile_pcf("3*n + 1", "-2*n**2 + n"), dr.compile_pcf("n + 2", "n**3 + 5*n")]
    reqs = [pcf_request(progs[i % 2], 1 + i % 3, 3000 + 97 * i, 32, shift_val=1 + i, checkpoint=700)
            for i in range(70)]
    out = []
    for pack in (0, 16):
        b = WalkBatch(reqs, chain_pack_depth=pack)
        b.run()
        out.append(b.read_arrays())
        b.close()
    for key in ("p_residues", "q_residues"):
        assert np.array_equal(out[0][key], out[1][key]), key
    assert np.array_equal(out[0]["shadow"], out[1]["shadow"])


def test_sweep_many_reports_a_bad_list_and_recovers():
    """An invalid list (a walk with K = 0) raises from sweep_many when its turn
    comes; the lists before it were yielded, the batches prepared after it are
    released, and the engine keeps working."""
    from dreams_rns.engine import pcf_request
    prog = dr.compile_pcf("2", "n**2")
    good = [pcf_request(prog, 2, 1500, 32, shift_val=s, checkpoint=300) for s in (1, 2, 3)]
    bad = [pcf_request(prog, 2, 1500, 32)]
    bad[0].K = 0
    gen = dr.sweep_many([good, bad, good, good], delta="self", topk=2)
    first = next(gen)
    with pytest.raises((ValueError, RuntimeError)):
        next(gen)
    gen.close()
    again = dr.sweep(good, delta="self", topk=2)
    assert np.array_equal(np.asarray(first["topk_idx"]), np.asarray(again["topk_idx"]))
    assert np.array_equal(first["p_residues"], again["p_residues"])
