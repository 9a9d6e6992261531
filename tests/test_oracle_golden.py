"""Pin the CPU oracles to the reference's own outputs (tests/golden).

The numpy and C restatements must reproduce every golden walk bit for bit
(residues and float shadow), the CRT values, the deltas and the prime table.
"""

import math

import numpy as np
import pytest

from oracle import walk_c, walk_np


def _shadow_equal(r, w):
    return (r["p_float"] == float.fromhex(w["p_float"]) and
            r["q_float"] == float.fromhex(w["q_float"]) and
            r["log_scale"] == float.fromhex(w["log_scale"]))


def test_primes_match_reference(golden):
    assert golden["primes_prefix_ok"]
    assert list(walk_np.primes(512)) == golden["primes_512"]
    # pins from the reference's C++ tests and README
    assert golden["primes_512"][0] == 2147483647
    assert golden["primes_512"][63] == 2147482237


@pytest.mark.parametrize("impl", ["np", "c"])
def test_pcf_walks(golden, impl):
    for w in golden["pcf_walks"]:
        if impl == "np" and w["depth"] * w["K"] > 200_000:
            continue
        blob = bytes.fromhex(w["blob"])
        mod = walk_np if impl == "np" else walk_c
        r = mod.pcf_walk(blob, w["a0"], w["depth"], w["K"], w["shift"])
        assert list(r["p_residues"]) == w["p_residues"], w["name"]
        assert list(r["q_residues"]) == w["q_residues"], w["name"]
        assert _shadow_equal(r, w), w["name"]


def test_config1_pins(golden):
    w = golden["pcf_walks"][0]
    assert w["name"] == "config1"
    assert w["p_residues"][:4] == [1351318807, 964958733, 777601130, 1778219253]
    assert w["q_residues"][:4] == [630692060, 1013274209, 1171650986, 1618286415]
    v = golden["verify_pcf"][0]["result"]
    assert abs(float(v["delta_float"]) - (-0.998855)) < 1e-6   # reference README.md:30
    assert v["p_bits"] == 992                                   # reference README.md:31


@pytest.mark.parametrize("impl", ["np", "c"])
def test_cmf_walks(golden, impl):
    for w in golden["cmf_walks"]:
        if impl == "np" and w["depth"] * w["K"] > 100_000:
            continue
        blob = bytes.fromhex(w["blob"])
        mod = walk_np if impl == "np" else walk_c
        tr = w["trajectory"]
        r = mod.cmf_walk(blob, w["depth"], w["K"], [tuple(x) for x in w["shifts"]],
                         None if tr is None else [tuple(x) for x in tr])
        assert list(r["p_residues"]) == w["p_residues"], w["name"]
        assert list(r["q_residues"]) == w["q_residues"], w["name"]
        assert _shadow_equal(r, w), w["name"]


def test_vec_walk(golden):
    from fractions import Fraction
    for w in golden["vec_walks"]:
        r = walk_np.cmf_walk_vec(bytes.fromhex(w["blob"]), w["depth"], w["K"],
                                 [tuple(x) for x in w["shifts"]],
                                 [Fraction(a, b) for a, b in w["initial_state"]],
                                 w["acc_idx"], w["const_idx"], [tuple(x) for x in w["trajectory"]])
        assert list(r["p_residues"]) == w["p_residues"]
        assert list(r["q_residues"]) == w["q_residues"]
        assert _shadow_equal(r, w)


def test_crt(golden):
    for c in golden["crt"]:
        x, M = walk_np.crt(c["residues"], c["primes"])
        assert hex(x) == c["x"] and hex(M) == c["M"]
        assert hex(walk_np.centered(x, M)) == c["centered"]
        if "value" in c:
            v = int(c["value"], 16)
            if 0 <= v < M:
                assert x == v


def test_delta_exact(golden):
    for d in golden["delta_exact"]:
        got = walk_np.delta_exact(int(d["p"], 16), int(d["q"], 16), d["target"], d["dps"])
        want = float(d["delta"])
        if math.isinf(want):
            assert got == want
        else:
            assert abs(got - want) < 1e-12, d["name"]


def test_delta_float(golden):
    for d in golden["delta_float"]:
        args = [float(a) for a in d["args"]]
        got, lq = walk_np.delta_float(*args)
        want, wlq = float(d["delta"]), float(d["log_q"])
        assert (got == want) or (math.isnan(got) and math.isnan(want))
        assert lq == wlq


def test_estimate_k_and_overflow_match_reference():
    """Auto-K and the CRT-overflow rule (host side) against the reference's
    own outputs (tests/golden/make_estimate_k.py)."""
    import json
    import os
    from dreams_rns.runner import crt_overflowed, estimate_K
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "estimate_k.json")))
    for a, b, d, want in g["estimate_K"]:
        assert estimate_K(a, b, d) == want, (a, b, d)
    for p, q, e, want in g["crt_overflowed"]:
        assert crt_overflowed(int(p), int(q), float(e)) == want, (p, q, e)


def test_constant_bank_host_side_matches_reference():
    """Registry, digit matching and proximity lists equal the reference's
    (tests/golden/make_constants.py)."""
    import json
    import os
    from dreams_rns import constants as C
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "constants.json")))
    assert [[e["name"], e["sympy_expr"]] for e in C.CONSTANTS_REGISTRY] == g["registry"]
    consts = C.load_constants(200)
    for e, name, digits in g["match_digits"]:
        got = C.compute_match_digits(e, consts)
        assert got[0] == name and abs(got[1] - digits) < 1e-9, (e, got, name, digits)
    for e, names in g["near"]:
        assert [m["name"] for m in C.match_against_constants(e, consts, 1e-2)] == names
