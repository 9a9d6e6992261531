"""Split FP64 shadows on the GPU: walks whose float intermediates are exact
integers below 2^53 only over their first steps (quartic b(n) with large
coefficients, deep walks) run those steps on integer differences and the
rest on the evaluated step matrices, inside one chain kernel.  The shadow
must equal the reference's (runner.py:393-398, through the C oracle) on
either side of the switch, with checkpoints before and after it, in full and
partial items; the residues are unaffected."""

import math

import numpy as np
import pytest

import dreams_rns as dr
from dreams_rns import _native as N
from dreams_rns.engine import WalkBatch, pcf_request
from oracle import walk_c

pytestmark = pytest.mark.gpu


def _close(a, b, rtol=1e-12):
    if a == b or (math.isnan(a) and math.isnan(b)):
        return True
    return abs(a - b) <= rtol * max(abs(a), abs(b), 1e-300)


def _shadow_ok(got, want):
    return (_close(got["p_float"], want["p_float"]) and _close(got["q_float"], want["q_float"])
            and _close(got["log_scale"], want["log_scale"], 1e-13))


def test_split_shadow_matches_oracle():
    rng = np.random.default_rng(11)
    walks = []
    for i in range(70):
        c4 = int(rng.integers(4, 11)) * (1 if i % 2 else -1)
        c2 = int(rng.integers(-9, 10))
        c0 = int(rng.integers(1, 10))
        a1, a0c = int(rng.integers(1, 6)), int(rng.integers(-5, 6))
        a, b = f"{a1}*n + {a0c}", f"{c4}*n**4 + {c2}*n**2 + {c0}"
        depth = int(rng.integers(6000, 9000))
        cp = (500, 7000, 0)[i % 3]
        walks.append((a, b, depth, cp))
    progs = {}
    reqs = []
    for a, b, depth, cp in walks:
        if (a, b) not in progs:
            progs[(a, b)] = dr.compile_pcf(a, b)
        reqs.append(pcf_request(progs[(a, b)], dr.pcf_initial_values(a), depth, 32,
                                checkpoint=cp if cp < depth else 0))
    batch = WalkBatch(reqs)
    prof = batch.profile()
    assert any(p["kind"] == 1 and p["degree"] > 0 for p in prof), prof      # the split path ran
    batch.run()
    res = batch.read()
    batch.close()
    for i, ((a, b, depth, cp), r) in enumerate(zip(walks, res)):
        blob = progs[(a, b)].serialize()
        a0 = dr.pcf_initial_values(a)
        fin = walk_c.pcf_walk(blob, a0, depth, 32)
        assert list(r["p_residues"]) == list(fin["p_residues"]), i
        assert list(r["q_residues"]) == list(fin["q_residues"]), i
        assert _shadow_ok(r, fin), (i, r["p_float"], fin["p_float"], r["log_scale"], fin["log_scale"])
        if cp and cp < depth:
            want = walk_c.pcf_walk(blob, a0, cp, 32)
            assert _shadow_ok(r["checkpoint"], want), (i, cp)
