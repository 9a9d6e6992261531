"""The DR_DEBUG build (device bounds checks on every table index a walk
tile uses, csrc/debug_check.cuh) gives the same results as the normal build
on the reference fixtures and the fuzzed programs, with no check failing.
It runs in a child process, since the library is chosen at import
(DREAMS_B200_DEBUG=1)."""

import os
import subprocess
import sys

import pytest

from conftest import PKG, ROOT

pytestmark = pytest.mark.gpu

CHILD = r"""
import ctypes, json, random, sys
sys.path[:0] = [{root!r}, {pkg!r}, {tests!r}]
import dreams_rns as dr
from dreams_rns import _native as N
from dreams_rns.engine import cmf_request, pcf_request, run_walks
from oracle import walk_c
from progfuzz import random_axis, random_program
assert N.LIB_PATH.endswith("libdreams_b200_debug.so"), N.LIB_PATH
flag = ctypes.c_int32()
N.check(N.lib().dr_debug_build_info(ctypes.byref(flag)), "build info")
assert flag.value == 1
g = json.load(open({golden!r}))
reqs = [pcf_request(bytes.fromhex(w["blob"]), w["a0"], w["depth"], w["K"], w["shift"]) for w in g["pcf_walks"]]
for chunk in (0, 97):
    for w, r in zip(g["pcf_walks"], run_walks(reqs, chunk_steps=chunk)):
        assert list(r["p_residues"]) == w["p_residues"], w["name"]
        assert list(r["q_residues"]) == w["q_residues"], w["name"]
import numpy as np
from dreams_rns.engine import WalkRequest
rng = random.Random(3)
reqs, refs = [], []
while len(reqs) < 60:
    blob, m, dim = random_program(rng)
    try:
        N.program_info(blob)
    except Exception:
        continue
    depth = rng.randrange(0, 300)
    axis = random_axis(rng, dim, rng.random() < 0.4)
    reqs.append(WalkRequest(blob=blob, K=40, depth=depth, q_row=m - 1,
                            axis=[tuple(axis[4 * a:4 * a + 4]) for a in range(dim)], shadow=False))
    refs.append(walk_c.walk(blob, depth, 40, np.array(axis, np.int64), np.eye(m, dtype=np.int64), 0, m - 1,
                            shadow=False))
for r, o in zip(run_walks(reqs, chunk_steps=37), refs):
    assert list(r["p_residues"]) == list(o["p_residues"])
    assert list(r["q_residues"]) == list(o["q_residues"])
print("debug build ok")
"""


def test_debug_build_matches_fixtures():
    lib = os.path.join(PKG, "dreams_rns", "_native", "libdreams_b200_debug.so")
    if not os.path.exists(lib):
        pytest.fail("libdreams_b200_debug.so is not built (build.py --debug)")
    code = CHILD.format(root=ROOT, pkg=PKG, tests=os.path.join(ROOT, "tests"),
                        golden=os.path.join(ROOT, "tests", "golden", "reference_golden.json"))
    env = dict(os.environ, DREAMS_B200_DEBUG="1")
    res = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-4000:]
    assert "debug build ok" in res.stdout
