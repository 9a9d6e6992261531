"""Generate the golden fixtures in this directory from the reference itself.

Run in a container where the reference checkout is mounted read-only::

    python tests/golden/make_golden.py <reference checkout>/python

It imports the reference ``dreams_rns`` package (numpy / sympy / mpmath only)
and records, for seeded and hand-picked inputs, what the reference computes:
compiled program blobs, walk residues and float shadows, CRT values, deltas
and ``verify_pcf`` results.  The GPU box has no reference checkout, so the
tests only ever read the JSON written here.
"""

from __future__ import annotations

import json
import math
import os
import sys
import time
from fractions import Fraction

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
PKG_DIR = os.path.join(REPO, "dreams-rns-cuda_b200")


def _fhex(x) -> str:
    return float(x).hex()


def _blob_hex(prog) -> str:
    return prog.serialize().hex()


def main(ref_python: str) -> None:
    sys.path.insert(0, ref_python)
    import numpy as np
    import mpmath as mp
    import dreams_rns as ref                        # the reference package
    from dreams_rns import cmf_walk as ref_cmf      # reference CMF engine

    sys.path.insert(0, PKG_DIR)
    # our synth generators only build input strings; import the module file
    # directly so that the reference package keeps the name dreams_rns
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "b200_synth", os.path.join(PKG_DIR, "dreams_rns", "synth.py"))
    synth = importlib.util.module_from_spec(spec)
    sys.modules["b200_synth"] = synth
    spec.loader.exec_module(synth)

    t0 = time.time()
    out = {}

    # ---- primes -------------------------------------------------------------
    out["primes_512"] = [int(p) for p in ref.generate_rns_primes(512)]
    out["primes_prefix_ok"] = all(
        [int(p) for p in ref.generate_rns_primes(k)] == out["primes_512"][:k]
        for k in (1, 8, 16, 32, 64, 128))

    # ---- compiler -------------------------------------------------------------
    comp_cases = []
    pcf_pairs = [("2", "n**2"), ("3*n**2-2*n+5", "n**4-3"), ("1", "(n**2+1)/(2*n+3)"),
                 ("-n", "2*n**3 + 7*n**2 - n/2"), ("n**5 + 1", "(3*n**3-2*n+1)/(n**3+5)"),
                 ("7", "n**-2 + 1"), ("n + 1/3", "-n**3"), ("0", "n*(n+1)*(2*n-1)"),
                 ("2*n+1", "-(n**2)*(n+1)**2")]
    for spec_rng_seed in range(3):
        for w in synth.uniform_pcfs(4, seed=100 + spec_rng_seed, depth=10, limit_depth=10):
            pcf_pairs.append((w.a, w.b))
    for w in synth.rational_pcfs(6, seed=7):
        pcf_pairs.append((w.a, w.b))
    for a, b in pcf_pairs:
        prog = ref.compile_pcf(a, b)
        comp_cases.append({"kind": "pcf", "a": a, "b": b,
                           "blob": None if prog is None else _blob_hex(prog)})
    comp_cases.append({"kind": "pcf", "a": "I*n", "b": "1",
                       "blob": None if ref.compile_pcf("I*n", "1") is None else "?"})
    for (c0, c1, c2) in synth.cmf3_polys(3, seed=11):
        mat = synth.cmf3_matrix(c0, c1, c2)
        prog = ref.compile_cmf_from_dict(mat, m=3, dim=3, axis_names=["x", "y", "z"],
                                         directions=[1, 2, 3])
        comp_cases.append({"kind": "dict", "matrix": [[r, c, e] for (r, c), e in mat.items()],
                           "m": 3, "dim": 3, "axis_names": ["x", "y", "z"],
                           "directions": [1, 2, 3], "blob": _blob_hex(prog)})
    dense = {(0, 0): "x + 1", (0, 1): "y * 2", (1, 0): "1", (1, 1): "x * y - n",
             (0, 0 + 1): "y*2"}
    prog = ref.compile_cmf_from_dict(dense, m=2, dim=2, axis_names=["x", "y"])
    comp_cases.append({"kind": "dict", "matrix": [[r, c, e] for (r, c), e in dense.items()],
                       "m": 2, "dim": 2, "axis_names": ["x", "y"], "directions": None,
                       "blob": _blob_hex(prog)})
    specs = [
        ({"p": 2, "q": 1, "a_params": ["1/2", "1"], "b_params": ["3/2"]}, [1, 1, 2]),
        ({"p": 3, "q": 2, "a_params": ["1", "1", "1"], "b_params": ["2", "2"]}, [1, 1, 1, 1, 1]),
        ({"p": 1, "q": 1, "a_params": ["1/3"], "b_params": ["2/3"]}, [2, 1]),
    ]
    for spec, traj in specs:
        prog = ref_cmf.compile_cmf_spec(spec, traj)
        comp_cases.append({"kind": "spec", "spec": spec, "trajectory": traj,
                           "blob": _blob_hex(prog)})
    err_cases = []
    for a, b in [("x", "n"), ("sqrt(n)", "1"), ("n**(1/2)", "1"), ("1.5*n", "1")]:
        try:
            ref.compile_pcf(a, b)
            err_cases.append({"a": a, "b": b, "error": None})
        except Exception as e:  # noqa: BLE001 - record the exception type
            err_cases.append({"a": a, "b": b, "error": type(e).__name__})
    out["compiler"] = comp_cases
    out["compiler_errors"] = err_cases

    # ---- PCF walks ----------------------------------------------------------
    def pcf_case(a, b, depth, K, shift=1, name=""):
        prog = ref.compile_pcf(a, b)
        a0 = ref.pcf_initial_values(a)
        r = ref.run_pcf_walk(prog, a0, depth, K, shift)
        return {"name": name, "a": a, "b": b, "a0": int(a0), "depth": depth, "K": K,
                "shift": shift, "blob": _blob_hex(prog),
                "p_residues": [int(v) for v in r["p_residues"]],
                "q_residues": [int(v) for v in r["q_residues"]],
                "p_float": _fhex(r["p_float"]), "q_float": _fhex(r["q_float"]),
                "log_scale": _fhex(r["log_scale"])}

    walks = [pcf_case("2", "n**2", 2000, 32, name="config1")]
    walks += [pcf_case("2", "n**2", d, 32, name=f"depth{d}") for d in (0, 1, 2, 3)]
    walks.append(pcf_case("3*n**2-2*n+5", "n**4-3", 300, 16, shift=-7, name="negshift"))
    walks.append(pcf_case("1", "(n**2+1)/(2*n+3)", 400, 64, name="rational"))
    walks.append(pcf_case("1", "(n**2+1)/(n-3)", 50, 32, name="int_root_inv0"))
    # n + 2147483642 == 2^31-1 at n = 5: INV(0) for the first prime only
    walks.append(pcf_case("n", "1/(n + 2147483642)", 40, 8, name="inv0_one_prime"))
    walks.append(pcf_case("n+1", "2/(2147483647) + n", 20, 4, name="const_inv0"))
    walks.append(pcf_case("n + 1/3", "n**2/2 + 1", 200, 32, name="rational_consts"))
    walks.append(pcf_case("-n", "2*n**3 + 7*n**2 - n/2", 250, 128, name="k128"))
    walks.append(pcf_case("2*n+1", "-(n**2)*(n+1)**2", 500, 32, name="pi_like"))
    for w in synth.uniform_pcfs(6, seed=21, depth=300, limit_depth=300):
        walks.append(pcf_case(w.a, w.b, 300, 32, name="uniform"))
    for w in synth.rational_pcfs(4, seed=22, depth_range=(200, 400)):
        walks.append(pcf_case(w.a, w.b, w.depth, w.K, name="rational_synth"))
    out["pcf_walks"] = walks
    print(f"pcf walks done {time.time() - t0:.1f}s", flush=True)

    # ---- CMF walks ----------------------------------------------------------
    def cmf_case(mat, m, dim, names, depth, K, shifts, traj, name="", directions=None):
        prog = ref.compile_cmf_from_dict(mat, m=m, dim=dim, axis_names=names,
                                         directions=directions)
        r = ref_cmf.run_cmf_walk(prog, depth, K, shifts, traj)
        enc = lambda vs: None if vs is None else [  # noqa: E731
            [v.numerator, v.denominator] if isinstance(v, Fraction) else
            (list(v) if isinstance(v, tuple) else [int(v), 1]) for v in vs]
        return {"name": name, "matrix": [[rr, cc, e] for (rr, cc), e in mat.items()],
                "m": m, "dim": dim, "axis_names": names, "directions": directions,
                "depth": depth, "K": K, "shifts": enc(shifts), "trajectory": enc(traj),
                "blob": _blob_hex(prog),
                "p_residues": [int(v) for v in r["p_residues"]],
                "q_residues": [int(v) for v in r["q_residues"]],
                "p_float": _fhex(r["p_float"]), "q_float": _fhex(r["q_float"]),
                "log_scale": _fhex(r["log_scale"])}

    cmfs = []
    polys = synth.cmf3_polys(4, seed=31)
    cmfs.append(cmf_case(synth.cmf3_matrix(*polys[0]), 3, 3, ["x", "y", "z"], 5000, 64,
                         [1, -2, 3], [1, 2, 3], name="config4_full"))
    for i, (s, d) in enumerate([([0, 0, 0], [1, 0, 0]), ([-3, 3, -1], [3, 3, 3]),
                                ([2, -3, 0], [0, 1, 2])]):
        cmfs.append(cmf_case(synth.cmf3_matrix(*polys[1 + i]), 3, 3, ["x", "y", "z"], 300,
                             64, s, d, name="cmf3"))
    cmfs.append(cmf_case(synth.cmf3_matrix(*polys[1]), 3, 3, ["x", "y", "z"], 200, 16,
                         [Fraction(1, 2), (2, 3), 1], [(1, 1), Fraction(3, 2), (2, 5)],
                         name="rational_shift"))
    cmfs.append(cmf_case(synth.cmf3_matrix(*polys[2]), 3, 3, ["x", "y", "z"], 150, 32,
                         [1, 1, 1], None, name="default_traj", directions=[2, 1, 3]))
    cmfs.append(cmf_case({(0, 0): "x + 1", (0, 1): "y * 2", (1, 0): "1",
                          (1, 1): "x * y - n"}, 2, 2, ["x", "y"], 300, 32, [1, 2], [1, 1],
                         name="dense2_loadn"))
    cmfs.append(cmf_case({(0, 0): "x", (0, 1): "1/(x+y)", (0, 2): "2",
                          (1, 0): "y**2", (1, 1): "0", (1, 2): "x - y",
                          (2, 0): "1", (2, 1): "x*y", (2, 2): "3*x + n"}, 3, 2, ["x", "y"],
                         200, 32, [1, 2], [1, 3], name="dense3_inv"))
    # pFq per-axis companion (m = 4) through the reference spec compiler
    spec = {"p": 3, "q": 2, "a_params": ["1", "1", "1"], "b_params": ["2", "2"]}
    prog = ref_cmf.compile_cmf_spec(spec, [1, 1, 1, 1, 1])
    r = ref_cmf.run_cmf_walk(prog, 300, 32, [1, 1, 1, 1, 1], [1, 1, 1, 1, 1])
    cmfs.append({"name": "pfq_3f2", "spec": spec, "spec_trajectory": [1, 1, 1, 1, 1],
                 "m": 4, "dim": 5, "depth": 300, "K": 32, "shifts": [[1, 1]] * 5,
                 "trajectory": [[1, 1]] * 5, "blob": _blob_hex(prog),
                 "p_residues": [int(v) for v in r["p_residues"]],
                 "q_residues": [int(v) for v in r["q_residues"]],
                 "p_float": _fhex(r["p_float"]), "q_float": _fhex(r["q_float"]),
                 "log_scale": _fhex(r["log_scale"])})
    out["cmf_walks"] = cmfs
    print(f"cmf walks done {time.time() - t0:.1f}s", flush=True)

    # ---- state-vector (matvec) walk ----------------------------------------
    vec = []
    spec = {"p": 2, "q": 1, "a_params": ["1/2", "1"], "b_params": ["3/2"]}
    prog = ref_cmf.compile_cmf_spec(spec, [1, 1, 1])
    init = [Fraction(1), Fraction(0), Fraction(1, 3)]
    r = ref_cmf.run_cmf_walk_vec(prog, 300, 32, [Fraction(1, 2), 1, (3, 2)], init, 0, 2,
                                 [1, (1, 2), 1])
    vec.append({"name": "vec_2f1", "blob": _blob_hex(prog), "depth": 300, "K": 32,
                "shifts": [[1, 2], [1, 1], [3, 2]], "trajectory": [[1, 1], [1, 2], [1, 1]],
                "initial_state": [[f.numerator, f.denominator] for f in init],
                "acc_idx": 0, "const_idx": 2,
                "p_residues": [int(v) for v in r["p_residues"]],
                "q_residues": [int(v) for v in r["q_residues"]],
                "p_float": _fhex(r["p_float"]), "q_float": _fhex(r["q_float"]),
                "log_scale": _fhex(r["log_scale"])})
    out["vec_walks"] = vec

    # ---- CRT / centered -------------------------------------------------------
    rng = np.random.default_rng(41)
    primes512 = out["primes_512"]
    crt_cases = []
    for K in (1, 2, 8, 32, 128, 512):
        for _ in range(3):
            res = [int(rng.integers(0, p)) for p in primes512[:K]]
            x, M = ref.crt_reconstruct(res, primes512[:K])
            crt_cases.append({"residues": res, "primes": primes512[:K], "x": hex(x),
                              "M": hex(M), "centered": hex(ref.centered(x, M))})
    cpp_primes = [2147483647, 2147483629, 2147483587, 2147483579, 2147483549, 2147483543,
                  2147483497, 2147483489]
    for v in (0, 1, 12345, 1000000007, 1 << 32, 1 << 40, 1 << 50, -12345, -(1 << 200)):
        res = [v % p for p in cpp_primes]
        x, M = ref.crt_reconstruct(res, cpp_primes)
        crt_cases.append({"residues": res, "primes": cpp_primes, "x": hex(x), "M": hex(M),
                          "centered": hex(ref.centered(x, M)), "value": hex(v)})
    out["crt"] = crt_cases

    # ---- deltas ---------------------------------------------------------------
    delta_cases = []
    cfg1 = walks[0]
    P = [int(v) for v in cfg1["p_residues"]]
    Q = [int(v) for v in cfg1["q_residues"]]
    pr = primes512[:32]
    pb, Mb = ref.crt_reconstruct(P, pr)
    qb, _ = ref.crt_reconstruct(Q, pr)
    pb, qb = ref.centered(pb, Mb), ref.centered(qb, Mb)
    mp.mp.dps = 200
    tgt = mp.mpf(2) / (4 - mp.pi)
    def add_delta(p, q, target_str, dps, name):
        d = ref.compute_dreams_delta_exact(p, q, mp.mpf(target_str) if dps else target_str, dps)
        delta_cases.append({"name": name, "p": hex(p), "q": hex(q), "target": target_str,
                            "dps": dps, "delta": repr(float(d))})
    add_delta(pb, qb, str(tgt), 200, "config1")
    for i in range(40):
        bits = int(rng.integers(2, 1000))
        p = int.from_bytes(rng.bytes(bits // 8 + 1), "little") >> (8 - bits % 8)
        q = int.from_bytes(rng.bytes(bits // 8 + 1), "little") >> (8 - bits % 8)
        if rng.integers(0, 2):
            p = -p
        if rng.integers(0, 2):
            q = -q
        t = str(mp.mpf(int(rng.integers(-50, 50))) / 7 + mp.pi * int(rng.integers(0, 3)))
        add_delta(p, q, t, 200, "random")
    add_delta(5, 0, "1.5", 200, "q_zero")
    add_delta(7, 1, "1.5", 200, "q_one")
    add_delta(7, -1, "1.5", 200, "q_minus_one")
    add_delta(3, 4, "0.75", 200, "exact")
    add_delta(3 * (10 ** 30) + 1, 4 * (10 ** 30), "0.75", 200, "close")
    add_delta(314159, 100000, str(mp.pi), 50, "dps50")
    out["delta_exact"] = delta_cases
    fl = []
    cfg1_shadow = (float.fromhex(cfg1["p_float"]), float.fromhex(cfg1["q_float"]),
                   float.fromhex(cfg1["log_scale"]), float(tgt))
    for (pf, qf, ls, t) in [(1.5, 2.0, 10.0, 0.7), (float("nan"), 1.0, 0.0, 1.0),
                            (1.0, 0.0, 0.0, 1.0), (1.0, 1e-301, 5.0, 1.0), (3.0, 4.0, 0.0, 0.75),
                            (3.0, 4.0, -5.0, 0.5), (2.0, 3.0, 100.0, 0.6), cfg1_shadow]:
        d, lq = ref.compute_dreams_delta_float(pf, qf, ls, t)
        fl.append({"args": [repr(pf), repr(qf), repr(ls), repr(t)],
                   "delta": repr(float(d)), "log_q": repr(float(lq))})
    out["delta_float"] = fl

    # ---- verify_pcf -----------------------------------------------------------
    ver = []
    for a, b, lim, depth, K in [("2", "n**2", "2/(4 - pi)", 2000, 32),
                                ("1", "n**2", "4/pi", 300, 16),
                                ("3", "-2*n**2 + n", "E", 100, 64),
                                ("2*n+1", "-(n**2)*(n+1)**2", "pi/4", 200, 32)]:
        r = ref.verify_pcf(a, b, lim, depth, K)
        ver.append({"a": a, "b": b, "limit": lim, "depth": depth, "K": K,
                    "result": {k: (repr(v) if isinstance(v, float) else v)
                               for k, v in r.items()}})
    out["verify_pcf"] = ver
    out["generated_by"] = "tests/golden/make_golden.py"
    out["reference_versions"] = {"numpy": np.__version__, "mpmath": mp.__version__,
                                 "sympy": __import__("sympy").__version__}
    with open(os.path.join(HERE, "reference_golden.json"), "w") as f:
        json.dump(out, f, indent=0, sort_keys=True)
    print(f"done {time.time() - t0:.1f}s")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <reference checkout>/python")
    main(sys.argv[1])
