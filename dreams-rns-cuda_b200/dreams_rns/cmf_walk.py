"""Drop-in CMF walk API on the B200 engine (reference python/dreams_rns/cmf_walk.py).

r x r walks with per-axis rational shift and trajectory: at 0-based step t
axis i takes shift[i] + t * trajectory[i]; P(N) = M(0) ... M(N-1) from
P = I; p = P[0, r-1], q = P[r-1, r-1] (cmf_walk.py:1-17).
"""

from __future__ import annotations

import itertools
from fractions import Fraction
from typing import Dict, List, Optional, Tuple

import numpy as np

from .compiler import CmfCompiler, CmfProgram, Opcode
from .engine import cmf_request, run_walks, vec_request
from .runner import centered, crt_reconstruct, generate_rns_primes

__all__ = ["compile_cmf_spec", "shift_to_axis_offsets", "run_cmf_walk", "run_cmf_walk_vec"]


def _build_per_axis_companion(p: int, q: int, a_params: List[Fraction],
                              b_params: List[Fraction]) -> Tuple[int, Dict[str, str], List[str]]:
    """Rank-r companion of a pFq CMF with one axis per parameter
    (cmf_walk.py:34-99): r = max(p, q) + 1, ones on the sub-diagonal, the last
    column holds prod(x_i + a_i), e_k(b-factors) - e_k(a-factors) for the
    middle rows and prod(y_j + b_j) in the last row (r == 2: the two
    products)."""
    r = max(p, q) + 1
    names = [f"x{i}" for i in range(p)] + [f"y{j}" for j in range(q)]
    a_f = [f"({names[i]} + {a_params[i]})" for i in range(p)]
    b_f = [f"({names[p + j]} + {b_params[j]})" for j in range(q)]
    mat = {f"{i},{j}": ("1" if i == j + 1 else "0") for i in range(r) for j in range(r)}
    prod = lambda fs: " * ".join(fs) if fs else "1"  # noqa: E731
    mat[f"0,{r - 1}"] = prod(a_f)
    if r == 2:
        mat[f"1,{r - 1}"] = prod(b_f)
    else:
        for row in range(1, r - 1):
            k = r - 1 - row
            def ek(fs):
                terms = [" * ".join(c) for c in itertools.combinations(fs, k)] if k <= len(fs) else []
                return " + ".join(terms) if terms else "0"
            mat[f"{row},{r - 1}"] = f"({ek(b_f)}) - ({ek(a_f)})"
        mat[f"{r - 1},{r - 1}"] = prod(b_f)
    return r, mat, names


def compile_cmf_spec(spec: Dict, trajectory: Optional[List[int]] = None) -> Optional[CmfProgram]:
    """pFq spec -> rank-r bytecode with per-axis variables (cmf_walk.py:104-152).
    Entries are compiled row-major; "0" entries are skipped."""
    import sympy as sp

    p, q = spec["p"], spec["q"]
    a_params = [Fraction(x) for x in spec["a_params"]]
    b_params = [Fraction(x) for x in spec["b_params"]]
    rank, mat, names = _build_per_axis_companion(p, q, a_params, b_params)
    dim = p + q
    if trajectory is None:
        trajectory = [1] * dim
    assert len(trajectory) == dim, f"trajectory len {len(trajectory)} != dim {dim}"
    comp = CmfCompiler(m=rank, dim=dim, directions=list(trajectory))
    axes = {name: i for i, name in enumerate(names)}
    local = {name: sp.Symbol(name) for name in names}
    for i in range(rank):
        for j in range(rank):
            text = mat[f"{i},{j}"]
            if text == "0":
                continue
            expr = sp.Integer(1) if text == "1" else sp.sympify(text, locals=local)
            if expr.has(sp.I):
                return None
            comp.compile_matrix_entry(i, j, expr, axes)
    return comp.build()


def shift_to_axis_offsets(shift: Dict, p: int) -> List[int]:
    """max(1, 1 + nums[i]) per axis (cmf_walk.py:157-169)."""
    return [max(1, 1 + n) for n in shift.get("nums", [])]


def _ref_dict(r: dict) -> dict:
    return {"p_residues": r["p_residues"], "q_residues": r["q_residues"],
            "p_float": np.float64(r["p_float"]), "q_float": np.float64(r["q_float"]),
            "log_scale": float(r["log_scale"]), "primes": r["primes"]}


def run_cmf_walk(program: CmfProgram, depth: int, K: int, shift_vals, trajectory_vals=None):
    """r x r walk on the GPU (reference cmf_walk.py:363-431)."""
    req = cmf_request(program, max(int(depth), 0), int(K), shift_vals, trajectory_vals)
    return _ref_dict(run_walks([req])[0])


def run_cmf_walk_vec(program: CmfProgram, depth: int, K: int, shift_vals, initial_state,
                     acc_idx: int, const_idx: int, trajectory_vals=None):
    """State-vector walk v(N) = M(N-1) ... M(0) v(0) on the GPU (reference
    cmf_walk.py:445-531): p = v[acc_idx], q = v[const_idx], with the FP64
    shadow of v rescaled like the reference's."""
    req = vec_request(program, max(int(depth), 0), int(K), shift_vals, initial_state, acc_idx,
                      const_idx, trajectory_vals)
    return _ref_dict(run_walks([req])[0])
