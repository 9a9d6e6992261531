"""Seeded synthetic walk workloads with the shapes of the benchmark configs.

The reference measures on research datasets that are not shipped with it, so
these generators stand in for them.  Everything is drawn from
``numpy.random.default_rng(seed)`` and is fully reproducible.

* ``single_pcf``      a(n)=2, b(n)=n^2, depth 2000, K=32, L = 2/(4-pi)
* ``uniform_pcfs``    deg a <= 2, deg b <= 4, coefficients in [-10, 10] with a
                      non-zero leading coefficient; depth 2000, K=32, and the
                      delta target of each PCF is its own depth-8000 convergent
* ``rational_pcfs``   b = u/v with deg u, deg v <= 3 and coefficients in
                      [-8, 8], v(n) != 0 for n in [1, depth]; a of degree <= 2;
                      depth log-uniform in [200, 50000]; K in {16, 32, 64, 128};
                      bytecode length kept within [10, 200] ops
* ``cmf3_sweep``      3x3 companion [[0,0,c0],[1,0,c1],[0,1,c2]], c_i integer
                      polynomials in (x, y, z) of total degree <= 3 with
                      coefficients in [-6, 6]; shifts in [-3, 3]^3 and
                      directions in {0..3}^3 minus 0; depth 5000, K=64
* ``deep_pcf``        the deep serving walk: deg a = deg b = 1, coefficients
                      in [-5, 5], depth 10^6, K=512
"""

from __future__ import annotations

import itertools
import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

__all__ = [
    "poly_str",
    "WalkSpec",
    "single_pcf",
    "uniform_pcfs",
    "rational_pcfs",
    "cmf3_polys",
    "cmf3_sweep",
    "deep_pcf",
]


def poly_str(coeffs: Sequence[int], var: str = "n") -> str:
    """Render integer coefficients (constant term first) as a sympy string."""
    terms = []
    for k, c in enumerate(coeffs):
        c = int(c)
        if c == 0:
            continue
        if k == 0:
            terms.append(f"({c})")
        elif k == 1:
            terms.append(f"({c})*{var}")
        else:
            terms.append(f"({c})*{var}**{k}")
    return " + ".join(terms) if terms else "0"


def _rand_poly(rng, max_deg: int, lo: int, hi: int, min_deg: int = 0) -> List[int]:
    deg = int(rng.integers(min_deg, max_deg + 1))
    coeffs = [int(v) for v in rng.integers(lo, hi + 1, size=deg + 1)]
    while coeffs[-1] == 0:
        coeffs[-1] = int(rng.integers(lo, hi + 1))
    return coeffs


@dataclass
class WalkSpec:
    """One walk request in host form.

    ``kind`` is ``"pcf"`` (P0 = [[1, a0], [0, 1]], axis value
    shift + step * direction, q = P[1, m-1]) or ``"cmf"`` (P0 = I, rational
    per-axis shift and trajectory, q = P[m-1, m-1]).
    """

    kind: str
    depth: int
    K: int
    a: Optional[str] = None
    b: Optional[str] = None
    a0: int = 0
    shift: int = 1
    matrix: Optional[dict] = None          # cmf: {(row, col): expr}
    m: int = 2
    axis_names: Optional[List[str]] = None
    shifts: Optional[List[Tuple[int, int]]] = None       # cmf: (num, den) per axis
    trajectory: Optional[List[Tuple[int, int]]] = None   # cmf: (num, den) per axis
    program_key: Optional[str] = None
    checkpoint: int = 0
    tag: dict = field(default_factory=dict)


def single_pcf() -> WalkSpec:
    return WalkSpec(kind="pcf", depth=2000, K=32, a="2", b="n**2", a0=2,
                    tag={"limit": "2/(4 - pi)"})


def uniform_pcfs(count: int = 4096, seed: int = 2, depth: int = 2000, K: int = 32,
                 limit_depth: int = 8000) -> List[WalkSpec]:
    """Uniform PCF batch; each walk also yields its depth-``limit_depth`` convergent."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        ac = _rand_poly(rng, 2, -10, 10)
        bc = _rand_poly(rng, 4, -10, 10)
        out.append(WalkSpec(kind="pcf", depth=limit_depth, K=K, a=poly_str(ac),
                            b=poly_str(bc), a0=int(ac[0]), checkpoint=depth,
                            tag={"a_coeffs": ac, "b_coeffs": bc}))
    return out


def _has_int_root(coeffs: Sequence[int], depth: int) -> bool:
    """True when the integer polynomial vanishes at some n in [1, depth]."""
    cs = [int(c) for c in coeffs]
    while cs and cs[0] == 0:      # v(n) = n^k w(n) and n >= 1: only w's roots matter
        cs.pop(0)
    if not cs:
        return True
    c0 = cs[0]
    # a positive integer root of w divides its constant term
    for d in range(1, min(abs(c0), depth) + 1):
        if c0 % d == 0:
            v = 0
            for c in reversed(cs):
                v = v * d + c
            if v == 0:
                return True
    return False


def rational_pcfs(count: int = 8192, seed: int = 3, k_choices=(16, 32, 64, 128),
                  depth_range=(200, 50000), op_band=(10, 200),
                  compile_fn=None) -> List[WalkSpec]:
    """Uneven rational PCF batch (INV every step).

    ``compile_fn(a, b) -> n_ops`` is used to keep programs inside ``op_band``;
    without it no length filter is applied.
    """
    rng = np.random.default_rng(seed)
    lo_d, hi_d = depth_range
    out = []
    while len(out) < count:
        depth = int(round(math.exp(rng.uniform(math.log(lo_d), math.log(hi_d)))))
        K = int(rng.choice(np.asarray(k_choices)))
        uc = _rand_poly(rng, 3, -8, 8)
        vc = _rand_poly(rng, 3, -8, 8, min_deg=1)
        ac = _rand_poly(rng, 2, -8, 8)
        if _has_int_root(vc, depth):
            continue
        b = f"({poly_str(uc)})/({poly_str(vc)})"
        a = poly_str(ac)
        if compile_fn is not None:
            n_ops = compile_fn(a, b)
            if n_ops is None or not (op_band[0] <= n_ops <= op_band[1]):
                continue
        out.append(WalkSpec(kind="pcf", depth=depth, K=K, a=a, b=b, a0=int(ac[0]),
                            tag={"u": uc, "v": vc, "a_coeffs": ac}))
    return out


_MONOMIALS3 = [e for d in range(4) for e in itertools.product(range(d + 1), repeat=3)
               if sum(e) == d]


def _poly3_str(coeffs) -> str:
    terms = []
    for (ex, ey, ez), c in zip(_MONOMIALS3, coeffs):
        c = int(c)
        if c == 0:
            continue
        factors = [f"({c})"]
        for name, e in (("x", ex), ("y", ey), ("z", ez)):
            if e == 1:
                factors.append(name)
            elif e > 1:
                factors.append(f"{name}**{e}")
        terms.append("*".join(factors))
    return " + ".join(terms) if terms else "0"


def cmf3_polys(n_cmfs: int, seed: int) -> List[Tuple[str, str, str]]:
    """``n_cmfs`` triples (c0, c1, c2) of cubic trivariate polynomials."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_cmfs):
        triple = []
        for _ in range(3):
            coeffs = rng.integers(-6, 7, size=len(_MONOMIALS3))
            while not coeffs.any():
                coeffs = rng.integers(-6, 7, size=len(_MONOMIALS3))
            triple.append(_poly3_str(coeffs))
        out.append(tuple(triple))
    return out


def cmf3_matrix(c0: str, c1: str, c2: str) -> dict:
    return {(0, 2): c0, (1, 0): "1", (1, 2): c1, (2, 1): "1", (2, 2): c2}


def cmf3_sweep(count: int = 16384, n_cmfs: int = 64, seed: int = 4, depth: int = 5000,
               K: int = 64) -> List[WalkSpec]:
    """(shift, direction) sweep over ``n_cmfs`` seeded cubic 3x3 companion CMFs."""
    rng = np.random.default_rng(seed + 1000)
    polys = cmf3_polys(n_cmfs, seed)
    shifts = list(itertools.product(range(-3, 4), repeat=3))
    dirs = [d for d in itertools.product(range(4), repeat=3) if any(d)]
    pairs = [(s, d) for s in shifts for d in dirs]
    pick = rng.choice(len(pairs), size=count, replace=count > len(pairs))
    out = []
    for i, idx in enumerate(pick):
        s, d = pairs[int(idx)]
        g = i % n_cmfs
        c0, c1, c2 = polys[g]
        out.append(WalkSpec(kind="cmf", depth=depth, K=K, m=3,
                            matrix=cmf3_matrix(c0, c1, c2), axis_names=["x", "y", "z"],
                            shifts=[(int(v), 1) for v in s],
                            trajectory=[(int(v), 1) for v in d],
                            program_key=f"cmf3:{seed}:{g}", tag={"cmf": g}))
    return out


def deep_pcf(rng) -> WalkSpec:
    ac = _rand_poly(rng, 1, -5, 5, min_deg=1)
    bc = _rand_poly(rng, 1, -5, 5, min_deg=1)
    return WalkSpec(kind="pcf", depth=1_000_000, K=512, a=poly_str(ac), b=poly_str(bc),
                    a0=int(ac[0]), tag={"deep": True})
