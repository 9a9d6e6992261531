"""Seeded random bytecode programs for parity sweeps.

Straight-line programs over a small register window (so registers are
reused, read before written, overwritten), random STOREs, INV in arbitrary
places, NOPs and dead code after END.  Half of them have the companion
shape so every execution class of the engine is exercised.
"""

from __future__ import annotations

import random
import struct
from typing import List, Tuple

CONST_POOL = [0, 1, -1, 2, 3, -5, 7, 2147483647, 2147483629 * 3, -(1 << 40), 12, -9]


def blob_of(m: int, dim: int, ops, consts, dirs) -> bytes:
    b = struct.pack("<IIII", m, dim, len(ops), len(consts))
    for o in ops:
        b += struct.pack("<IIII", *o)
    for c in consts:
        b += struct.pack("<q", c)
    for d in dirs:
        b += struct.pack("<i", d)
    return b


def _expr(rng, ops, nreg, dim, nconst, depth, allow_inv):
    r = rng.randrange(nreg)
    if depth == 0 or rng.random() < 0.3:
        k = rng.random()
        if k < 0.4:
            ops.append((1, rng.randrange(dim), r, 0))
        elif k < 0.8:
            ops.append((2, rng.randrange(nconst), r, 0))
        elif k < 0.9:
            ops.append((3, r, 0, 0))
        return r
    if rng.random() < 0.45:
        a = _expr(rng, ops, nreg, dim, nconst, depth - 1, allow_inv)
        b = _expr(rng, ops, nreg, dim, nconst, depth - 1, allow_inv)
        ops.append((rng.choice([4, 5, 6]), a, b, r))
        return r
    a = _expr(rng, ops, nreg, dim, nconst, depth - 1, allow_inv)
    ops.append((rng.choice([7, 8, 9, 10] if allow_inv else [7, 8, 9]), a, r, 0))
    return r


def random_program(rng: random.Random, m_choices=(2, 2, 3, 3, 4)) -> Tuple[bytes, int, int]:
    m = rng.choice(m_choices)
    dim = rng.choice([1, 2, 3])
    consts = [rng.choice(CONST_POOL + [rng.randrange(-100, 100)]) for _ in range(rng.randrange(1, 6))]
    if 1 not in consts:
        consts.append(1)
    ops: List[tuple] = []
    nreg = rng.choice([3, 8, 40])
    allow_inv = rng.random() < 0.5
    if rng.random() < 0.5:
        for i in range(m):
            r = _expr(rng, ops, nreg, dim, len(consts), rng.randrange(0, 4), allow_inv)
            ops.append((11, r, i, m - 1))
        one = consts.index(1)
        for j in range(m - 1):
            ops.append((2, one, 0, 0))
            ops.append((11, 0, j + 1, j))
    else:
        for _ in range(rng.randrange(1, 2 * m * m)):
            r = _expr(rng, ops, nreg, dim, len(consts), rng.randrange(0, 4), allow_inv)
            ops.append((11, r, rng.randrange(m), rng.randrange(m)))
    if rng.random() < 0.2:
        ops.insert(rng.randrange(len(ops) + 1), (0, 0, 0, 0))
    ops.append((12, 0, 0, 0))
    if rng.random() < 0.2:
        ops.append((6, 0, 0, 1))
    dirs = [rng.randrange(-3, 4) for _ in range(dim)]
    return blob_of(m, dim, ops, consts, dirs), m, dim


def random_axis(rng: random.Random, dim: int, rational: bool):
    out = []
    for _ in range(dim):
        sd = rng.choice([1, 2, 3]) if rational else 1
        td = rng.choice([1, 2, 5]) if rational else 1
        out += [rng.randrange(-5, 6), sd, rng.randrange(-3, 4), td]
    return out
