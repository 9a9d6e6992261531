"""numpy restatement of the reference walk path (test infrastructure only).

Each function below restates one reference function; the citation is on the
function.  Per walk step the program is interpreted once with every register
a length-K int64 vector (one entry per prime), exactly the reference's
evaluation order, so results are bit-identical and timing is representative
of the reference's own CPU implementation.
"""

from __future__ import annotations

import math
import struct
from fractions import Fraction
from functools import lru_cache
from typing import Dict, List, Sequence, Tuple

import numpy as np

# opcode numbers of the bytecode wire format (reference compiler.py:14-28)
NOP, LOAD_X, LOAD_C, LOAD_N, ADD, SUB, MUL, NEG, POW2, POW3, INV, STORE, END = range(13)


def parse_blob(blob: bytes):
    """Split a serialized program (reference compiler.py:53-89)."""
    m, dim, n_ops, n_consts = struct.unpack_from("<IIII", blob, 0)
    pos = 16
    ops = [struct.unpack_from("<IIII", blob, pos + 16 * i) for i in range(n_ops)]
    pos += 16 * n_ops
    consts = list(struct.unpack_from("<%dq" % n_consts, blob, pos))
    pos += 8 * n_consts
    dirs = list(struct.unpack_from("<%di" % dim, blob, pos))
    return m, dim, ops, consts, dirs


@lru_cache(maxsize=None)
def _prime_list(K: int) -> Tuple[int, ...]:
    """runner.py:33-52: the K largest primes below 2^31, by trial division."""
    out = []
    c = (1 << 31) - 1
    while len(out) < K and c >= (1 << 30):
        if c % 2 and all(c % d for d in range(3, math.isqrt(c) + 1, 2)):
            out.append(c)
        c -= 2
    return tuple(out)


def primes(K: int) -> np.ndarray:
    return np.array(_prime_list(K), dtype=np.int64)


def const_residues(consts: Sequence[int], pp: np.ndarray) -> np.ndarray:
    """runner.py:182-195: table[i, k] = consts[i] mod p_k in [0, p_k)."""
    table = np.zeros((len(consts), len(pp)), dtype=np.int64)
    for i, c in enumerate(consts):
        table[i] = [int(c) % int(p) for p in pp]
    return table


def _modinv_vec(vals: np.ndarray, pp: np.ndarray) -> np.ndarray:
    """runner.py:252-256: pow(v, p-2, p) per prime, so 0 maps to 0."""
    return np.array([pow(int(v), int(p) - 2, int(p)) for v, p in zip(vals, pp)],
                    dtype=np.int64)


def eval_modp(ops, m: int, step: int, axis_res, pp: np.ndarray, table: np.ndarray):
    """runner.py:198-260 and cmf_walk.py:193-258: one step matrix mod every prime.

    ``axis_res(axis, step)`` returns the (K,) residue vector of LOAD_X.
    Registers start at zero every step; unwritten matrix entries are zero.
    """
    K = len(pp)
    regs: Dict[int, np.ndarray] = {}
    zero = np.zeros(K, dtype=np.int64)
    M = np.zeros((m, m, K), dtype=np.int64)
    get = lambda r: regs.get(r, zero)  # noqa: E731
    for op, a0, a1, a2 in ops:
        if op == END:
            break
        if op == LOAD_X:
            regs[a1] = axis_res(a0, step)
        elif op == LOAD_C:
            regs[a1] = table[a0].copy()
        elif op == LOAD_N:
            regs[a0] = np.int64(step) % pp
        elif op == ADD:
            regs[a2] = (get(a0) + get(a1)) % pp
        elif op == SUB:
            regs[a2] = (get(a0) - get(a1)) % pp
        elif op == MUL:
            regs[a2] = (get(a0) * get(a1)) % pp
        elif op == NEG:
            regs[a1] = (pp - get(a0)) % pp
        elif op == POW2:
            regs[a1] = (get(a0) * get(a0)) % pp
        elif op == POW3:
            v = get(a0)
            regs[a1] = (v * v % pp * v) % pp
        elif op == INV:
            regs[a1] = _modinv_vec(get(a0), pp)
        elif op == STORE:
            M[a1, a2] = get(a0) % pp
    return M


def eval_float(ops, m: int, step: int, axis_val, consts) -> np.ndarray:
    """runner.py:263-316 / cmf_walk.py:261-313: the same program in float64."""
    regs: Dict[int, float] = {}
    M = np.zeros((m, m), dtype=np.float64)
    get = lambda r: regs.get(r, 0.0)  # noqa: E731
    for op, a0, a1, a2 in ops:
        if op == END:
            break
        if op == LOAD_X:
            regs[a1] = axis_val(a0, step)
        elif op == LOAD_C:
            regs[a1] = float(consts[a0])
        elif op == LOAD_N:
            regs[a0] = float(step)
        elif op == ADD:
            regs[a2] = get(a0) + get(a1)
        elif op == SUB:
            regs[a2] = get(a0) - get(a1)
        elif op == MUL:
            regs[a2] = get(a0) * get(a1)
        elif op == NEG:
            regs[a1] = -get(a0)
        elif op == POW2:
            regs[a1] = get(a0) ** 2
        elif op == POW3:
            regs[a1] = get(a0) ** 3
        elif op == INV:
            v = get(a0)
            regs[a1] = 1.0 / v if abs(v) > 1e-300 else 0.0
        elif op == STORE:
            M[a1, a2] = get(a0)
    return M


def matmul_mod(A: np.ndarray, B: np.ndarray, pp: np.ndarray) -> np.ndarray:
    """runner.py:321-333 and cmf_walk.py:174-188: (A @ B) mod p per prime."""
    r = A.shape[0]
    C = np.zeros_like(A)
    for i in range(r):
        for j in range(r):
            acc = np.zeros_like(pp)
            for k in range(r):
                acc = (acc + A[i, k] * B[k, j]) % pp
            C[i, j] = acc
    return C


def _shadow_step(P_f: np.ndarray, M_f: np.ndarray, log_scale: float):
    """runner.py:394-398: P_f <- P_f @ M_f, renormalised when max |P_f| > 1e10."""
    P_f = P_f @ M_f
    mx = np.max(np.abs(P_f))
    if mx > 1e10:
        P_f /= mx
        log_scale += math.log(mx)
    return P_f, log_scale


def _result(P, P_f, log_scale, pp, prow, qrow, col):
    return {"p_residues": P[prow, col].copy(), "q_residues": P[qrow, col].copy(),
            "p_float": P_f[prow, col], "q_float": P_f[qrow, col],
            "log_scale": log_scale, "primes": pp}


def pcf_walk(blob: bytes, a0: int, depth: int, K: int = 32, shift: int = 1,
             checkpoints: Sequence[int] = ()):
    """runner.py:338-413: P = A * M(1) ... M(depth), A = [[1, a0], [0, 1]].

    LOAD_X axis a at 0-based step s is shift + s * directions[a].  Returns the
    reference dict; with ``checkpoints`` also ``{"checkpoints": {d: dict}}``
    holding the same outputs after ``d`` steps.
    """
    m, dim, ops, consts, dirs = parse_blob(blob)
    assert m == 2, "run_pcf_walk only supports 2x2 companion matrices"
    pp = primes(K)
    table = const_residues(consts, pp)
    P = np.zeros((2, 2, K), dtype=np.int64)
    P[0, 0] = 1
    P[0, 1] = [int(a0) % int(p) for p in pp]
    P[1, 1] = 1
    P_f = np.array([[1.0, float(a0)], [0.0, 1.0]])
    log_scale = 0.0
    axis_res = lambda a, s: np.int64(shift + s * dirs[a]) % pp  # noqa: E731
    axis_val = lambda a, s: float(shift + s * dirs[a])  # noqa: E731
    cps = {}
    for s in range(depth):
        P = matmul_mod(P, eval_modp(ops, m, s, axis_res, pp, table), pp)
        P_f, log_scale = _shadow_step(P_f, eval_float(ops, m, s, axis_val, consts), log_scale)
        if s + 1 in checkpoints:
            cps[s + 1] = _result(P, P_f.copy(), log_scale, pp, 0, 1, m - 1)
    out = _result(P, P_f, log_scale, pp, 0, 1, m - 1)
    if checkpoints:
        out["checkpoints"] = cps
    return out


def _rationals(vals) -> Tuple[List[int], List[int]]:
    """cmf_walk.py:332-345: int, Fraction or (num, den) to numerators/denominators."""
    nums, dens = [], []
    for v in vals:
        if isinstance(v, Fraction):
            nums.append(v.numerator)
            dens.append(v.denominator)
        elif isinstance(v, (tuple, list)):
            nums.append(int(v[0]))
            dens.append(int(v[1]))
        else:
            nums.append(int(v))
            dens.append(1)
    return nums, dens


def _axis_fns(sn, sd, tn, td, pp):
    """cmf_walk.py:221-224, 278-281, 348-358: rational per-axis trajectory."""
    inv_cd = []
    for s, t in zip(sd, td):
        cd = s * t
        inv_cd.append(np.ones(len(pp), dtype=np.int64) if cd == 1 else
                      np.array([pow(cd, int(p) - 2, int(p)) for p in pp], dtype=np.int64))

    def axis_res(a, s):
        k = sn[a] * td[a] + s * tn[a] * sd[a]
        return (np.int64(k) % pp * inv_cd[a]) % pp

    def axis_val(a, s):
        k = sn[a] * td[a] + s * tn[a] * sd[a]
        return float(k) / float(sd[a] * td[a])

    return axis_res, axis_val


def cmf_walk(blob: bytes, depth: int, K: int, shift_vals, trajectory_vals=None,
             checkpoints: Sequence[int] = ()):
    """cmf_walk.py:363-431: P = M(0) ... M(depth-1) from P = I; q = P[m-1, m-1]."""
    m, dim, ops, consts, dirs = parse_blob(blob)
    pp = primes(K)
    table = const_residues(consts, pp)
    sn, sd = _rationals(shift_vals)
    if trajectory_vals is not None:
        tn, td = _rationals(trajectory_vals)
    else:
        tn, td = list(dirs), [1] * len(dirs)
    axis_res, axis_val = _axis_fns(sn, sd, tn, td, pp)
    P = np.zeros((m, m, K), dtype=np.int64)
    for i in range(m):
        P[i, i] = 1
    P_f = np.eye(m)
    log_scale = 0.0
    cps = {}
    for s in range(depth):
        P = matmul_mod(P, eval_modp(ops, m, s, axis_res, pp, table), pp)
        P_f, log_scale = _shadow_step(P_f, eval_float(ops, m, s, axis_val, consts), log_scale)
        if s + 1 in checkpoints:
            cps[s + 1] = _result(P, P_f.copy(), log_scale, pp, 0, m - 1, m - 1)
    out = _result(P, P_f, log_scale, pp, 0, m - 1, m - 1)
    if checkpoints:
        out["checkpoints"] = cps
    return out


def cmf_walk_vec(blob: bytes, depth: int, K: int, shift_vals, initial_state, acc_idx: int,
                 const_idx: int, trajectory_vals=None):
    """cmf_walk.py:445-531: v(N) = M(N-1) ... M(0) v(0), rational v(0)."""
    m, dim, ops, consts, dirs = parse_blob(blob)
    pp = primes(K)
    table = const_residues(consts, pp)
    sn, sd = _rationals(shift_vals)
    if trajectory_vals is not None:
        tn, td = _rationals(trajectory_vals)
    else:
        tn, td = list(dirs), [1] * len(dirs)
    axis_res, axis_val = _axis_fns(sn, sd, tn, td, pp)
    v = np.zeros((m, K), dtype=np.int64)
    for i, f in enumerate(initial_state):
        f = Fraction(f)
        if f == 0:
            continue
        for k, p in enumerate(int(q) for q in pp):
            num = f.numerator % p
            v[i, k] = num if f.denominator == 1 else num * pow(f.denominator, p - 2, p) % p
    v_f = np.array([float(Fraction(f)) for f in initial_state])
    log_scale = 0.0
    for s in range(depth):
        M = eval_modp(ops, m, s, axis_res, pp, table)
        w = np.zeros_like(v)
        for i in range(m):
            for j in range(m):
                w[i] = (w[i] + M[i, j] * v[j]) % pp
        v = w
        v_f = eval_float(ops, m, s, axis_val, consts) @ v_f
        mx = np.max(np.abs(v_f))
        if mx > 1e10:
            v_f /= mx
            log_scale += math.log(mx)
    return {"p_residues": v[acc_idx], "q_residues": v[const_idx], "p_float": v_f[acc_idx],
            "q_float": v_f[const_idx], "log_scale": log_scale, "primes": pp}


def crt(residues, primes_) -> Tuple[int, int]:
    """runner.py:57-76: iterative CRT, x in [0, M) for reduced residues."""
    x = int(residues[0])
    M = int(primes_[0])
    for a, p in zip(list(residues)[1:], list(primes_)[1:]):
        a, p = int(a), int(p)
        t = ((a - x % p) % p) * pow(M % p, p - 2, p) % p
        x += M * t
        M *= p
    return x, M


def centered(x: int, M: int) -> int:
    """runner.py:79-81."""
    return x - M if x > M // 2 else x


def delta_exact(p: int, q: int, target, dps: int = 200) -> float:
    """runner.py:103-125: -(1 + log|p/q - L| / log|q|) in mpmath at ``dps``."""
    import mpmath as mp
    mp.mp.dps = dps
    if q == 0:
        return float("-inf")
    err = abs(mp.mpf(p) / mp.mpf(q) - mp.mpf(str(target)))
    qq = abs(mp.mpf(q))
    if err == 0:
        return float("inf")
    if qq <= 1:
        return float("-inf")
    return float(-(1 + mp.log(err) / mp.log(qq)))


def delta_float(p_val: float, q_val: float, log_scale: float, target: float):
    """runner.py:86-100: approximate delta from the float shadow."""
    if not math.isfinite(p_val) or not math.isfinite(q_val) or abs(q_val) < 1e-300:
        return -1e10, 0.0
    abs_err = abs(p_val / q_val - target)
    log_abs_q = log_scale + math.log(abs(q_val))
    if abs_err < 1e-300 or log_abs_q <= 0.0:
        return (100.0 if abs_err < 1e-300 else -1e10), log_abs_q
    return -(1.0 + math.log(abs_err) / log_abs_q), log_abs_q
