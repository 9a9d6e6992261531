"""Drop-in PCF walk API on the B200 engine.

Same names, arguments, return values and exceptions as the reference module
python/dreams_rns/runner.py; the walk, the CRT and the exact delta run on the
GPU through the C ABI (``_native``).  Conventions (runner.py:4-9):

    M(n) = [[0, b(n)], [1, a(n)]],   P(N) = A * M(1) * ... * M(N),
    A = [[1, a(0)], [0, 1]],  p = P[0, m-1],  q = P[1, m-1],
    delta = -(1 + log|p/q - L| / log|q|)
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _native as N
from .compiler import CmfCompiler, CmfProgram, Opcode
from .compiler import compile_pcf as _compile_pcf
from .engine import pcf_request, run_walks

__all__ = [
    "WalkConfig", "generate_rns_primes", "crt_reconstruct", "centered", "crt_batch",
    "compute_dreams_delta_float", "compute_dreams_delta_exact", "delta_batch",
    "compile_pcf", "pcf_initial_values", "run_pcf_walk", "verify_pcf", "target_ratio",
]


@dataclass
class WalkConfig:
    """Walk configuration (reference runner.py:23-28)."""

    K: int = 32
    depth: int = 2000
    delta_threshold: float = -2.0


def generate_rns_primes(K: int) -> np.ndarray:
    """The K largest primes below 2^31, descending (reference runner.py:33-52)."""
    if K <= 0:
        return np.zeros(0, dtype=np.int64)
    if K > N.DR_MAX_K:
        raise ValueError(f"K above {N.DR_MAX_K}")
    return N.prime_table(int(K)).astype(np.int64)


# ---- big integers as limbs ---------------------------------------------------

def int_to_limbs(x: int, stride: int) -> Tuple[int, np.ndarray]:
    """Sign and little-endian u32 magnitude limbs of a Python int."""
    sign = (x > 0) - (x < 0)
    mag = abs(x)
    nbytes = 4 * stride
    if mag.bit_length() > 8 * nbytes:
        raise OverflowError("integer wider than the limb stride")
    return sign, np.frombuffer(mag.to_bytes(nbytes, "little"), dtype=np.uint32).copy()


def limbs_to_int(limbs: np.ndarray, sign: int = 1) -> int:
    mag = int.from_bytes(np.ascontiguousarray(limbs, dtype=np.uint32).tobytes(), "little")
    return -mag if sign < 0 else mag


def _limbs_for(K: int) -> int:
    return (31 * K + 31) // 32 + 2


# ---- CRT ---------------------------------------------------------------------

def crt_batch(residues: np.ndarray, K: int, moduli: Optional[Sequence[int]] = None,
              unsigned: bool = False):
    """GPU Garner CRT of an (n, K) residue array.

    Returns the centred values ``x - M if x > M // 2 else x`` as Python ints
    (and the unsigned reference values ``x`` when ``unsigned``).
    """
    N.init()
    res = np.ascontiguousarray(residues, dtype=np.uint32).reshape(-1, K)
    n = res.shape[0]
    stride = _limbs_for(K)
    limbs = np.zeros((n, stride), dtype=np.uint32)
    ul = np.zeros((n, stride), dtype=np.uint32) if unsigned else None
    sign = np.zeros(n, dtype=np.int32)
    nl = np.zeros(n, dtype=np.int32)
    mod = None
    if moduli is not None:
        mod = np.ascontiguousarray(moduli, dtype=np.uint32)
        if np.array_equal(mod, N.prime_table(K)):
            mod = None
    N.check(N.lib().dr_crt_batch(N.ptr(res), K, n, N.ptr(mod) if mod is not None else None,
                                 N.ptr(limbs), stride, N.ptr(sign), N.ptr(nl),
                                 N.ptr(ul) if ul is not None else None), "dr_crt_batch")
    cen = [limbs_to_int(limbs[i], int(sign[i])) for i in range(n)]
    if unsigned:
        return cen, [limbs_to_int(ul[i]) for i in range(n)]
    return cen


def crt_reconstruct(residues, primes):
    """(x, M): x = sum of mixed-radix digits, M = prod(primes) (runner.py:57-76).

    Moduli must be odd and in [3, 2^31); the first residue is used as given
    (as the reference does) and must lie in [0, 2^32).
    """
    K = len(residues)
    if K == 0:
        raise IndexError("crt_reconstruct of an empty residue list")
    pr = [int(p) for p in list(primes)[:K]]
    if len(pr) < K:
        raise IndexError("fewer primes than residues")
    res = [int(r) for r in residues]
    if not 0 <= res[0] < (1 << 32):
        raise ValueError("first residue must be in [0, 2^32) for the GPU CRT")
    for i in range(1, K):
        if not 0 <= res[i] < (1 << 32):
            res[i] %= pr[i]   # only a_i mod p_i enters the reference formula
    for p in pr:
        if not (3 <= p < (1 << 31) and p % 2 == 1):
            raise ValueError(f"modulus {p} outside odd [3, 2^31)")
    _, (x,) = crt_batch(np.array([res], dtype=np.uint64).astype(np.uint32), K, pr, unsigned=True)
    return x, math.prod(pr)


def centered(x, M):
    """runner.py:79-81."""
    return x - M if x > M // 2 else x


# ---- delta ------------------------------------------------------------------

def compute_dreams_delta_float(p_val: float, q_val: float, log_scale: float,
                               target: float) -> Tuple[float, float]:
    """Approximate delta from the float shadow (runner.py:86-100)."""
    if not math.isfinite(p_val) or not math.isfinite(q_val) or abs(q_val) < 1e-300:
        return -1e10, 0.0
    est = p_val / q_val
    abs_err = abs(est - target)
    log_abs_q = log_scale + math.log(abs(q_val))
    if abs_err < 1e-300 or log_abs_q <= 0.0:
        return (100.0 if abs_err < 1e-300 else -1e10), log_abs_q
    return -(1.0 + math.log(abs_err) / log_abs_q), log_abs_q


def target_ratio(target) -> Tuple[int, int]:
    """Exact (numerator, denominator) of mpf(str(target)) at the current mpmath
    precision: the value compute_dreams_delta_exact compares against."""
    import mpmath as mp
    v = mp.mpf(str(target))
    if not mp.isfinite(v):
        raise OverflowError("non-finite target")
    sign, man, exp, _ = v._mpf_
    man = int(man)
    num = -man if sign else man
    if exp >= 0:
        return num << exp, 1
    return num, 1 << (-exp)


def delta_batch(ps: Sequence[int], qs: Sequence[int], targets: Sequence[Tuple[int, int]]) -> List[float]:
    """GPU exact delta for many (p, q); ``targets`` holds one (Lnum, Lden) or
    one per item."""
    N.init()
    n = len(ps)
    if n == 0:
        return []
    width = max(max(abs(int(v)).bit_length() for v in list(ps) + list(qs)), 1)
    stride = (width + 31) // 32 + 1
    lw = max(max(abs(a).bit_length(), abs(b).bit_length()) for a, b in targets)
    lstride = (lw + 31) // 32 + 1
    P = np.zeros((n, stride), dtype=np.uint32)
    Q = np.zeros((n, stride), dtype=np.uint32)
    Ps = np.zeros(n, dtype=np.int32)
    Qs = np.zeros(n, dtype=np.int32)
    for i in range(n):
        Ps[i], P[i] = int_to_limbs(int(ps[i]), stride)
        Qs[i], Q[i] = int_to_limbs(int(qs[i]), stride)
    nt = len(targets)
    LN = np.zeros((nt, lstride), dtype=np.uint32)
    LD = np.zeros((nt, lstride), dtype=np.uint32)
    LS = np.zeros(nt, dtype=np.int32)
    for i, (a, b) in enumerate(targets):
        LS[i], LN[i] = int_to_limbs(int(a), lstride)
        _, LD[i] = int_to_limbs(int(b), lstride)
    out = np.zeros(n, dtype=np.float64)
    N.check(N.lib().dr_delta_batch(N.ptr(P), N.ptr(Ps), N.ptr(Q), N.ptr(Qs), n, stride, N.ptr(LN),
                                   N.ptr(LS), N.ptr(LD), lstride, 1 if nt > 1 else 0, N.ptr(out)),
            "dr_delta_batch")
    return [float(v) for v in out]


def estimate_K(a_str: str, b_str: str, depth: int, safety: float = 1.5) -> int:
    """Primes needed for an exact CRT of a depth-N PCF convergent
    (reference euler2ai_full_verify.py:40-93): bits ~ d*log2(N!) + N*log2(c)
    for entries of degree d and largest coefficient c, times ``safety`` plus
    100, at least 64 primes; 1000+ when the expressions do not parse."""
    import sympy as sp
    try:
        a_expr = sp.sympify(a_str)
        b_expr = sp.sympify(b_str)
        n = sp.Symbol("n")
        deg_a = sp.degree(a_expr, n) if a_expr.has(n) else 0
        deg_b = sp.degree(b_expr, n) if b_expr.has(n) else 0
        max_deg = max(int(deg_a), int(deg_b), 1)
        max_coeff = 1
        for expr in (a_expr, b_expr):
            try:
                for c in sp.Poly(expr, n).all_coeffs():
                    max_coeff = max(max_coeff, abs(int(c)))
            except Exception:  # noqa: BLE001 - non-polynomial entries, as the reference
                max_coeff = max(max_coeff, 100)
        if depth > 1:
            log2_fact = depth * math.log2(depth / math.e) + 0.5 * math.log2(2 * math.pi * depth)
        else:
            log2_fact = 1
        coeff_bits = math.log2(max_coeff + 1) if max_coeff > 1 else 0
        bits = int((max_deg * log2_fact + depth * coeff_bits) * safety) + 100
        return max(bits // 31 + 1, 64)
    except Exception:  # noqa: BLE001 - the reference's conservative fallback
        log2_fact = depth * math.log2(max(depth, 2) / math.e)
        return max(int(4 * log2_fact * safety / 31) + 1, 1000)


def crt_overflowed(p_big: int, q_big: int, est_float: float) -> bool:
    """CRT overflow test (reference euler2ai_full_verify.py:152-167): the
    exact p/q must agree with the float shadow's estimate to 1%.  The device
    pipeline sets DR_STATUS_CRT_OVERFLOW by the same rule."""
    import mpmath as mp
    if q_big == 0:
        return True
    try:
        crt_ratio = float(mp.mpf(p_big) / mp.mpf(q_big))
        if not math.isfinite(crt_ratio) or not math.isfinite(est_float):
            return True
        if abs(est_float) > 1e-10:
            return abs(crt_ratio - est_float) / abs(est_float) > 0.01
        return abs(crt_ratio - est_float) > 0.01
    except Exception:  # noqa: BLE001 - as the reference
        return True


def compute_dreams_delta_exact(p_big: int, q_big: int, target, dps: int = 200):
    """Exact delta from big integers (runner.py:103-125), computed on the GPU.

    Like the reference it sets the process-wide mpmath precision to ``dps``;
    the target is taken as mpf(str(target)) at that precision.
    """
    import mpmath as mp
    mp.mp.dps = dps
    if q_big == 0:
        return float("-inf")
    try:
        num, den = target_ratio(target)
    except OverflowError:
        # err = |approx - L| is inf (L infinite) or nan (L nan); runner.py:120-125
        if abs(q_big) <= 1 or mp.isinf(mp.mpf(str(target))):
            return float("-inf")
        return float("nan")
    return delta_batch([int(p_big)], [int(q_big)], [(num, den)])[0]


# ---- PCF compilation ----------------------------------------------------------

def compile_pcf(a_str: str, b_str: str) -> Optional[CmfProgram]:
    """Companion bytecode of PCF(a, b) (runner.py:130-166): n is axis 0 with
    direction 1, entries (0,1)=b, (1,0)=1, (1,1)=a; None for imaginary input."""
    return _compile_pcf(a_str, b_str)


def pcf_initial_values(a_str: str):
    """a(0) as an int (runner.py:169-177)."""
    import sympy as sp
    from sympy.abc import n
    return int(sp.sympify(a_str).subs(n, 0))


# ---- walk ------------------------------------------------------------------

def _as_reference_dict(r: dict) -> dict:
    return {"p_residues": r["p_residues"], "q_residues": r["q_residues"],
            "p_float": np.float64(r["p_float"]), "q_float": np.float64(r["q_float"]),
            "log_scale": float(r["log_scale"]), "primes": r["primes"]}


def run_pcf_walk(program: CmfProgram, a0: int, depth: int, K: int = 32, shift_val: int = 1):
    """P = A * M(1) ... M(depth) on the GPU (reference runner.py:338-413).

    Returns p_residues, q_residues (int64 (K,)), p_float, q_float, log_scale
    (FP64 shadow) and primes, exactly like the reference.
    """
    assert program.m == 2, "run_pcf_walk only supports 2×2 companion matrices"
    if K <= 0:
        e = np.zeros(0, dtype=np.int64)
        P_f = np.array([[1.0, float(a0)], [0.0, 1.0]])
        return {"p_residues": e, "q_residues": e.copy(), "p_float": P_f[0, 1],
                "q_float": P_f[1, 1], "log_scale": 0.0, "primes": e.copy()}
    req = pcf_request(program, a0, max(int(depth), 0), int(K), int(shift_val))
    return _as_reference_dict(run_walks([req])[0])


def verify_pcf(a_str: str, b_str: str, limit_str: str, depth: int = 2000, K: int = 32,
               dps: int = 200):
    """compile -> walk -> CRT -> delta (reference runner.py:416-476)."""
    import sympy as sp
    import mpmath as mp
    mp.mp.dps = dps
    program = compile_pcf(a_str, b_str)
    if program is None:
        return None
    a0 = pcf_initial_values(a_str)
    res = run_pcf_walk(program, a0, depth, K)
    target_expr = sp.sympify(limit_str, locals={"pi": sp.pi, "E": sp.E})
    target_mp = mp.mpf(str(sp.N(target_expr, dps)))
    delta_float, log_q = compute_dreams_delta_float(res["p_float"], res["q_float"],
                                                    res["log_scale"], float(target_mp))
    pr = [int(p) for p in res["primes"]]
    K_eff = len(pr)
    (p_big, q_big) = crt_batch(np.stack([res["p_residues"], res["q_residues"]]).astype(np.uint32),
                               K_eff)
    Mp = math.prod(pr)
    delta_exact = compute_dreams_delta_exact(p_big, q_big, target_mp, dps)
    est_float = res["p_float"] / res["q_float"] if abs(res["q_float"]) > 1e-300 else float("nan")
    return {"a": a_str, "b": b_str, "limit": limit_str, "target": float(target_mp),
            "est_float": est_float, "delta_float": delta_float, "delta_exact": delta_exact,
            "log_q": log_q, "depth": depth, "K": K, "p_bits": Mp.bit_length()}
