"""Constant bank for limit matching (reference python/dreams_rns/constants.py).

The registry lists the same constants under the same names as the reference
(constants.py:21-67), so matches are reported with the reference's labels.
Values are evaluated with sympy/mpmath on the host (load_constants); the
delta of walk convergents against every constant runs on the GPU, after the
device top-k (``WalkBatch.set_bank`` / ``sweep(..., bank=...)``), or for one
(p, q) pair through ``compute_delta_against_constant``.
"""

from __future__ import annotations

import math
from typing import Any, Dict, List, Sequence, Tuple

# (name, sympy expression, description); zeta(2) .. zeta(30), pi variants and
# classical constants, in the reference's order
_ZETA = [(f"zeta{k}", f"zeta({k})", f"zeta({k})") for k in range(2, 31)]
CONSTANTS_REGISTRY: List[Dict[str, str]] = [
    {"name": n, "sympy_expr": e, "description": d} for n, e, d in _ZETA + [
        ("pi", "pi", "pi"),
        ("pi2", "pi**2", "pi^2"),
        ("pi_sq6", "pi**2/6", "pi^2/6 = zeta(2)"),
        ("1/pi", "1/pi", "1/pi"),
        ("4/pi", "4/pi", "4/pi"),
        ("catalan", "catalan", "Catalan's constant G"),
        ("euler_gamma", "EulerGamma", "Euler-Mascheroni gamma"),
        ("ln2", "log(2)", "ln(2)"),
        ("e", "E", "Euler's number e"),
        ("sqrt2", "sqrt(2)", "sqrt(2)"),
        ("phi", "(1+sqrt(5))/2", "golden ratio"),
    ]]


def load_constants(dps: int = 200) -> List[Dict[str, Any]]:
    """Every registry constant at ``dps`` digits: dicts with name, value (mpf),
    value_float, sympy_expr, description (reference constants.py:70-106)."""
    import sys
    if hasattr(sys, "set_int_max_str_digits"):
        sys.set_int_max_str_digits(max(sys.get_int_max_str_digits(), dps * 4))
    import mpmath as mp
    import sympy as sp
    mp.mp.dps = dps
    ns = {"pi": sp.pi, "E": sp.E, "zeta": sp.zeta, "catalan": sp.Catalan,
          "EulerGamma": sp.EulerGamma, "log": sp.log, "sqrt": sp.sqrt}
    out = []
    for entry in CONSTANTS_REGISTRY:
        try:
            expr = sp.sympify(entry["sympy_expr"], locals=ns)
            v = mp.mpf(str(sp.N(expr, dps + 10)))
        except Exception as exc:  # noqa: BLE001 - reported and skipped, as the reference
            print(f"WARNING: Could not evaluate constant '{entry['name']}': {exc}")
            continue
        out.append({"name": entry["name"], "value": v, "value_float": float(v),
                    "sympy_expr": entry["sympy_expr"], "description": entry["description"]})
    return out


def compute_match_digits(estimate: float, constants: Sequence[Dict[str, Any]]) -> Tuple[str, float]:
    """Best-matching constant by digits of agreement (reference
    constants.py:109-156): ratio matching of the tails when both the estimate
    and the constant are within 0.5 of 1, relative error otherwise."""
    near_one = abs(estimate - 1.0) < 0.5
    best_name, best = "none", -1.0
    for c in constants:
        cv = c["value_float"]
        if near_one and abs(cv - 1.0) < 0.5:
            te, tc = estimate - 1.0, cv - 1.0
            if abs(tc) < 1e-300:
                continue
            err = abs(te - tc)
            digits = 16.0 if err == 0 else -math.log10(err / max(abs(tc), 1e-300))
        else:
            err = abs(estimate - cv)
            if err == 0:
                digits = 16.0
            elif abs(cv) > 1e-300:
                digits = -math.log10(err / max(abs(cv), 1e-300))
            else:
                digits = 0.0
        if digits > best:
            best, best_name = digits, c["name"]
    return best_name, max(best, 0.0)


def match_against_constants(estimate: float, constants: Sequence[Dict[str, Any]],
                            proximity_threshold: float = 1e-3) -> List[Dict[str, Any]]:
    """Constants within ``proximity_threshold`` of the estimate, nearest first
    (reference constants.py:159-179)."""
    m = [{"name": c["name"], "distance": abs(estimate - c["value_float"]),
          "value_float": c["value_float"], "description": c["description"]}
         for c in constants if abs(estimate - c["value_float"]) < proximity_threshold]
    m.sort(key=lambda x: x["distance"])
    return m


def bank_ratios(constants: Sequence[Dict[str, Any]]) -> List[Tuple[int, int]]:
    """Exact (num, den) of each constant's mpf value: the targets the device
    bank scores against (den a power of two)."""
    out = []
    for c in constants:
        sign, man, exp, _ = c["value"]._mpf_
        num = -int(man) if sign else int(man)
        out.append((num << exp, 1) if exp >= 0 else (num, 1 << (-exp)))
    return out


def compute_delta_against_constant(p_big: int, q_big: int, constant_mp, dps: int = 200) -> float:
    """Dreams delta of p/q against one constant (reference constants.py:182-207),
    computed exactly on the GPU from the constant's mpf value at ``dps``."""
    import mpmath as mp
    from .runner import delta_batch
    mp.mp.dps = dps
    v = mp.mpf(constant_mp)
    sign, man, exp, _ = v._mpf_
    num = -int(man) if sign else int(man)
    tgt = (num << exp, 1) if exp >= 0 else (num, 1 << (-exp))
    return delta_batch([int(p_big)], [int(q_big)], [tgt])[0]
