"""Batched GPU walk API (reference python/dreams_rns/gpu_walk.py), on the B200 engine.

Same entry points and result dicts as the reference's CuPy module.  Two
behaviours differ on purpose: every walk gets its own FP64 shadow (the
reference reports the first walk's shadow for a whole batch,
gpu_walk.py:345-363), and INV runs on the device (the reference copies to the
host for it, gpu_walk.py:133-145).  ``batch_size`` is accepted for API
compatibility; the engine sizes its own device batches.
"""

from __future__ import annotations

from typing import Any, Dict, List, Optional

from . import _native as N
from .engine import cmf_request, pcf_request, run_walks

__all__ = ["gpu_available", "run_pcf_walk_gpu", "run_pcf_walk_batch_gpu", "run_cmf_walk_gpu",
           "run_cmf_walk_batch_gpu"]


def gpu_available() -> bool:
    """True when the native engine loads and binds to a CUDA device."""
    try:
        N.init()
        return True
    except Exception:  # noqa: BLE001 - probe
        return False


def _clean(r: dict) -> dict:
    import numpy as np
    return {"p_residues": r["p_residues"], "q_residues": r["q_residues"],
            "p_float": float(r["p_float"]), "q_float": float(r["q_float"]),
            "log_scale": float(r["log_scale"]), "primes": r["primes"]}


def run_pcf_walk_batch_gpu(program, a0: int, depth: int, K: int = 32,
                           shift_vals: Optional[List[int]] = None,
                           batch_size: int = 256) -> List[Dict[str, Any]]:
    """One PCF program walked from several integer shifts (gpu_walk.py:279-379)."""
    assert program.m == 2, "GPU walk only supports 2×2 companion matrices"
    shifts = shift_vals if shift_vals is not None else [1]
    reqs = [pcf_request(program, a0, max(int(depth), 0), int(K), int(s)) for s in shifts]
    out = []
    for s, r in zip(shifts, run_walks(reqs)):
        d = _clean(r)
        d["shift_val"] = s
        out.append(d)
    return out


def run_pcf_walk_gpu(program, a0: int, depth: int, K: int = 32, shift_val: int = 1) -> Dict[str, Any]:
    return run_pcf_walk_batch_gpu(program, a0, depth, K, [shift_val])[0]


def run_cmf_walk_batch_gpu(program, depth: int, K: int = 32,
                           shift_val_list: Optional[List[List[int]]] = None,
                           batch_size: int = 128) -> List[Dict[str, Any]]:
    """One CMF program from several integer shift vectors (gpu_walk.py:395-489):
    axis i at step t is shift[i] + t * directions[i], P0 = I."""
    if shift_val_list is None:
        shift_val_list = [[1] * program.dim]
    reqs = [cmf_request(program, max(int(depth), 0), int(K), list(sv), None) for sv in shift_val_list]
    out = []
    for sv, r in zip(shift_val_list, run_walks(reqs)):
        d = _clean(r)
        d["shift_vals"] = list(sv)
        out.append(d)
    return out


def run_cmf_walk_gpu(program, depth: int, K: int, shift_vals: List[int]) -> Dict[str, Any]:
    return run_cmf_walk_batch_gpu(program, depth, K, [shift_vals])[0]
