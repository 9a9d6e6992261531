"""ctypes wrapper of the C oracle ``walk_oracle.c`` (test infrastructure only)."""

from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

import numpy as np

from . import build as _build
from .walk_np import _rationals, parse_blob, primes

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = _build.LIB
        if not os.path.exists(path):
            path = _build.build()
        L = ctypes.CDLL(path)
        L.oracle_walk_mt.restype = ctypes.c_int
        L.oracle_walk_mt.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_int,
                                     ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                     ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_int]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def default_threads() -> int:
    """Host threads for the prime walks: every core this process may use."""
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except (AttributeError, OSError):
        return max(1, os.cpu_count() or 1)


def walk(blob: bytes, depth: int, K: int, axis: np.ndarray, init: np.ndarray,
         prow: int, qrow: int, shadow: bool = True, threads: Optional[int] = None):
    """Residues of P[prow][m-1], P[qrow][m-1] after ``depth`` steps (+ shadow).
    The K prime walks run on ``threads`` host threads (default: all cores);
    the result does not depend on the thread count."""
    pp = primes(K).astype(np.uint32)
    p_out = np.zeros(K, dtype=np.uint32)
    q_out = np.zeros(K, dtype=np.uint32)
    sh = np.zeros(3, dtype=np.float64)
    axis = np.ascontiguousarray(axis, dtype=np.int64)
    init = np.ascontiguousarray(init, dtype=np.int64)
    nt = default_threads() if threads is None else int(threads)
    rc = lib().oracle_walk_mt(blob, len(blob), K, _ptr(pp), int(depth), _ptr(axis), _ptr(init),
                              prow, qrow, _ptr(p_out), _ptr(q_out), _ptr(sh) if shadow else None,
                              nt)
    if rc:
        raise ValueError(f"oracle_walk failed ({rc})")
    return {"p_residues": p_out.astype(np.int64), "q_residues": q_out.astype(np.int64),
            "p_float": float(sh[0]), "q_float": float(sh[1]), "log_scale": float(sh[2]),
            "primes": pp.astype(np.int64)}


def pcf_walk(blob: bytes, a0: int, depth: int, K: int = 32, shift: int = 1,
             shadow: bool = True, threads: Optional[int] = None):
    """Same outputs as ``walk_np.pcf_walk`` (reference runner.py:338-413)."""
    m, dim, _, _, dirs = parse_blob(blob)
    axis = np.array([[shift, 1, d, 1] for d in dirs], dtype=np.int64).reshape(-1)
    init = np.array([[1, a0], [0, 1]], dtype=np.int64)
    return walk(blob, depth, K, axis, init, 0, 1, shadow, threads)


def cmf_walk(blob: bytes, depth: int, K: int, shift_vals, trajectory_vals=None,
             shadow: bool = True, threads: Optional[int] = None):
    """Same outputs as ``walk_np.cmf_walk`` (reference cmf_walk.py:363-431)."""
    m, dim, _, _, dirs = parse_blob(blob)
    sn, sd = _rationals(shift_vals)
    if trajectory_vals is not None:
        tn, td = _rationals(trajectory_vals)
    else:
        tn, td = list(dirs), [1] * len(dirs)
    axis = np.array([[sn[a], sd[a], tn[a], td[a]] for a in range(dim)],
                    dtype=np.int64).reshape(-1)
    init = np.eye(m, dtype=np.int64)
    return walk(blob, depth, K, axis, init, 0, m - 1, shadow, threads)
