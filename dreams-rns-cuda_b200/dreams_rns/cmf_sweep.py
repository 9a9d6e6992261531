"""Batched CMF sweep front-end (reference python/a100_sweep.py:336-528).

Every (CMF spec, trajectory) pair is compiled once; all its shifts, and the
pairs that follow, go to the engine in large batches.  On the device each
batch runs the walks, reconstructs p and q by CRT, flags CRT overflow and
scores every walk's p/q against every bank constant; the host then applies
the reference's hit rule per walk:

- est = p_float / q_float (walks with a non-finite estimate are skipped);
- the CRT is trusted when q != 0, p and q convert to finite floats and their
  ratio agrees with est to 1% (a100_sweep.py:445-460);
- proximity matches: constants within ``proximity`` of est; the candidates
  are those, or every constant within 1.0 of est when there are none;
- each candidate's delta is the exact one (device) when the CRT is trusted,
  else the float estimate -(1 + ln|est - c| / ln|q|);
- a hit has a positive best delta or a proximity match.
"""

from __future__ import annotations

import math
import time
from typing import Any, Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _native as N
from .cmf_walk import compile_cmf_spec, shift_to_axis_offsets
from .constants import load_constants, match_against_constants
from .engine import WalkBatch, cmf_request

__all__ = ["run_cmf_sweep"]


def _bit_lengths(limbs: np.ndarray) -> np.ndarray:
    """Bit length of each row of little-endian uint32 limbs."""
    nz = limbs != 0
    top = np.where(nz.any(axis=1), limbs.shape[1] - 1 - np.argmax(nz[:, ::-1], axis=1), -1)
    out = np.zeros(limbs.shape[0], dtype=np.int64)
    ok = top >= 0
    hi = limbs[np.arange(limbs.shape[0])[ok], top[ok]].astype(np.float64)
    out[ok] = 32 * top[ok] + np.floor(np.log2(hi)).astype(np.int64) + 1
    return out


def _limbs_int(row: np.ndarray, sign: int) -> int:
    v = int.from_bytes(np.ascontiguousarray(row, dtype=np.uint32).tobytes(), "little")
    return -v if sign < 0 else v


def run_cmf_sweep(specs: Sequence[Dict[str, Any]], trajectories: Sequence[Sequence[int]],
                  shifts: Sequence[Dict[str, Any]], depth: int, K: int = 0,
                  constants: Optional[List[Dict[str, Any]]] = None, proximity: float = 1e-3,
                  dps: int = 200, batch_walks: int = 32768) -> Tuple[list, List[dict], dict]:
    """All specs x trajectories x shifts; returns ([], hits, stats) as the
    reference's run_cmf_sweep_mode.  K = 0 uses the reference's default 1000."""
    K = K if K > 0 else 1000
    constants = constants if constants is not None else load_constants(dps)
    names = [c["name"] for c in constants]
    cval = np.array([c["value_float"] for c in constants])
    primes = [int(p) for p in N.prime_table(K)]
    p_bits = math.prod(primes).bit_length()
    hits: List[dict] = []
    run_count = 0
    t0 = time.time()
    pending: List[Tuple[dict, int, list, int, list]] = []   # (spec, traj_idx, traj, shift_idx, offsets)
    reqs = []

    def flush():
        nonlocal run_count
        if not reqs:
            return
        b = WalkBatch(reqs)
        try:
            b.set_pipeline(crt=True)
            b.set_bank(constants)
            b.run()
            arr = b.read_arrays()
            stride = (31 * K + 31) // 32 + 2
            limbs = np.zeros((4 * len(reqs), stride), dtype=np.uint32)
            signs = np.zeros(4 * len(reqs), dtype=np.int32)
            N.check(N.lib().dr_batch_read_pipeline(b.handle, None, None, None, N.ptr(limbs),
                                                  N.ptr(signs), stride), "dr_batch_read_pipeline")
            bank = b.read_bank()["bank_delta"]
        finally:
            b.close()
        bits = _bit_lengths(limbs)
        for w, (spec, ti, traj, si, offs) in enumerate(pending):
            run_count += 1
            pf, qf, ls = arr["shadow"][w]
            est = pf / qf if abs(qf) > 1e-300 else float("nan")
            if not math.isfinite(est):
                continue
            sp_, sq = int(signs[4 * w]), int(signs[4 * w + 1])
            crt_ok = sq != 0 and bits[4 * w] <= 1024 and bits[4 * w + 1] <= 1024
            if crt_ok:
                try:
                    cr = float(_limbs_int(limbs[4 * w], sp_)) / float(_limbs_int(limbs[4 * w + 1], sq))
                    crt_ok = math.isfinite(cr) and ((abs(cr - est) / abs(est) < 0.01) if abs(est) > 1e-10
                                                    else abs(cr - est) < 0.01)
                except (OverflowError, ZeroDivisionError):
                    crt_ok = False
            prox = match_against_constants(est, constants, proximity)
            log_q = ls + (math.log(abs(qf)) if abs(qf) > 1e-300 else 0.0)
            if prox:
                cand = [names.index(m["name"]) for m in prox]
            else:
                cand = [j for j in range(len(constants)) if abs(est - cval[j]) < 1.0]
            best, best_c = float("-inf"), None
            for j in cand:
                if crt_ok:
                    d = float(bank[w][j])
                else:
                    err = abs(est - cval[j])
                    d = -(1.0 + math.log(err) / log_q) if err > 0 and log_q > 0 else float("-inf")
                if d > best:
                    best, best_c = d, names[j]
            if best > 0 or prox:
                hits.append({"cmf_name": spec.get("name", ""), "spec_hash": spec.get("spec_hash", ""),
                             "rank": spec.get("rank", 2), "traj_idx": ti, "traj": list(traj),
                             "shift_idx": si, "shift_offsets": offs, "est_float": est,
                             "best_const": best_c, "best_delta": best, "p_bits": p_bits,
                             "proximity_matches": [m["name"] for m in prox],
                             "delta_positive": best > 0})
        reqs.clear()
        pending.clear()

    for ci, spec in enumerate(specs):
        spec = dict(spec, name=spec.get("name", f"CMF_{ci}"))
        dim = spec.get("dim", spec["p"] + spec["q"])
        offsets = []
        for sh in shifts:
            so = shift_to_axis_offsets(sh, spec["p"])
            while len(so) < dim:
                so.append(1)
            offsets.append(so[:dim])
        for ti, traj in enumerate(trajectories):
            try:
                prog = compile_cmf_spec(spec, trajectory=list(traj))
            except Exception:  # noqa: BLE001 - the reference skips pairs that fail to compile
                prog = None
            if prog is None:
                run_count += len(offsets)
                continue
            blob = prog.serialize()
            for si, so in enumerate(offsets):
                reqs.append(cmf_request(blob, depth, K, so))
                pending.append((spec, ti, list(traj), si, so))
                if len(reqs) >= batch_walks:
                    flush()
    flush()
    return [], hits, {"total_runs": run_count, "total_hits": len(hits), "elapsed_s": time.time() - t0}
