"""Batched walk execution on the B200 engine (host side of the C ABI).

A :class:`WalkRequest` describes one walk; :func:`run_walks` runs a list of
them in one engine call (host buffers in, host results out) and
:class:`WalkBatch` keeps a prepared batch resident on the device so the same
walks can be re-run with no host work (CUDA-graph replay).
"""

from __future__ import annotations

import collections
import ctypes
import threading
import time
from dataclasses import dataclass, field
from fractions import Fraction
from typing import Dict, Iterable, Iterator, List, Optional, Sequence, Tuple

import numpy as np

from . import _native as N
from .compiler import CmfProgram

__all__ = ["WalkRequest", "pcf_request", "cmf_request", "run_walks", "WalkBatch", "program_blob",
           "stage_times"]


def program_blob(program) -> bytes:
    if isinstance(program, (bytes, bytearray)):
        return bytes(program)
    if isinstance(program, CmfProgram):
        return program.serialize()
    if hasattr(program, "serialize"):
        return program.serialize()
    raise TypeError("program must be a CmfProgram or its serialized bytes")


def _directions(blob: bytes) -> List[int]:
    m, dim, n_ops, n_consts = np.frombuffer(blob[:16], dtype="<u4")
    off = 16 + 16 * int(n_ops) + 8 * int(n_consts)
    return [int(v) for v in np.frombuffer(blob[off:off + 4 * int(dim)], dtype="<i4")]


def _dims(blob: bytes) -> Tuple[int, int]:
    m, dim = np.frombuffer(blob[:8], dtype="<u4")
    return int(m), int(dim)


def _rational(v) -> Tuple[int, int]:
    """cmf_walk.py:332-345: int, Fraction or (num, den)."""
    if isinstance(v, Fraction):
        return v.numerator, v.denominator
    if isinstance(v, (tuple, list)):
        return int(v[0]), int(v[1])
    return int(v), 1


@dataclass(slots=True)
class WalkRequest:
    blob: bytes
    K: int
    depth: int
    axis: List[Tuple[int, int, int, int]]   # per program axis: (sn, sd, tn, td)
    a0: int = 0
    pcf_init: bool = False
    q_row: int = 1
    checkpoint: int = 0
    shadow: bool = True
    tag: dict = field(default_factory=dict)
    p_row: int = 0
    vec: Optional[List[int]] = None     # state-vector walk: v(0) residues then float bits


def pcf_request(program, a0: int, depth: int, K: int = 32, shift_val: int = 1,
                checkpoint: int = 0, shadow: bool = True) -> WalkRequest:
    """PCF walk: P0 = [[1, a0], [0, 1]], LOAD_X = shift + step * direction
    (reference runner.py:338-413)."""
    blob = program_blob(program)
    dirs = _directions(blob)
    return WalkRequest(blob=blob, K=K, depth=depth, a0=int(a0), pcf_init=True, q_row=1,
                       axis=[(int(shift_val), 1, d, 1) for d in dirs], checkpoint=checkpoint,
                       shadow=shadow)


def vec_request(program, depth: int, K: int, shift_vals, initial_state, acc_idx: int,
                const_idx: int, trajectory_vals=None, shadow: bool = True) -> WalkRequest:
    """State-vector walk v(N) = M(N-1) ... M(0) v(0) with p = v[acc_idx],
    q = v[const_idx] (reference cmf_walk.py:445-531).  v(0) entries are
    rationals: their residues per prime are num * den^(p-2) mod p, as the
    reference computes them (a denominator divisible by p gives 0)."""
    from fractions import Fraction
    req = cmf_request(program, depth, K, shift_vals, trajectory_vals, shadow=shadow)
    m = req.q_row + 1
    if len(initial_state) < m:
        raise IndexError("initial_state has fewer entries than the matrix size")
    if not (0 <= acc_idx < m and 0 <= const_idx < m):
        raise IndexError("acc_idx / const_idx outside the state vector")
    primes = [int(p) for p in N.prime_table(K)]
    res: List[int] = []
    fl = []
    for i in range(m):
        f = Fraction(initial_state[i])
        fl.append(float(f))
        if f == 0:
            res.extend([0] * K)
            continue
        num, den = f.numerator, f.denominator
        for p in primes:
            n = num % p
            res.append(n if den == 1 else n * pow(den, p - 2, p) % p)
    bits = np.array(fl, dtype=np.float64).view(np.int64)
    req.vec = res + [int(b) for b in bits]
    req.p_row = int(acc_idx)
    req.q_row = int(const_idx)
    req.pcf_init = False
    return req


def cmf_request(program, depth: int, K: int, shift_vals, trajectory_vals=None,
                checkpoint: int = 0, shadow: bool = True) -> WalkRequest:
    """CMF walk: P0 = I, rational per-axis shift/trajectory, q = P[m-1][m-1]
    (reference cmf_walk.py:363-431)."""
    blob = program_blob(program)
    m, dim = _dims(blob)
    sh = [_rational(v) for v in shift_vals]
    if trajectory_vals is not None:
        tr = [_rational(v) for v in trajectory_vals]
    else:
        tr = [(d, 1) for d in _directions(blob)]
    if len(sh) < dim or len(tr) < dim:
        raise IndexError("fewer shift/trajectory values than program axes")
    return WalkRequest(blob=blob, K=K, depth=depth, pcf_init=False, q_row=m - 1,
                       axis=[(sh[a][0], sh[a][1], tr[a][0], tr[a][1]) for a in range(dim)],
                       checkpoint=checkpoint, shadow=shadow)


try:
    from . import _pack as _pack_ext
except ImportError:        # not built: _pack_py below computes the same arrays
    _pack_ext = None


def _pack_py(reqs: Sequence[WalkRequest]):
    """Flat C-ABI arrays for a list of requests (the pure-Python statement of
    csrc/pack.c, which _Packed uses when built): (n_programs, offsets, blobs,
    desc, res_off, cp_off, axis, n_axis, n_res) with the arrays as bytearrays."""
    n = len(reqs)
    index: Dict[bytes, int] = {}
    blobs: List[bytes] = []
    flat: List[int] = []                 # 10 scalars per request
    axis_vals: List[int] = []
    vec_vals: List[int] = []
    put_row, put_axis = flat.extend, axis_vals.extend
    f_init, f_shadow, f_vec = N.DR_WALK_INIT_PCF, N.DR_WALK_SHADOW, N.DR_WALK_VEC
    for r in reqs:
        b = r.blob
        j = index.get(b)
        if j is None:
            j = index[b] = len(blobs)
            blobs.append(b)
        ax = r.axis
        for t in ax:
            put_axis(t)
        v = r.vec
        if r.depth < 0:          # the reference treats a negative depth as no steps
            r.depth = 0
        put_row((j, r.K, r.depth, r.checkpoint, r.a0,
                 (f_init if r.pcf_init else 0) | (f_shadow if r.shadow else 0) | (f_vec if v is not None else 0),
                 r.q_row, r.p_row, 4 * len(ax), 0 if v is None else len(v)))
        if v is not None:
            vec_vals.extend(v)
    n_programs = len(blobs)
    offs = np.zeros(len(blobs) + 1, dtype=np.uint64)
    np.cumsum(np.fromiter(map(len, blobs), dtype=np.uint64, count=len(blobs)), out=offs[1:])
    blob = bytearray(b"".join(blobs) or b"\0")
    try:
        cols = np.fromiter(flat, dtype=np.int64, count=len(flat)).reshape(n, 10)
    except OverflowError:
        if any(not -2**63 <= int(r.a0) < 2**63 for r in reqs):
            raise OverflowError("a0 outside int64") from None
        raise
    prog, Ks, depth, cps, a0, flags, q_row, p_row, alen, vlen = cols.T
    if n and (Ks.min() < 1 or Ks.max() > N.DR_MAX_K):
        raise ValueError(f"K must be in 1..{N.DR_MAX_K}")
    if n and cps.min() < 0:
        raise OverflowError("negative checkpoint")
    try:
        axis = np.array(axis_vals + vec_vals, dtype=np.int64)
    except OverflowError:
        raise OverflowError("axis parameter outside int64") from None
    sizes = Ks + np.where(cps > 0, Ks, 0)
    res_off = np.zeros(n, dtype=np.int64)
    if n:
        np.cumsum(sizes[:-1], out=res_off[1:])
    desc = np.zeros(n, dtype=N.WALK_DTYPE)
    desc["program"] = prog
    desc["K"] = Ks
    desc["depth"] = depth
    desc["checkpoint"] = cps
    desc["a0"] = a0
    desc["flags"] = flags
    desc["q_row"] = q_row
    desc["p_row"] = p_row
    a_total = int(alen.sum()) if n else 0
    n_axis = int(axis.size)
    voff = np.zeros(n, dtype=np.int64)
    if n:
        np.cumsum(vlen[:-1], out=voff[1:])
    desc["vec_offset"] = np.where(vlen > 0, voff + a_total, 0)
    aoff = np.zeros(n, dtype=np.int64)
    if n:
        np.cumsum(alen[:-1], out=aoff[1:])
    desc["axis_offset"] = aoff
    desc["res_offset"] = res_off
    cp_off = np.where(cps > 0, res_off + Ks, -1)
    desc["cp_res_offset"] = np.where(cps > 0, cp_off, 0)
    if not axis.size:
        axis = np.zeros(1, dtype=np.int64)
    return (n_programs, bytearray(offs.tobytes()), blob, bytearray(desc.tobytes()),
            bytearray(res_off.tobytes()), bytearray(cp_off.astype(np.int64).tobytes()),
            bytearray(axis.tobytes()), n_axis, max(int(sizes.sum()) if n else 0, 1))


class _Packed:
    """Flat C-ABI arrays for a list of requests: the blobs of the distinct
    programs with their offsets, one dr_walk_desc per request, the axis
    parameters (then state-vector entries) and the residue offsets."""

    def __init__(self, reqs: Sequence[WalkRequest]):
        global _pack_ms, _pack_calls
        t0 = time.perf_counter()
        n = len(reqs)
        packed = _pack_ext.pack(reqs) if _pack_ext is not None else _pack_py(reqs)
        self.n_programs, off, blob, desc, res, cp, axis, self.n_axis, self.n_res = packed
        self.offsets = np.frombuffer(off, dtype=np.uint64)
        self.blobs = np.frombuffer(blob, dtype=np.uint8)
        self.desc = np.frombuffer(desc, dtype=N.WALK_DTYPE)[:n]
        self.res_off = np.frombuffer(res, dtype=np.int64)[:n]
        self.cp_off = np.frombuffer(cp, dtype=np.int64)[:n]
        self.axis = np.frombuffer(axis, dtype=np.int64)
        self.n = n
        with _pack_lock:
            _pack_ms += (time.perf_counter() - t0) * 1e3
            _pack_calls += 1


_pack_ms = 0.0
_pack_calls = 0
_pack_lock = threading.Lock()
_STAGES = ("build", "upload", "run", "read", "device")


def stage_times(reset: bool = False) -> dict:
    """Milliseconds spent per stage of the engine calls since the last reset:
    request packing (host, this module), then the C ABI's batch build,
    allocation + upload, run, read-back and the device time of the runs read
    back (dr_stage_times), each with its number of calls."""
    global _pack_ms, _pack_calls
    ms = np.zeros(len(_STAGES), dtype=np.float64)
    calls = np.zeros(len(_STAGES), dtype=np.uint64)
    N.check(N.lib().dr_stage_times(N.ptr(ms), N.ptr(calls), len(_STAGES), 1 if reset else 0),
            "dr_stage_times")
    with _pack_lock:
        out = {"pack_ms": _pack_ms, "pack_calls": _pack_calls}
        if reset:
            _pack_ms, _pack_calls = 0.0, 0
    for i, s in enumerate(_STAGES):
        out[f"{s}_ms"] = float(ms[i])
        out[f"{s}_calls"] = int(calls[i])
    return out


def _tune(chunk_steps=0, engine=N.DR_ENGINE_AUTO, warps_per_block=0, shadow_buffer_mb=0,
          chain_pack_depth=0):
    t = N.Tune()
    t.chunk_steps = chunk_steps
    t.engine = engine
    t.warps_per_block = warps_per_block
    t.shadow_buffer_mb = shadow_buffer_mb
    t.chain_pack_depth = chain_pack_depth
    return t


def _unpack(pk: _Packed, reqs, p, q, sh, st):
    out = []
    primes_cache: Dict[int, np.ndarray] = {}
    for i, r in enumerate(reqs):
        if r.K not in primes_cache:
            primes_cache[r.K] = N.prime_table(r.K).astype(np.int64)
        o = int(pk.res_off[i])
        d = {"p_residues": p[o:o + r.K].astype(np.int64), "q_residues": q[o:o + r.K].astype(np.int64),
             "p_float": float(sh[3 * i]), "q_float": float(sh[3 * i + 1]),
             "log_scale": float(sh[3 * i + 2]), "primes": primes_cache[r.K],
             "status": int(st[i])}
        if r.checkpoint:
            c = int(pk.cp_off[i])
            j = 3 * (pk.n + i)
            d["checkpoint"] = {"depth": r.checkpoint, "p_residues": p[c:c + r.K].astype(np.int64),
                               "q_residues": q[c:c + r.K].astype(np.int64), "p_float": float(sh[j]),
                               "q_float": float(sh[j + 1]), "log_scale": float(sh[j + 2])}
        out.append(d)
    return out


def run_walks(reqs: Sequence[WalkRequest], chunk_steps: int = 0,
              engine: int = N.DR_ENGINE_AUTO, shadow_buffer_mb: int = 0) -> List[dict]:
    """Run every request in one engine call; one result dict per request."""
    N.init()
    reqs = list(reqs)
    if not reqs:
        return []
    pk = _Packed(reqs)
    p = np.zeros(pk.n_res, dtype=np.uint32)
    q = np.zeros(pk.n_res, dtype=np.uint32)
    sh = np.zeros(6 * pk.n, dtype=np.float64)
    st = np.zeros(pk.n, dtype=np.uint32)
    t = _tune(chunk_steps, engine, 0, shadow_buffer_mb)
    N.check(N.lib().dr_walk_batch(N.ptr(pk.desc), pk.n, N.ptr(pk.blobs), N.ptr(pk.offsets),
                                  pk.n_programs, N.ptr(pk.axis), pk.n_axis, ctypes.byref(t),
                                  N.ptr(p), N.ptr(q), pk.n_res, N.ptr(sh), N.ptr(st)),
            "dr_walk_batch")
    return _unpack(pk, reqs, p, q, sh, st)


def sweep(reqs: Sequence[WalkRequest], delta: Optional[str] = None,
          target: Optional[Tuple[int, int]] = None, topk: int = 0, values: bool = False,
          chunk_steps: int = 0, bank=None) -> dict:
    """One call for a sweep of many walks: walk every request, then on the
    device reconstruct p and q by CRT, score the Dreams delta (``delta="fixed"``
    against ``target`` = (Lnum, Lden), or ``"self"``: each walk's checkpoint
    convergent against its own final one) and select the ``topk`` best.

    Returns arrays (see ``WalkBatch.read_arrays``) plus ``delta``, ``topk_idx``,
    ``topk_val`` and, with ``values``, the centred p, q (and checkpoint p, q) as
    Python ints.  With ``bank`` (constants from constants.load_constants) each
    top-k hit is also scored against every constant (``bank_delta``,
    ``bank_best``).  The batched counterpart of calling run_pcf_walk /
    run_cmf_walk, crt_reconstruct and compute_dreams_delta_exact per walk.
    """
    b = WalkBatch(reqs, chunk_steps=chunk_steps)
    try:
        piped = bool(delta) or topk > 0 or values
        if piped:
            b.set_pipeline(delta=delta, target=target, topk=topk)
        if bank:
            b.set_bank(bank)
        b.run()
        out = b.read_arrays()
        if piped:
            out.update(b.read_pipeline(values=values))
        if bank and topk > 0:
            out.update(b.read_bank())
        return out
    finally:
        b.close()


def sweep_many(batches: Iterable[Sequence[WalkRequest]], delta: Optional[str] = None,
               target: Optional[Tuple[int, int]] = None, topk: int = 0, values: bool = False,
               chunk_steps: int = 0, bank=None, lookahead: int = 2) -> Iterator[dict]:
    """sweep() over a sequence of request lists, yielding each list's result
    dict in order.  While the device walks one list, up to ``lookahead``
    threads pack, build and upload the next ones (the batch build runs in C
    with the GIL released), and every run goes to one stream of its own, so a
    long sweep is bound by the slower of the host and the device instead of
    their sum.  Results equal sweep()'s for each list."""
    from concurrent.futures import ThreadPoolExecutor
    N.init()
    lookahead = max(1, int(lookahead))
    piped = bool(delta) or topk > 0 or values
    stream = ctypes.c_void_p()
    N.check(N.lib().dr_stream_create(ctypes.byref(stream)), "dr_stream_create")

    def prepare(reqs):
        b = WalkBatch(reqs, chunk_steps=chunk_steps)
        try:
            if piped:
                b.set_pipeline(delta=delta, target=target, topk=topk)
            if bank:
                b.set_bank(bank)
            b.run(stream.value)
        except BaseException:
            b.close()
            raise
        return b

    def collect(b):
        try:
            out = b.read_arrays()
            if piped:
                out.update(b.read_pipeline(values=values))
            if bank and topk > 0:
                out.update(b.read_bank())
            return out
        finally:
            b.close()

    pool = ThreadPoolExecutor(max_workers=lookahead)
    pending: collections.deque = collections.deque()
    try:
        for reqs in batches:
            pending.append(pool.submit(prepare, list(reqs)))
            if len(pending) > lookahead:
                yield collect(pending.popleft().result())
        while pending:
            yield collect(pending.popleft().result())
    finally:
        # batches prepared but not collected (early close, or an error)
        while pending:
            f = pending.popleft()
            try:
                f.result().close()
            except Exception:  # noqa: BLE001 - its error was or will be raised elsewhere
                pass
        pool.shutdown(wait=True)
        N.lib().dr_stream_destroy(stream)


def autotune(reqs: Sequence[WalkRequest]) -> dict:
    """Time candidate launch shapes (depth-chunk length, warps per block) on
    these walks and remember the fastest for every later batch of the same
    workload shape.  Returns the choice and its time per run."""
    N.init()
    pk = _Packed(list(reqs))
    t = _tune()
    ms = ctypes.c_float()
    N.check(N.lib().dr_autotune(N.ptr(pk.desc), pk.n, N.ptr(pk.blobs), N.ptr(pk.offsets),
                                pk.n_programs, N.ptr(pk.axis), pk.n_axis, ctypes.byref(t),
                                ctypes.byref(ms)), "dr_autotune")
    return {"chunk_steps": t.chunk_steps, "warps_per_block": t.warps_per_block,
            "chain_pack_depth": t.chain_pack_depth, "ms": ms.value}


class WalkBatch:
    """A batch of walks prepared once and resident on the device."""

    def __init__(self, reqs: Sequence[WalkRequest], chunk_steps: int = 0,
                 engine: int = N.DR_ENGINE_AUTO, warps_per_block: int = 0, shadow_buffer_mb: int = 0,
                 chain_pack_depth: int = 0):
        N.init()
        self.reqs = list(reqs)
        self.pk = _Packed(self.reqs)
        t = _tune(chunk_steps, engine, warps_per_block, shadow_buffer_mb, chain_pack_depth)
        h = ctypes.c_int32(0)
        N.check(N.lib().dr_batch_create(N.ptr(self.pk.desc), self.pk.n, N.ptr(self.pk.blobs),
                                        N.ptr(self.pk.offsets), self.pk.n_programs,
                                        N.ptr(self.pk.axis), self.pk.n_axis, ctypes.byref(t),
                                        ctypes.byref(h)), "dr_batch_create")
        self.handle = h.value

    def run(self, stream: Optional[int] = None) -> None:
        """Enqueue one run on ``stream`` (a cudaStream_t as int; None = the engine's
        own stream).  Use a created stream: handle 0, the legacy default
        stream, also selects the engine's stream."""
        N.check(N.lib().dr_batch_run(self.handle, ctypes.c_void_p(stream) if stream else None),
                "dr_batch_run")

    def read(self) -> List[dict]:
        pk = self.pk
        p = np.zeros(pk.n_res, dtype=np.uint32)
        q = np.zeros(pk.n_res, dtype=np.uint32)
        sh = np.zeros(6 * pk.n, dtype=np.float64)
        st = np.zeros(pk.n, dtype=np.uint32)
        N.check(N.lib().dr_batch_read(self.handle, N.ptr(p), N.ptr(q), pk.n_res, N.ptr(sh), N.ptr(st)),
                "dr_batch_read")
        return _unpack(pk, self.reqs, p, q, sh, st)

    def read_arrays(self) -> dict:
        """Results as arrays, without per-walk dicts: residues of walk i at
        ``res_offset[i]`` (``K`` entries; the checkpoint's at ``cp_res_offset[i]``),
        shadows ``(n, 3)`` rows of (p_float, q_float, log_scale)."""
        pk = self.pk
        p = np.zeros(pk.n_res, dtype=np.uint32)
        q = np.zeros(pk.n_res, dtype=np.uint32)
        sh = np.zeros(6 * pk.n, dtype=np.float64)
        st = np.zeros(pk.n, dtype=np.uint32)
        N.check(N.lib().dr_batch_read(self.handle, N.ptr(p), N.ptr(q), pk.n_res, N.ptr(sh), N.ptr(st)),
                "dr_batch_read")
        return {"p_residues": p, "q_residues": q, "res_offset": pk.res_off,
                "cp_res_offset": pk.cp_off, "shadow": sh[:3 * pk.n].reshape(pk.n, 3),
                "checkpoint_shadow": sh[3 * pk.n:].reshape(pk.n, 3), "status": st}

    def set_pipeline(self, delta: Optional[str] = None, target: Optional[Tuple[int, int]] = None,
                     topk: int = 0, crt: bool = True) -> None:
        """Run CRT (and optionally delta and top-k) on the device after every walk.

        ``delta="fixed"`` scores each final convergent against ``target`` =
        (Lnum, Lden); ``delta="self"`` scores each checkpoint convergent against
        the walk's own final convergent (every walk needs a checkpoint).
        """
        pl = N.Pipeline()
        pl.crt = 1 if crt else 0
        pl.delta_mode = {None: N.DR_DELTA_NONE, "fixed": N.DR_DELTA_FIXED,
                         "self": N.DR_DELTA_SELF}[delta]
        pl.topk = int(topk)
        self._tgt = None
        if delta == "fixed":
            from .runner import int_to_limbs
            num, den = target
            if den <= 0:
                raise ValueError("target denominator must be positive")
            width = max(abs(num).bit_length(), den.bit_length(), 1)
            nl = (width + 31) // 32 + 1
            sgn, ln = int_to_limbs(int(num), nl)
            _, ld = int_to_limbs(int(den), nl)
            self._tgt = (ln, ld)
            pl.l_limbs = nl
            pl.lnum = ln.ctypes.data
            pl.lden = ld.ctypes.data
            pl.lnum_sign = sgn
        N.check(N.lib().dr_batch_set_pipeline(self.handle, ctypes.byref(pl)), "dr_batch_set_pipeline")
        self.pipeline = {"delta": delta, "topk": int(topk), "crt": crt}

    def read_pipeline(self, values: bool = False) -> dict:
        """Deltas, top-k and (with ``values``) the centred p, q as Python ints."""
        n = self.pk.n
        k = min(self.pipeline["topk"], n)
        delta = np.zeros(max(n, 1), dtype=np.float64)
        ti = np.zeros(max(k, 1), dtype=np.int32)
        tv = np.zeros(max(k, 1), dtype=np.float64)
        limbs = signs = None
        stride = 0
        if values:
            Kmax = int(self.pk.desc["K"].max()) if n else 1
            stride = (31 * Kmax + 31) // 32 + 2
            limbs = np.zeros((4 * n, stride), dtype=np.uint32)
            signs = np.zeros(4 * n, dtype=np.int32)
        N.check(N.lib().dr_batch_read_pipeline(
            self.handle, N.ptr(delta) if self.pipeline["delta"] else None,
            N.ptr(ti) if k else None, N.ptr(tv) if k else None,
            N.ptr(limbs) if values else None, N.ptr(signs) if values else None, stride),
            "dr_batch_read_pipeline")
        out = {"delta": delta[:n] if self.pipeline["delta"] else None,
               "topk_idx": ti[:k], "topk_val": tv[:k]}
        if values:
            from .runner import limbs_to_int
            vals = [limbs_to_int(limbs[i], int(signs[i])) for i in range(4 * n)]
            out["p"] = vals[0::4]
            out["q"] = vals[1::4]
            out["cp_p"] = vals[2::4]
            out["cp_q"] = vals[3::4]
        return out

    def set_bank(self, constants) -> None:
        """Score every top-k hit's final p/q against each constant (dicts from
        constants.load_constants) on the device after each run."""
        from .constants import bank_ratios
        from .runner import int_to_limbs
        self.bank = list(constants)
        if not self.bank:
            N.check(N.lib().dr_batch_set_bank(self.handle, 0, 0, None, None, None), "dr_batch_set_bank")
            return
        rat = bank_ratios(self.bank)
        width = max(max(abs(a).bit_length(), b.bit_length()) for a, b in rat)
        nl = (width + 31) // 32 + 1
        num = np.zeros((len(rat), nl), dtype=np.uint32)
        den = np.zeros((len(rat), nl), dtype=np.uint32)
        sg = np.zeros(len(rat), dtype=np.int32)
        for i, (a, b) in enumerate(rat):
            sg[i], num[i] = int_to_limbs(int(a), nl)
            _, den[i] = int_to_limbs(int(b), nl)
        N.check(N.lib().dr_batch_set_bank(self.handle, len(rat), nl, N.ptr(num), N.ptr(sg), N.ptr(den)),
                "dr_batch_set_bank")

    def read_bank(self) -> dict:
        """delta[hit][constant] for the top-k hits, and each hit's best match."""
        k = min(self.pipeline["topk"], self.pk.n)
        nb = len(self.bank)
        d = np.zeros(max(k * nb, 1), dtype=np.float64)
        N.check(N.lib().dr_batch_read_bank(self.handle, N.ptr(d), k * nb), "dr_batch_read_bank")
        d = d[:k * nb].reshape(k, nb)
        best = [self.bank[int(np.argmax(row))]["name"] if nb else None for row in d]
        return {"bank_delta": d, "bank_names": [c["name"] for c in self.bank], "bank_best": best}

    def stats(self) -> dict:
        ps, nt, nl, ms = ctypes.c_uint64(), ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_float()
        N.check(N.lib().dr_batch_stats(self.handle, ctypes.byref(ps), ctypes.byref(nt),
                                       ctypes.byref(nl), ctypes.byref(ms)), "dr_batch_stats")
        return {"prime_steps": ps.value, "tiles": nt.value, "launches": nl.value,
                "last_ms": ms.value}

    def profile(self) -> List[dict]:
        """Each launch group run alone and timed (kind 0 walk, 1 interpreted
        shadow, 2 integer-difference shadow)."""
        cap = 64
        n = ctypes.c_int32()
        arrs = [np.zeros(cap, dtype=np.int32) for _ in range(4)]
        items = np.zeros(cap, dtype=np.uint32)
        ms = np.zeros(cap, dtype=np.float32)
        ms2 = np.zeros(cap, dtype=np.float32)
        N.check(N.lib().dr_batch_profile(self.handle, cap, ctypes.byref(n), *[N.ptr(a) for a in arrs],
                                         N.ptr(items), N.ptr(ms), N.ptr(ms2)), "dr_batch_profile")
        return [{"kind": int(arrs[0][i]), "class": int(arrs[1][i]), "m": int(arrs[2][i]),
                 "degree": int(arrs[3][i]), "items": int(items[i]), "ms": float(ms[i]),
                 "ms2": float(ms2[i])} for i in range(min(n.value, cap))]

    def close(self) -> None:
        if self.handle:
            N.lib().dr_batch_destroy(self.handle)
            self.handle = 0

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass
